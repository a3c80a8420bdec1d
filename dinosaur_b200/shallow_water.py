"""Shallow-water equations on the GPU (dinosaur/shallow_water.py:121-230).

``ShallowWaterEquations`` keeps the reference's constructor and its
``ImplicitExplicitODE`` methods; each call runs the CUDA kernels of
``csrc/swe.cu`` through the C ABI on a packed
[vorticity][divergence][potential] buffer.  The steppers of
``dinosaur_b200.time_integration`` (``imex_rk_sil3``, ``step_with_filters``,
``repeated``) apply unchanged.
"""

from __future__ import annotations

import ctypes
import dataclasses
from typing import Any

import numpy as np
import torch

from dinosaur_b200 import _lib
from dinosaur_b200 import coordinate_systems
from dinosaur_b200 import pytree
from dinosaur_b200 import spherical_harmonic as sh
from dinosaur_b200 import time_integration
from dinosaur_b200 import units

Array = Any


def _binary(op):
  def f(self, other):
    if isinstance(other, State):
      return pytree.tree_map(op, self, other)
    return pytree.tree_map(lambda a: op(a, other), self)
  return f


@dataclasses.dataclass
class State:
  """State of the shallow-water equations (shallow_water.py:42-48)."""

  vorticity: Array
  divergence: Array
  potential: Array

  __add__ = _binary(lambda a, b: a + b)
  __sub__ = _binary(lambda a, b: a - b)
  __mul__ = _binary(lambda a, b: a * b)
  __rmul__ = _binary(lambda a, b: b * a)
  __truediv__ = _binary(lambda a, b: a / b)

  def __neg__(self):
    return pytree.tree_map(lambda a: -a, self)


ShallowWaterSpecs = units.SimUnits


def state_to_nodal(state: State, grid: sh.Grid) -> State:
  """shallow_water.py:57-59."""
  return pytree.tree_map(lambda x: grid.to_nodal(grid.clip_wavenumbers(x)), state)


def state_to_modal(state: State, grid: sh.Grid) -> State:
  """shallow_water.py:62-64."""
  return pytree.tree_map(grid.to_modal, state)


def get_density_ratios(density) -> np.ndarray:
  """shallow_water.py:67-86: D[i, j] = min(density[j] / density[i], 1), zero
  diagonal."""
  density = np.asarray(density)
  ratios = np.minimum(density / density[..., np.newaxis], 1)
  np.fill_diagonal(ratios, 0)
  return ratios


def get_coriolis(grid: sh.Grid) -> np.ndarray:
  """shallow_water.py:89-92."""
  _, sin_lat = grid.nodal_mesh
  return sin_lat


class _Engine:
  """A ``dino_swe`` for one member count."""

  def __init__(self, eq: 'ShallowWaterEquations', members: int):
    grid = eq.coords.horizontal
    self.grid = grid
    self.K = eq.coords.vertical.layers
    # Real modal layout inside; Fast-layout arrays are converted at the edges.
    self.M, self.L = 2 * grid.longitude_wavenumbers - 1, grid.total_wavenumbers
    self.members = members
    self._ref = np.ascontiguousarray(np.broadcast_to(
        np.asarray(eq.reference_potential, np.float64), (self.K,)))
    self._dens = np.ascontiguousarray(np.broadcast_to(
        np.asarray(eq.densities, np.float64), (self.K,)))
    orog = eq.orography
    if orog is not None and sh.is_fast_layout(grid):
      orog = sh.to_real_layout(grid, orog)
    if isinstance(orog, torch.Tensor):
      orog = orog.detach().cpu().numpy()
    self._orog = None if orog is None else np.ascontiguousarray(
        np.asarray(orog, np.float32).reshape(self.M, self.L))
    desc = _lib.SWEDesc(
        layers=self.K, members=members,
        reference_potential=_lib.dptr(self._ref),
        densities=_lib.dptr(self._dens),
        orography_modal=(None if self._orog is None else self._orog.ctypes.data_as(
            ctypes.POINTER(ctypes.c_float))),
        angular_velocity=eq.physics_specs.angular_velocity)
    self.plan = grid.plan
    handle = ctypes.c_void_p()
    _lib.check(_lib.lib().dino_swe_create(self.plan.handle, ctypes.byref(desc),
                                          ctypes.byref(handle)), 'dino_swe_create')
    self.handle = handle
    self.size = int(_lib.lib().dino_swe_state_size(handle))

  def __del__(self):
    h = getattr(self, 'handle', None)
    if h is not None and h.value:
      try:
        _lib.lib().dino_swe_destroy(h)
      except Exception:
        pass

  def pack(self, state: State) -> torch.Tensor:
    n = self.members * self.K
    parts = [sh.to_real_layout(self.grid, getattr(state, k)).reshape(n, self.M, self.L)
             for k in ('vorticity', 'divergence', 'potential')]
    return torch.cat(parts).reshape(-1).contiguous()

  def unpack(self, buf: torch.Tensor, like: State) -> State:
    n = self.members * self.K
    planes = buf.view(-1, self.M, self.L)
    shape = tuple(like.vorticity.shape)
    conv = lambda x: sh.from_real_layout(self.grid, x).view(shape)
    return State(conv(planes[0:n]), conv(planes[n:2 * n]), conv(planes[2 * n:]))

  def call(self, name, buf, *extra):
    out = torch.empty(self.size, device='cuda', dtype=torch.float32)
    fn = getattr(_lib.lib(), name)
    _lib.check(fn(self.handle, sh.ptr(buf), sh.ptr(out), *extra, sh.stream_handle()),
               name)
    return out


@dataclasses.dataclass(eq=False)
class ShallowWaterEquations(time_integration.ImplicitExplicitODE):
  """A semi-implicit description of the shallow-water equations
  (shallow_water.py:121-230)."""

  coords: coordinate_systems.CoordinateSystem
  physics_specs: Any
  orography: Array
  reference_potential: Array
  densities: Array = dataclasses.field(default_factory=lambda: np.ones((1,)))

  def __post_init__(self):
    self._engines = {}

  @property
  def coriolis_parameter(self):
    """2 Omega sin(lat) (shallow_water.py:142-146)."""
    _, sin_lat = self.coords.horizontal.nodal_mesh
    return 2 * self.physics_specs.angular_velocity * sin_lat

  @property
  def density_ratios(self):
    return get_density_ratios(self.densities)

  @property
  def ref_potential(self):
    return np.asarray(self.reference_potential)[..., np.newaxis, np.newaxis]

  def _engine(self, state: State) -> _Engine:
    K = self.coords.vertical.layers
    M, L = self.coords.horizontal.modal_shape  # in the grid's own layout
    shape = tuple(state.vorticity.shape)
    if shape[-3:] != (K, M, L) or len(shape) not in (3, 4):
      raise ValueError(f'expected state arrays of shape [members,] {(K, M, L)}; '
                       f'got {shape}')
    members = shape[0] if len(shape) == 4 else 1
    eng = self._engines.get(members)
    if eng is None:
      eng = _Engine(self, members)
      self._engines[members] = eng
    return eng

  def explicit_terms(self, state: State) -> State:
    """shallow_water.py:158-205."""
    eng = self._engine(state)
    return eng.unpack(eng.call('dino_swe_explicit', eng.pack(state)), state)

  def implicit_terms(self, state: State) -> State:
    """shallow_water.py:207-213."""
    eng = self._engine(state)
    return eng.unpack(eng.call('dino_swe_implicit', eng.pack(state)), state)

  def implicit_inverse(self, state: State, step_size: float) -> State:
    """shallow_water.py:215-230."""
    if isinstance(step_size, torch.Tensor):
      raise TypeError('`step_size` must be concrete')
    eng = self._engine(state)
    return eng.unpack(eng.call('dino_swe_implicit_inverse', eng.pack(state),
                               ctypes.c_double(float(step_size))), state)
