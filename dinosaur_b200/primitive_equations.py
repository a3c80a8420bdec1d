"""Primitive equations on sigma levels with CUDA explicit/implicit terms.

Mirrors the sigma-coordinate part of ``dinosaur/primitive_equations.py``
(reference v1.3.6): ``State`` (:61-84), ``validate_state_shape`` (:87-120),
the vertical weight matrices (:283-541, FP64 on the host exactly as the
reference builds them), ``truncated_modal_orography`` (:626-636) and
``PrimitiveEquationsSigma`` (:835-1458) with ``explicit_terms``,
``implicit_terms`` and ``implicit_inverse`` ('split' method).  The terms run
in ``libdino_b200`` on a packed state; ensemble members may be stacked on a
leading axis of every field.
"""

from __future__ import annotations

import ctypes
import dataclasses
import functools
from typing import Any, Mapping

import numpy as np
import torch

from dinosaur_b200 import _lib
from dinosaur_b200 import coordinate_systems
from dinosaur_b200 import hybrid_coordinates
from dinosaur_b200 import pytree
from dinosaur_b200 import sigma_coordinates
from dinosaur_b200 import spherical_harmonic as sh
from dinosaur_b200 import time_integration
from dinosaur_b200 import units

Array = Any


# ---------------------------------------------------------------------------
# State
# ---------------------------------------------------------------------------


def _binary(op):
  def f(self, other):
    if isinstance(other, State):
      return pytree.tree_map(lambda a, b: op(a, b) if a is not None else None,
                             self, other)
    return pytree.tree_map(lambda a: op(a, other) if a is not None else None,
                           self)
  return f


@dataclasses.dataclass
class State:
  """State of the primitive equations (primitive_equations.py:61-84)."""

  vorticity: Array
  divergence: Array
  temperature_variation: Array
  log_surface_pressure: Array
  tracers: Mapping[str, Array] = dataclasses.field(default_factory=dict)
  sim_time: float | None = None

  __add__ = _binary(lambda a, b: a + b)
  __sub__ = _binary(lambda a, b: a - b)
  __mul__ = _binary(lambda a, b: a * b)
  __rmul__ = _binary(lambda a, b: b * a)
  __truediv__ = _binary(lambda a, b: a / b)

  def __neg__(self):
    return pytree.tree_map(lambda a: -a, self)

  @property
  def fields(self):
    return dataclasses.fields(self)

  def asdict(self):
    return {f.name: getattr(self, f.name) for f in dataclasses.fields(self)
            if f.name != 'sim_time' or self.sim_time is not None}


class StateShapeError(Exception):
  """Exceptions for unexpected state shapes."""


def validate_state_shape(state: State,
                         coords: coordinate_systems.CoordinateSystem):
  """primitive_equations.py:87-120 (a leading member axis is allowed)."""
  def check(name, arr, expected):
    shape = tuple(arr.shape)
    if shape[-len(expected):] != tuple(expected) or len(shape) > len(expected) + 1:
      raise StateShapeError(f'Expected {name} shape {expected}; got shape {shape}.')
  check('vorticity', state.vorticity, coords.modal_shape)
  check('divergence', state.divergence, coords.modal_shape)
  check('temperature_variation', state.temperature_variation, coords.modal_shape)
  check('log_surface_pressure', state.log_surface_pressure,
        coords.surface_modal_shape)
  for name, arr in state.tracers.items():
    if tuple(arr.shape[-3:]) != tuple(coords.modal_shape):
      raise StateShapeError(f'Expected tracer {name} shape {coords.modal_shape}; '
                            f'got shape {tuple(arr.shape)}.')


# ---------------------------------------------------------------------------
# Vertical weights (host, FP64 with the reference's dtype behaviour)
# ---------------------------------------------------------------------------


def get_sigma_ratios(coordinates: sigma_coordinates.SigmaCoordinates):
  """Half log-sigma increments between level centres (primitive_equations.py:283-303).

  alpha_k = (ln sigma_{k+1} - ln sigma_k) / 2 for k < K - 1 and
  alpha_{K-1} = -ln sigma_{K-1}.  As in the reference, the logarithms are
  taken in the level centres' dtype (float32 for equidistant levels) and
  differenced in float64.
  """
  log_sigma = np.log(coordinates.centers)
  alpha = np.empty(log_sigma.shape, np.float64)
  alpha[:-1] = 0.5 * (log_sigma[1:].astype(np.float64) - log_sigma[:-1])
  alpha[-1] = -log_sigma[-1]
  return alpha


def get_geopotential_weights_sigma(coordinates, ideal_gas_constant):
  """G of the hydrostatic geopotential, Phi = Phi_s + G T (primitive_equations.py:306-338).

  Integrating d Phi = -R T d ln sigma upwards from the surface with
  midpoint weights gives, for level r and temperature level c:
    G[r, c] = R alpha_r                  (c = r)
    G[r, c] = R (alpha_c + alpha_{c-1})  (c > r, the levels below r)
    G[r, c] = 0                          (c < r).
  """
  alpha = get_sigma_ratios(coordinates)
  k = coordinates.layers
  r, c = np.indices((k, k))
  pair = alpha[c] + alpha[np.maximum(c - 1, 0)]
  weights = np.where(c == r, alpha[c], np.where(c > r, pair, 0.0))
  return ideal_gas_constant * weights


def get_temperature_implicit_weights_sigma(coordinates, reference_temperature,
                                           kappa):
  """H of the linearised temperature tendency, dT/dt = -H div (primitive_equations.py:419-502).

  Durran (2010) section 8.6.5: with the lower-triangular indicator
  [c <= r], the interface sigma_{r+1/2} = sum_{i <= r} dsigma_i and the
  centred reference-temperature gradient g_r = (T_{r+1} - T_r) /
  (dsigma_r + dsigma_{r+1}) (g_{K-1} = 0), entry (r, c) is dsigma_c times
    kappa T_r / dsigma_r (alpha_r [c <= r] + alpha_{r-1} [c <= r - 1])
    - g_r ([c <= r] - sigma_{r+1/2}) - g_{r-1} ([c <= r - 1] - sigma_{r-1/2}),
  the terms with index r - 1 absent on the top level.  The interface sums
  and the thickness pairs are formed in the thicknesses' dtype, as the
  reference does.
  """
  t_ref = np.asarray(reference_temperature)
  k = coordinates.layers
  if t_ref.ndim != 1 or t_ref.shape[-1] != k:
    raise ValueError(
        '`reference_temp` must be a vector of length `coordinates.layers`; '
        f'got shape {t_ref.shape} and {k} layers.')
  dsigma = coordinates.layer_thickness
  alpha = get_sigma_ratios(coordinates)
  interface = np.cumsum(dsigma)                   # sigma_{r+1/2}
  grad = np.zeros(k)
  grad[:-1] = np.diff(t_ref) / (dsigma[:-1] + dsigma[1:])
  r, c = np.indices((k, k))
  on = (c <= r).astype(np.float64)                # [c <= r]
  has_above = r >= 1
  ra = np.maximum(r - 1, 0)                       # index of the level above
  on_above = np.where(has_above, (c <= r - 1), 0.0)
  adiabatic = kappa * t_ref[r] * (alpha[r] * on + np.where(has_above, alpha[ra], 0.0)
                                  * on_above) / dsigma[r]
  advection = (grad[r] * (on - interface[r])
               + np.where(has_above, grad[ra] * (on_above - interface[ra]), 0.0))
  return (adiabatic - advection) * dsigma[c]


def truncated_modal_orography(orography, coords, wavenumbers_to_clip: int = 1):
  """primitive_equations.py:626-636."""
  grid = coords.horizontal
  if tuple(np.shape(orography)) != tuple(grid.nodal_shape):
    raise ValueError(f'Expected nodal orography with shape={grid.nodal_shape}')
  return grid.clip_wavenumbers(grid.to_modal(orography), n=wavenumbers_to_clip)


# ---------------------------------------------------------------------------
# Packed-state engine
# ---------------------------------------------------------------------------


class _Engine:
  """A ``dino_pe`` for one (members, tracer names) combination."""

  def __init__(self, eq: PrimitiveEquationsSigma, members: int,
               tracer_names: tuple[str, ...]):
    grid = eq.coords.horizontal
    vert = eq.coords.vertical
    ps = eq.physics_specs
    self.grid = grid
    self.members = members
    self.tracer_names = tracer_names
    self.K = vert.layers
    # The engine works in the Real modal layout; a Fast-layout grid's arrays
    # are converted in pack() / unpack().
    self.M, self.L = 2 * grid.longitude_wavenumbers - 1, grid.total_wavenumbers
    hum = -1
    if eq.humidity_key is not None:
      if eq.humidity_key not in tracer_names:
        raise ValueError(f'`{eq.humidity_key}` is not found in tracers: '
                         f'{tracer_names}.')
      hum = tracer_names.index(eq.humidity_key)
    K = self.K
    f64 = lambda x: np.ascontiguousarray(x, np.float64)
    hybrid = isinstance(eq, PrimitiveEquationsHybrid)
    # Host constants, kept alive for the duration of the create call.
    if not hybrid:
      self._arrays = dict(
          bounds=f64(vert.boundaries),
          centers=f64(vert.centers),
          thick=f64(vert.layer_thickness),
          inv_c2c=f64((1 / vert.center_to_center) if K > 1 else np.zeros(1)),
          tref=f64(eq.reference_temperature),
          G=f64(get_geopotential_weights_sigma(vert, ps.R)),
          H=f64(get_temperature_implicit_weights_sigma(
              vert, eq.reference_temperature, ps.kappa)),
          alpha=f64(get_sigma_ratios(vert)),
      )
    else:
      lev, psr = eq.nondim_levels, eq.p_s_ref
      # The implicit operator at p_s_ref (_get_implicit_term_matrix_hybrid,
      # primitive_equations.py:1890-1938); the sigma-only arrays are
      # placeholders of the right sizes.
      thick = lev.pressure_thickness / psr + lev.sigma_thickness
      self._arrays = dict(
          bounds=f64(lev.b_boundaries),
          centers=f64(lev.b_centers),
          thick=f64(thick),
          inv_c2c=f64(np.zeros(max(K - 1, 1))),
          tref=f64(eq.reference_temperature),
          G=f64(get_geopotential_weights_hybrid(lev, ps.R, psr)),
          H=f64(get_temperature_implicit_weights_hybrid(
              lev, eq.reference_temperature, ps.kappa, psr)),
          alpha=f64(np.zeros(K)),
          a_b=f64(lev.a_boundaries),
          b_b=f64(lev.b_boundaries),
          col=f64(pgf_lps_coefficient_hybrid(eq.reference_temperature, psr, lev,
                                             ps.R)),
          row=f64(thick),
      )
    orog = eq.orography
    if sh.is_fast_layout(grid):
      orog = sh.to_real_layout(grid, torch.as_tensor(np.asarray(orog, np.float32)
                                                     if not isinstance(orog, torch.Tensor)
                                                     else orog))
    if isinstance(orog, torch.Tensor):
      orog = orog.detach().cpu().numpy()
    self._orog = np.ascontiguousarray(np.asarray(orog, np.float32).reshape(
        self.M, self.L))
    a = self._arrays
    hs = eq.held_suarez
    desc = _lib.PEDesc(
        layers=K, members=members, n_tracers=len(tracer_names),
        humidity_tracer=hum,
        include_vertical_advection=int(eq.include_vertical_advection),
        held_suarez=int(hs is not None),
        sigma_boundaries=_lib.dptr(a['bounds']),
        sigma_centers=_lib.dptr(a['centers']),
        layer_thickness=_lib.dptr(a['thick']),
        inv_center_to_center=_lib.dptr(a['inv_c2c']),
        reference_temperature=_lib.dptr(a['tref']),
        geopotential_weights=_lib.dptr(a['G']),
        temperature_weights=_lib.dptr(a['H']),
        sigma_ratios=_lib.dptr(a['alpha']),
        orography_modal=self._orog.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
        angular_velocity=ps.angular_velocity, gravity=ps.g, R=ps.R,
        R_vapor=ps.R_vapor, Cp_vapor=ps.Cp_vapor, kappa=ps.kappa)
    if hybrid:
      desc.vertical_scheme = 1
      desc.hybrid_a_boundaries = _lib.dptr(a['a_b'])
      desc.hybrid_b_boundaries = _lib.dptr(a['b_b'])
      desc.reference_surface_pressure = eq.p_s_ref
      desc.implicit_lnps_column = _lib.dptr(a['col'])
      desc.implicit_thickness = _lib.dptr(a['row'])
    if hs is not None:
      desc.hs_p0 = hs.p0
      desc.hs_sigma_b = hs.sigma_b
      desc.hs_kf = hs.kf
      desc.hs_ka = hs.ka
      desc.hs_ks = hs.ks
      desc.hs_minT = hs.minT
      desc.hs_maxT = hs.maxT
      desc.hs_dTy = hs.dTy
      desc.hs_dThz = hs.dThz
    plan = grid.plan
    self.plan = plan  # keep the plan alive while the engine lives
    handle = ctypes.c_void_p()
    _lib.check(_lib.lib().dino_pe_create(plan.handle, ctypes.byref(desc),
                                         ctypes.byref(handle)), 'dino_pe_create')
    self.handle = handle
    self.size = int(_lib.lib().dino_pe_state_size(handle))
    self.plane = self.M * self.L

  def __del__(self):
    h = getattr(self, 'handle', None)
    if h is not None and h.value:
      try:
        _lib.lib().dino_pe_destroy(h)
      except Exception:
        pass

  # -- packing -------------------------------------------------------------
  def pack(self, state: State) -> torch.Tensor:
    mK = self.members * self.K
    real = lambda x: sh.to_real_layout(self.grid, x)
    parts = [real(state.vorticity).reshape(mK, self.M, self.L),
             real(state.divergence).reshape(mK, self.M, self.L),
             real(state.temperature_variation).reshape(mK, self.M, self.L)]
    for name in self.tracer_names:
      parts.append(real(state.tracers[name]).reshape(mK, self.M, self.L))
    parts.append(real(state.log_surface_pressure).reshape(
        self.members, self.M, self.L))
    buf = torch.cat(parts).reshape(-1).contiguous()
    assert buf.numel() == self.size
    return buf

  def unpack(self, buf: torch.Tensor, like: State, sim_time=None) -> State:
    mK = self.members * self.K
    planes = buf.view(-1, self.M, self.L)

    def leaf(p0, p1, like_leaf):
      shape = tuple(like_leaf.shape)
      x = planes[p0:p1]
      if sh.is_fast_layout(self.grid):
        return sh.from_real_layout(self.grid, x).view(shape)
      return x.view(shape)

    nT = len(self.tracer_names)
    out = State(
        vorticity=leaf(0, mK, like.vorticity),
        divergence=leaf(mK, 2 * mK, like.divergence),
        temperature_variation=leaf(2 * mK, 3 * mK, like.temperature_variation),
        log_surface_pressure=leaf((3 + nT) * mK, (3 + nT) * mK + self.members,
                                  like.log_surface_pressure),
        tracers={name: leaf((3 + t) * mK, (4 + t) * mK, like.tracers[name])
                 for t, name in enumerate(self.tracer_names)},
        sim_time=sim_time)
    return out

  # -- calls ---------------------------------------------------------------
  def _out(self):
    return torch.empty(self.size, device='cuda', dtype=torch.float32)

  def explicit(self, buf):
    out = self._out()
    _lib.check(_lib.lib().dino_pe_explicit(self.handle, sh.ptr(buf), sh.ptr(out),
                                           sh.stream_handle()), 'explicit_terms')
    return out

  def implicit(self, buf):
    out = self._out()
    _lib.check(_lib.lib().dino_pe_implicit(self.handle, sh.ptr(buf), sh.ptr(out),
                                           sh.stream_handle()), 'implicit_terms')
    return out

  def inverse(self, buf, eta):
    out = self._out()
    _lib.check(_lib.lib().dino_pe_implicit_inverse(
        self.handle, sh.ptr(buf), sh.ptr(out), float(eta), sh.stream_handle()),
               'implicit_inverse')
    return out

  def _filter_ptr(self, filt):
    if filt is None:
      return None
    self._filt = np.ascontiguousarray(filt, np.float64)
    if self._filt.shape != (self.L,):
      raise ValueError(f'filter scaling must have shape ({self.L},)')
    return _lib.dptr(self._filt)

  def trajectory_(self, buf, dt, filt, outer_steps, inner_steps, start_with_input):
    """Advances buf in place by outer_steps x inner_steps filtered steps and
    returns the (outer_steps, size) frames (dino_pe_trajectory)."""
    fptr = self._filter_ptr(filt)
    frames = torch.empty((outer_steps, self.size), device='cuda', dtype=torch.float32)
    _lib.check(_lib.lib().dino_pe_trajectory(
        self.handle, sh.ptr(buf), float(dt), fptr, int(outer_steps), int(inner_steps),
        int(bool(start_with_input)), sh.ptr(frames) if outer_steps else None,
        sh.stream_handle()), 'trajectory')
    return frames

  def unpack_frames(self, frames: torch.Tensor, like: State, sim_times=None) -> State:
    """The (frames, size) buffer as one State whose leaves lead with the frame
    axis."""
    n = frames.shape[0]
    per = [self.unpack(frames[i], like) for i in range(n)] if n else []
    stack = lambda xs, like_leaf: (torch.stack(xs) if xs else
                                   torch.empty((0,) + tuple(like_leaf.shape),
                                               device='cuda'))
    return State(
        vorticity=stack([p.vorticity for p in per], like.vorticity),
        divergence=stack([p.divergence for p in per], like.divergence),
        temperature_variation=stack([p.temperature_variation for p in per],
                                    like.temperature_variation),
        log_surface_pressure=stack([p.log_surface_pressure for p in per],
                                   like.log_surface_pressure),
        tracers={k: stack([p.tracers[k] for p in per], like.tracers[k])
                 for k in like.tracers},
        sim_time=sim_times)

  def step_(self, buf, dt, filt, n_steps, graph=False):
    fptr = self._filter_ptr(filt)
    fn = (_lib.lib().dino_pe_step_graph if graph else _lib.lib().dino_pe_step)
    _lib.check(fn(self.handle, sh.ptr(buf), float(dt), fptr, int(n_steps),
                  sh.stream_handle()), 'step')
    return buf

  # -- reverse mode ----------------------------------------------------------
  def explicit_vjp(self, buf, ct):
    out = self._out()
    _lib.check(_lib.lib().dino_pe_explicit_vjp(
        self.handle, sh.ptr(buf), sh.ptr(ct), sh.ptr(out), sh.stream_handle()),
               'explicit_terms vjp')
    return out

  def implicit_vjp(self, ct):
    out = self._out()
    _lib.check(_lib.lib().dino_pe_implicit_vjp(
        self.handle, sh.ptr(ct), sh.ptr(out), sh.stream_handle()),
               'implicit_terms vjp')
    return out

  def inverse_vjp(self, ct, eta):
    out = self._out()
    _lib.check(_lib.lib().dino_pe_implicit_inverse_vjp(
        self.handle, sh.ptr(ct), sh.ptr(out), float(eta), sh.stream_handle()),
               'implicit_inverse vjp')
    return out

  def step_vjp_(self, buf, ct, dt, filt):
    """Overwrites ct with the VJP of one filtered step taken from buf."""
    fptr = self._filter_ptr(filt)
    _lib.check(_lib.lib().dino_pe_step_vjp(
        self.handle, sh.ptr(buf), sh.ptr(ct), sh.ptr(ct), float(dt), fptr,
        sh.stream_handle()), 'step vjp')
    return ct


# ---------------------------------------------------------------------------
# Reverse mode on packed buffers
# ---------------------------------------------------------------------------


class _ExplicitFn(torch.autograd.Function):

  @staticmethod
  def forward(ctx, buf, eng):
    ctx.eng = eng
    ctx.save_for_backward(buf)
    return eng.explicit(buf)

  @staticmethod
  def backward(ctx, g):
    (buf,) = ctx.saved_tensors
    return ctx.eng.explicit_vjp(buf, g.contiguous()), None


class _ImplicitFn(torch.autograd.Function):

  @staticmethod
  def forward(ctx, buf, eng):
    ctx.eng = eng
    return eng.implicit(buf)

  @staticmethod
  def backward(ctx, g):
    return ctx.eng.implicit_vjp(g.contiguous()), None


class _InverseFn(torch.autograd.Function):

  @staticmethod
  def forward(ctx, buf, eng, eta):
    ctx.eng, ctx.eta = eng, eta
    return eng.inverse(buf, eta)

  @staticmethod
  def backward(ctx, g):
    return ctx.eng.inverse_vjp(g.contiguous(), ctx.eta), None, None


class _RolloutFn(torch.autograd.Function):
  """n filtered SIL3 steps; the backward pass recomputes each step from its
  saved input state (per-step checkpointing, the role of
  nested_checkpoint_scan in time_integration.py:573-637)."""

  @staticmethod
  def forward(ctx, buf, eng, dt, filt, n_steps):
    ckpts = []
    y = buf.detach().clone()
    for _ in range(n_steps):
      ckpts.append(y.clone())
      eng.step_(y, dt, filt, 1)
    ctx.eng, ctx.dt, ctx.filt = eng, dt, filt
    ctx.ckpts = ckpts
    return y

  @staticmethod
  def backward(ctx, g):
    ct = g.detach().clone().contiguous()
    for y in reversed(ctx.ckpts):
      ctx.eng.step_vjp_(y, ct, ctx.dt, ctx.filt)
    ctx.ckpts = None
    return ct, None, None, None, None


def _needs_grad(buf):
  return torch.is_grad_enabled() and buf.requires_grad


# ---------------------------------------------------------------------------
# Equations
# ---------------------------------------------------------------------------


@dataclasses.dataclass(eq=False)
class PrimitiveEquationsSigma(time_integration.ImplicitExplicitODE):
  """Primitive equations on sigma coordinates (primitive_equations.py:835-1458).

  ``implicit_inverse_method`` accepts the reference's values; all of them are
  evaluated with the per-wavenumber dense inverse ('split'), which the
  reference's 'stacked' and 'blockwise' methods equal up to round-off.
  """

  reference_temperature: np.ndarray
  orography: Array
  coords: coordinate_systems.CoordinateSystem
  physics_specs: units.SimUnits
  vertical_matmul_method: str | None = dataclasses.field(default=None,
                                                          kw_only=True)
  implicit_inverse_method: str = dataclasses.field(default='split',
                                                   kw_only=True)
  include_vertical_advection: bool = dataclasses.field(default=True,
                                                       kw_only=True)
  humidity_key: str | None = dataclasses.field(default=None, kw_only=True)
  cloud_keys: tuple[str, ...] | None = dataclasses.field(default=None,
                                                         kw_only=True)
  held_suarez: Any = dataclasses.field(default=None, kw_only=True)

  def __post_init__(self):
    if not np.allclose(self.coords.horizontal.radius,
                       self.physics_specs.radius, rtol=1e-5):
      raise ValueError(
          'inconsistent radius between coordinates and constants: '
          f'{self.coords.horizontal.radius=} != {self.physics_specs.radius=}')
    if self.cloud_keys is not None and self.humidity_key is None:
      raise ValueError('cloud_keys requires humidity_key to be set.')
    if self.cloud_keys is not None:
      raise NotImplementedError('cloud_keys are not supported by this build')
    if self.implicit_inverse_method not in ('split', 'stacked', 'blockwise'):
      raise ValueError(
          f'invalid implicit_inverse_method {self.implicit_inverse_method}')
    self.reference_temperature = np.asarray(self.reference_temperature)
    self._engines = {}

  @property
  def T_ref(self):
    return self.reference_temperature[..., None, None]

  @property
  def coriolis_parameter(self):
    _, sin_lat = self.coords.horizontal.nodal_mesh
    return 2 * self.physics_specs.angular_velocity * sin_lat

  def _members(self, state: State) -> int:
    nd = state.vorticity.ndim
    if nd == 3:
      return 1
    if nd == 4:
      return int(state.vorticity.shape[0])
    raise StateShapeError(f'unexpected vorticity rank {nd}')

  def engine(self, state: State) -> _Engine:
    validate_state_shape(state, self.coords)
    key = (self._members(state), tuple(state.tracers.keys()))
    eng = self._engines.get(key)
    if eng is None:
      eng = _Engine(self, *key)
      self._engines[key] = eng
    return eng

  def explicit_terms(self, state: State) -> State:
    """primitive_equations.py:1126-1194."""
    eng = self.engine(state)
    buf = eng.pack(state)
    out = _ExplicitFn.apply(buf, eng) if _needs_grad(buf) else eng.explicit(buf)
    return eng.unpack(out, state,
                      None if state.sim_time is None else 1.0)

  def implicit_terms(self, state: State) -> State:
    """primitive_equations.py:1196-1249."""
    eng = self.engine(state)
    buf = eng.pack(state)
    out = _ImplicitFn.apply(buf, eng) if _needs_grad(buf) else eng.implicit(buf)
    return eng.unpack(out, state, None if state.sim_time is None else 0.0)

  def implicit_inverse(self, state: State, step_size: float) -> State:
    """(1 - step_size * implicit_terms)^-1 (primitive_equations.py:1251-1330)."""
    if isinstance(step_size, torch.Tensor):
      raise TypeError(
          f'`step_size` must be concrete but a tensor was passed: {step_size}.')
    eng = self.engine(state)
    buf = eng.pack(state)
    eta = float(step_size)
    out = (_InverseFn.apply(buf, eng, eta) if _needs_grad(buf)
           else eng.inverse(buf, eta))
    return eng.unpack(out, state, state.sim_time)



# ---------------------------------------------------------------------------
# Hybrid sigma-pressure levels (primitive_equations.py:1467-2533)
# ---------------------------------------------------------------------------


def _hybrid_vertical_coeffs(levels: hybrid_coordinates.HybridCoordinates,
                            p_s_ref: float):
  """alpha_k and log(p_{k+1/2} / p_{k-1/2}) at a uniform surface pressure
  (Simmons & Burridge 1981; _get_vertical_discretization_coeffs_numpy,
  primitive_equations.py:1483-1504)."""
  p_half = levels.a_boundaries + levels.b_boundaries * p_s_ref
  dp = np.diff(p_half)
  if np.any(dp <= 0):
    raise ValueError('Pressure must decrease monotonically with height.')
  upper, lower = p_half[:-1], p_half[1:]
  log_ratio = np.log(np.maximum(lower, 1e-6 * p_s_ref)
                     / np.maximum(upper, 1e-6 * p_s_ref))
  return 1 - (upper / dp) * log_ratio, log_ratio


def get_geopotential_weights_hybrid(levels, ideal_gas_constant, p_s_ref):
  """G with Phi'_k = R (alpha_k T_k + sum_{j>k} log-ratio_j T_j) (:1605-1625)."""
  alpha, log_ratio = _hybrid_vertical_coeffs(levels, p_s_ref)
  k = levels.layers
  return ideal_gas_constant * (np.diag(alpha)
                               + np.triu(np.broadcast_to(log_ratio, (k, k)), 1))


def get_temperature_implicit_weights_hybrid(levels, reference_temperature, kappa,
                                            p_s_ref):
  """H of the implicit temperature term on hybrid levels (:1736-1783)."""
  tref = np.asarray(reference_temperature)
  if tref.ndim != 1 or tref.shape[-1] != levels.layers:
    raise ValueError(
        '`reference_temp` must be a vector of length `coordinates.layers`; '
        f'got shape {tref.shape} and {levels.layers} layers.')
  k = levels.layers
  lower = np.tril(np.ones([k, k]))
  alpha, _ = _hybrid_vertical_coeffs(levels, p_s_ref)
  p_alpha = lower * alpha[:, None]
  p_alpha_up = np.concatenate([np.zeros([1, k]), p_alpha[:-1]], axis=0)
  dp_ref = levels.pressure_thickness + levels.sigma_thickness * p_s_ref
  h0 = kappa * tref[:, None] * (p_alpha + p_alpha_up) / dp_ref[:, None]
  k0 = np.concatenate((np.diff(tref) / (dp_ref[:-1] + dp_ref[1:]), [0]))[:, None]
  k1 = lower - np.cumsum(levels.sigma_thickness)[:, None]
  kk = k0 * k1
  kk_up = np.concatenate([np.zeros([1, k]), kk[:-1]], axis=0)
  return (h0 - kk - kk_up) * dp_ref[None, :]


def pgf_lps_coefficient_hybrid(temperature, surface_pressure, levels,
                               ideal_gas_constant):
  """C_k = (R T_k / dp_k) (log-ratio_k b_{k-1/2} + alpha_k db_k) p_s at a
  uniform surface pressure (_get_pgf_lps_coefficient_numpy, :1859-1887)."""
  alpha, log_ratio = _hybrid_vertical_coeffs(levels, surface_pressure)
  b = levels.b_boundaries
  dp = np.maximum(np.diff(levels.a_boundaries + b * surface_pressure),
                  1e-6 * surface_pressure)
  weight = log_ratio * b[:-1] + alpha * np.diff(b)
  return (ideal_gas_constant * np.asarray(temperature) / dp) * weight * surface_pressure


@dataclasses.dataclass(eq=False)
class PrimitiveEquationsHybrid(PrimitiveEquationsSigma):
  """Primitive equations on hybrid sigma-pressure levels
  (primitive_equations.py:1961-2533).

  ``coords.vertical`` is a ``HybridCoordinates`` with ``a_boundaries`` in
  units of ``hpa_quantity`` pascals (hPa by default);
  ``reference_surface_pressure`` (pascals) is where the implicit terms are
  linearised.  The explicit terms run in one CUDA column kernel
  (Simmons & Burridge discretisation, surface pressure varying per column);
  the implicit terms and their inverse, the fused imex_rk_sil3 step and CUDA
  graphs are the sigma engine's with the hybrid operators.  Reverse mode
  through the explicit terms and Held-Suarez forcing are sigma-only.
  """

  reference_surface_pressure: float = dataclasses.field(default=101325.0,
                                                        kw_only=True)
  hpa_quantity: float = dataclasses.field(default=100.0, kw_only=True)

  def __post_init__(self):
    super().__post_init__()
    if self.held_suarez is not None:
      raise NotImplementedError('Held-Suarez forcing is defined on sigma levels')
    if not isinstance(self.coords.vertical, hybrid_coordinates.HybridCoordinates):
      raise TypeError('PrimitiveEquationsHybrid needs HybridCoordinates levels')
    p_s_ref = units.nondim_pressure(float(self.reference_surface_pressure))
    if p_s_ref <= 0:
      raise ValueError('`reference_surface_pressure` must be positive.')
    self._p_s_ref = p_s_ref
    vert = self.coords.vertical
    self.nondim_levels = hybrid_coordinates.HybridCoordinates(
        a_boundaries=units.nondim_pressure(
            np.asarray(vert.a_boundaries, np.float64) * self.hpa_quantity),
        b_boundaries=vert.b_boundaries)

  @property
  def p_s_ref(self) -> float:
    return self._p_s_ref

  def explicit_terms(self, state: State) -> State:
    """primitive_equations.py:2249-2360."""
    eng = self.engine(state)
    buf = eng.pack(state)
    if _needs_grad(buf):
      raise NotImplementedError(
          'reverse mode through the explicit terms is built for sigma levels only')
    return eng.unpack(eng.explicit(buf), state,
                      None if state.sim_time is None else 1.0)


PrimitiveEquations = PrimitiveEquationsSigma


def MoistPrimitiveEquations(*args, **kwargs):  # pylint: disable=invalid-name
  """Deprecated alias of the reference (primitive_equations.py:2560-2596)."""
  kwargs.setdefault('humidity_key', 'specific_humidity')
  return PrimitiveEquationsSigma(*args, **kwargs)
