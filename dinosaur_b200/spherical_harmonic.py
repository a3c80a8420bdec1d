"""Spherical-harmonic grids whose transforms run as sm_100a CUDA kernels.

Mirrors the public surface of ``dinosaur/spherical_harmonic.py`` (reference
v1.3.6): the ``SphericalHarmonics`` plugin interface (:76-158), the Real
(m = 0, +1, -1, ...) modal layout (:161-283), and ``Grid`` with its standard
constructors and spectral operators (:678-1151).  Arrays are ``torch``
tensors on the current CUDA device (NumPy inputs are copied there); nodal
arrays are ``[..., lon, lat]`` and modal arrays ``[..., m, l]`` exactly as in
the reference.  Transforms and operators call ``libdino_b200.so``; there is no
CPU path.  Host-side constants (axes, masks, eigenvalues, the basis matrices
exposed through ``basis``) are FP64 NumPy like the reference's.
"""

from __future__ import annotations

import ctypes
import dataclasses
import functools
import math
from typing import Any, Callable

import numpy as np
import torch

from dinosaur_b200 import _lib
from dinosaur_b200 import pytree

Array = Any

# ---------------------------------------------------------------------------
# Host FP64 helpers (nodes for non-Gauss spacings, basis matrices)
# ---------------------------------------------------------------------------


def _legendre_host(n_m: int, n_l: int, x: np.ndarray) -> np.ndarray:
  """p[m, j, l]: associated Legendre functions normalised to unit L2 norm on
  [-1, 1] (associated_legendre.py:23-101), entries with l < m zero.

  Every order advances together: the sectoral values P_m^m come from one
  cumulative product over m, and each step in l applies the normalised
  three-term recurrence to all orders m < l at once (O(n_l) vector steps).
  """
  x = np.asarray(x, np.float64)
  m = np.arange(n_m, dtype=np.float64)[:, None]
  s = np.sqrt(1 - x * x)[None, :]
  scale = np.concatenate([[1 / np.sqrt(2)], -np.sqrt(1 + 1 / (2 * m[1:, 0]))])
  sectoral = np.cumprod(scale[:, None] * np.where(m > 0, s, 1.0), axis=0)
  out = np.zeros((n_m, len(x), n_l))
  prev = np.zeros((n_m, len(x)))   # P_{l-2}^m
  cur = np.zeros((n_m, len(x)))    # P_{l-1}^m
  for l in range(n_l):
    nxt = np.zeros_like(cur)
    lower = m[:, 0] < l
    if l > 0:
      mm = m[lower]
      a = np.sqrt((4.0 * l * l - 1) / (l * l - mm * mm))
      b = np.sqrt(((l - 1.0) ** 2 - mm * mm) / (4.0 * (l - 1.0) ** 2 - 1))
      nxt[lower] = a * (x[None, :] * cur[lower] - b * prev[lower])
    if l < n_m:
      nxt[l] = sectoral[l]
    out[:, :, l] = nxt
    prev, cur = cur, nxt
  return out


def _interpolatory_weights(n: int, with_poles: bool) -> np.ndarray:
  """Weights of the n-point interpolatory rule on equiangular nodes, in the
  order of ascending sin(latitude).

  The reference solves sum_j w_j P_k(x_j) = delta_k0 for k < n
  (associated_legendre.py:160-175): the unique n-point rule exact for
  polynomials of degree < n.  On equiangular nodes that rule has a closed
  form in the colatitudes phi: Fejer's first rule on the cell centres
  phi_k = (k + 1/2) pi / n, and the Clenshaw-Curtis rule on
  phi_k = k pi / (n - 1) with the poles (Waldvogel, BIT 46 (2006) 195-202).
  Both node sets are symmetric, so the colatitude order needs no reversal.
  """
  if with_poles:
    big_n = n - 1
    phi = np.arange(n) * np.pi / big_n
    j = np.arange(1, big_n // 2 + 1)
    b = np.where(2 * j == big_n, 1.0, 2.0)
    c = np.full(n, 2.0)
    c[0] = c[-1] = 1.0
    series = (b / (4.0 * j * j - 1))[None, :] * np.cos(2 * np.outer(phi, j))
    return c / big_n * (1 - series.sum(axis=1))
  phi = (np.arange(n) + 0.5) * np.pi / n
  j = np.arange(1, n // 2 + 1)
  series = np.cos(2 * np.outer(phi, j)) / (4.0 * j * j - 1)
  return 2.0 / n * (1 - 2 * series.sum(axis=1))


def _equiangular(n: int, with_poles: bool):
  """Equiangular latitudes (associated_legendre.py:117-157) and their weights."""
  if with_poles:
    theta = np.linspace(-np.pi / 2, np.pi / 2, n)
  else:
    s = np.pi / n
    theta = np.linspace(-np.pi / 2 + s / 2, np.pi / 2 - s / 2, n)
  return np.sin(theta), _interpolatory_weights(n, with_poles)


def _real_basis(wavenumbers: int, nodes: int) -> np.ndarray:
  """Real Fourier basis (fourier.py:24-60): columns 1/sqrt(2 pi), then
  cos(k lambda)/sqrt(pi) and sin(k lambda)/sqrt(pi) interleaved for k >= 1."""
  if nodes < wavenumbers:
    raise ValueError('`real_basis` requires nodes >= wavenumbers; '
                     f'got m = {nodes} and n = {wavenumbers}.')
  lam = 2 * np.pi * np.arange(nodes) / nodes
  k = np.arange(1, wavenumbers)
  f = np.empty((nodes, 2 * wavenumbers - 1))
  f[:, 0] = 1 / np.sqrt(2 * np.pi)
  f[:, 1::2] = np.cos(np.outer(lam, k)) / np.sqrt(np.pi)
  f[:, 2::2] = np.sin(np.outer(lam, k)) / np.sqrt(np.pi)
  return f


LATITUDE_SPACINGS = ('gauss', 'equiangular', 'equiangular_with_poles')


@dataclasses.dataclass
class _SphericalHarmonicBasis:
  """f: Fourier matrix, p: Legendre coefficients, w: nodal weights."""
  f: np.ndarray
  p: np.ndarray
  w: np.ndarray


# ---------------------------------------------------------------------------
# Tensor plumbing
# ---------------------------------------------------------------------------


def as_device_tensor(x, dtype=torch.float32) -> torch.Tensor:
  """Contiguous CUDA float32 tensor view/copy of x (NumPy or torch)."""
  if not torch.cuda.is_available():
    raise RuntimeError('dinosaur_b200 needs a CUDA device; none is available '
                       '(there is no CPU fallback)')
  if isinstance(x, torch.Tensor):
    t = x
    if not t.is_cuda:
      t = t.cuda()
  else:
    t = torch.as_tensor(np.asarray(x), device='cuda')
  if t.dtype != dtype:
    t = t.to(dtype)
  return t.contiguous()


def stream_handle() -> ctypes.c_void_p:
  return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def ptr(t: torch.Tensor) -> ctypes.c_void_p:
  return ctypes.c_void_p(t.data_ptr())


# ---------------------------------------------------------------------------
# Plan
# ---------------------------------------------------------------------------


class Plan:
  """Owns a ``dino_plan``: GPU tables and the transform workspace."""

  def __init__(self, lw, tw, nodes_lon, nodes_lat, spacing, radius=1.0,
               precision='fp32', max_fields=None, host_nodes=None):
    self.lw, self.L, self.I, self.J = lw, tw, nodes_lon, nodes_lat
    self.M = 2 * lw - 1
    if max_fields is None:
      per_field = self.M * self.J * 4
      max_fields = int(max(1, min(8192, (256 << 20) // per_field)))
    self.max_fields = max_fields
    self.precision = precision
    desc = _lib.GridDesc(lw, tw, nodes_lon, nodes_lat, _lib.SPACING[spacing],
                         0, float(radius), None, None)
    if host_nodes is not None:
      self._hx = np.ascontiguousarray(host_nodes[0], np.float64)
      self._hw = np.ascontiguousarray(host_nodes[1], np.float64)
      desc.host_nodes = _lib.dptr(self._hx)
      desc.host_weights = _lib.dptr(self._hw)
    if not torch.cuda.is_available():
      raise RuntimeError('dinosaur_b200 needs a CUDA device (no CPU fallback)')
    torch.cuda.current_device()  # initialise the context on this device
    handle = ctypes.c_void_p()
    _lib.check(_lib.lib().dino_plan_create(
        ctypes.byref(desc), max_fields, _lib.PRECISION[precision],
        ctypes.byref(handle)), 'dino_plan_create')
    self.handle = handle
    self.device = torch.cuda.current_device()

  def __del__(self):
    h = getattr(self, 'handle', None)
    if h is not None and h.value:
      try:
        _lib.lib().dino_plan_destroy(h)
      except Exception:  # interpreter shutdown
        pass

  @functools.cached_property
  def nodes(self) -> tuple[np.ndarray, np.ndarray]:
    x = np.zeros(self.J)
    w = np.zeros(self.J)
    _lib.check(_lib.lib().dino_plan_nodes(self.handle, _lib.dptr(x),
                                          _lib.dptr(w)))
    return x, w

  # -- raw calls on flat batches -------------------------------------------
  def _check(self, x: torch.Tensor, trailing: tuple[int, int], what: str):
    if not isinstance(x, torch.Tensor) or not x.is_cuda:
      raise ValueError(f'{what}: expected a CUDA tensor')
    if x.dtype != torch.float32 or not x.is_contiguous():
      raise ValueError(f'{what}: expected a contiguous float32 tensor')
    if x.ndim < 2 or tuple(x.shape[-2:]) != tuple(trailing):
      raise ValueError(f'{what}: expected trailing shape {trailing}, '
                       f'got {tuple(x.shape)}')
    if x.device.index != self.device:
      raise ValueError(f'{what}: tensor on cuda:{x.device.index}, plan on '
                       f'cuda:{self.device}')

  def _call(self, name, x: torch.Tensor, out_shape, nfields):
    out = torch.empty(out_shape, device=x.device, dtype=torch.float32)
    fn = getattr(_lib.lib(), name)
    _lib.check(fn(self.handle, ptr(x), ptr(out), nfields, stream_handle()),
               name)
    return out

  def inverse(self, x: torch.Tensor) -> torch.Tensor:
    self._check(x, (self.M, self.L), 'inverse')
    lead = x.shape[:-2]
    n = int(np.prod(lead)) if lead else 1
    return self._call('dino_sht_inverse', x, lead + (self.I, self.J), n)

  def forward(self, z: torch.Tensor) -> torch.Tensor:
    self._check(z, (self.I, self.J), 'forward')
    lead = z.shape[:-2]
    n = int(np.prod(lead)) if lead else 1
    return self._call('dino_sht_forward', z, lead + (self.M, self.L), n)

  def inverse_adjoint(self, g: torch.Tensor) -> torch.Tensor:
    self._check(g, (self.I, self.J), 'inverse_adjoint')
    lead = g.shape[:-2]
    n = int(np.prod(lead)) if lead else 1
    return self._call('dino_sht_inverse_adjoint', g, lead + (self.M, self.L), n)

  def forward_adjoint(self, g: torch.Tensor) -> torch.Tensor:
    self._check(g, (self.M, self.L), 'forward_adjoint')
    lead = g.shape[:-2]
    n = int(np.prod(lead)) if lead else 1
    return self._call('dino_sht_forward_adjoint', g, lead + (self.I, self.J), n)

  def describe(self) -> str:
    """Shapes, Legendre form and (split-BF16) the autotuned launch shapes."""
    buf = ctypes.create_string_buffer(1024)
    _lib.check(_lib.lib().dino_plan_describe(self.handle, buf, len(buf)), 'describe')
    return buf.value.decode()

  def relayout(self, x: torch.Tensor, to_fast: bool) -> torch.Tensor:
    """Real <-> FastSphericalHarmonics modal rows (dino_modal_relayout)."""
    rows_in = self.M + (0 if to_fast else 1)
    rows_out = self.M + (1 if to_fast else 0)
    if tuple(x.shape[-2:]) != (rows_in, self.L):
      raise ValueError(f'expected [..., {rows_in}, {self.L}] modal array; got '
                       f'{tuple(x.shape)}')
    x = x.contiguous()
    nf = x.numel() // (rows_in * self.L)
    out = torch.empty(x.shape[:-2] + (rows_out, self.L), device=x.device,
                      dtype=torch.float32)
    _lib.check(_lib.lib().dino_modal_relayout(self.handle, int(to_fast), ptr(x),
                                              ptr(out), nf, stream_handle()),
               'modal_relayout')
    return out

  def modal_op(self, op: str, x: torch.Tensor, arg: int = 0,
               transpose: bool = False) -> torch.Tensor:
    self._check(x, (self.M, self.L), op)
    lead = x.shape[:-2]
    n = int(np.prod(lead)) if lead else 1
    out = torch.empty_like(x)
    code = _lib.OPS[op] | (8 if transpose else 0)
    _lib.check(_lib.lib().dino_modal_op(self.handle, code, ptr(x), ptr(out), n,
                                        arg, stream_handle()), op)
    return out


# ---------------------------------------------------------------------------
# SphericalHarmonics implementations
# ---------------------------------------------------------------------------


@dataclasses.dataclass(frozen=True)
class SphericalHarmonics:
  """Plugin interface of spherical_harmonic.py:76-158."""

  longitude_wavenumbers: int = 0
  total_wavenumbers: int = 0
  longitude_nodes: int = 0
  latitude_nodes: int = 0
  latitude_spacing: str = 'gauss'

  @property
  def nodal_axes(self): raise NotImplementedError
  @property
  def nodal_shape(self): raise NotImplementedError
  @property
  def nodal_padding(self): raise NotImplementedError
  @property
  def modal_axes(self): raise NotImplementedError
  @property
  def modal_shape(self): raise NotImplementedError
  @property
  def modal_padding(self): raise NotImplementedError
  @property
  def modal_dtype(self): raise NotImplementedError
  @property
  def mask(self): raise NotImplementedError
  @property
  def basis(self): raise NotImplementedError

  def inverse_transform(self, x): raise NotImplementedError
  def transform(self, x): raise NotImplementedError
  def longitudinal_derivative(self, x): raise NotImplementedError


@dataclasses.dataclass(frozen=True)
class CudaSphericalHarmonics(SphericalHarmonics):
  """Real-layout spherical harmonics on sm_100a (same layout as
  RealSphericalHarmonics, spherical_harmonic.py:161-283).

  ``precision`` selects the Legendre contraction: 'fp32' (SIMT FMA),
  'bf16x3' or 'tf32x3' (tcgen05 tensor cores, operands split into bf16 or
  tf32 hi / lo pairs, three products per pair, FP32 accumulation).
  """

  precision: str = 'fp32'

  @functools.cached_property
  def plan(self) -> Plan:
    host = None
    if self.latitude_spacing != 'gauss':
      host = _equiangular(self.latitude_nodes,
                          self.latitude_spacing == 'equiangular_with_poles')
    return Plan(self.longitude_wavenumbers, self.total_wavenumbers,
                self.longitude_nodes, self.latitude_nodes,
                self.latitude_spacing, precision=self.precision,
                host_nodes=host)

  @functools.cached_property
  def nodal_axes(self):
    longitude = np.linspace(0, 2 * np.pi, self.longitude_nodes, endpoint=False)
    if self.latitude_spacing == 'gauss':
      sin_latitude = self.plan.nodes[0]
    else:
      sin_latitude = _equiangular(
          self.latitude_nodes,
          self.latitude_spacing == 'equiangular_with_poles')[0]
    return longitude, sin_latitude

  @functools.cached_property
  def quadrature_weights_lat(self) -> np.ndarray:
    if self.latitude_spacing == 'gauss':
      return self.plan.nodes[1]
    return _equiangular(self.latitude_nodes,
                        self.latitude_spacing == 'equiangular_with_poles')[1]

  @property
  def nodal_shape(self):
    return (self.longitude_nodes, self.latitude_nodes)

  @property
  def nodal_padding(self):
    return (0, 0)

  @functools.cached_property
  def modal_axes(self):
    m_pos = np.arange(1, self.longitude_wavenumbers)
    m_pos_neg = np.stack([m_pos, -m_pos], axis=1).ravel()
    return (np.concatenate([[0], m_pos_neg]),
            np.arange(self.total_wavenumbers))

  @property
  def modal_shape(self):
    return (2 * self.longitude_wavenumbers - 1, self.total_wavenumbers)

  @property
  def modal_padding(self):
    return (0, 0)

  @property
  def modal_dtype(self):
    return np.dtype(np.float32)

  @functools.cached_property
  def mask(self):
    m, l = np.meshgrid(*self.modal_axes, indexing='ij')
    return abs(m) <= l

  @functools.cached_property
  def basis(self) -> _SphericalHarmonicBasis:
    """FP64 (f, p, w) as in spherical_harmonic.py:219-260 (host copies)."""
    f = _real_basis(self.longitude_wavenumbers, self.longitude_nodes)
    x = self.nodal_axes[1]
    w = (2 * np.pi / self.longitude_nodes) * self.quadrature_weights_lat
    p = _legendre_host(self.longitude_wavenumbers, self.total_wavenumbers, x)
    p = np.repeat(p, 2, axis=0)[1:]
    return _SphericalHarmonicBasis(f=f, p=p, w=w)

  def inverse_transform(self, x):
    from dinosaur_b200 import autograd  # pylint: disable=g-import-not-at-top
    return autograd.sht_inverse(self.plan, as_device_tensor(x))

  def transform(self, x):
    from dinosaur_b200 import autograd  # pylint: disable=g-import-not-at-top
    return autograd.sht_forward(self.plan, as_device_tensor(x))

  def longitudinal_derivative(self, x):
    from dinosaur_b200 import autograd  # pylint: disable=g-import-not-at-top
    return autograd.modal_op(self.plan, 'd_dlon', as_device_tensor(x))


# The reference's default implementation name maps to the CUDA one.
RealSphericalHarmonics = CudaSphericalHarmonics


class _Relayout(torch.autograd.Function):
  """Real <-> Fast modal layout (a row insertion / deletion: its transpose is
  the opposite conversion)."""

  @staticmethod
  def forward(ctx, x, plan, to_fast):
    ctx.plan, ctx.to_fast = plan, to_fast
    return plan.relayout(x, to_fast)

  @staticmethod
  def backward(ctx, g):
    return ctx.plan.relayout(g.contiguous(), not ctx.to_fast), None, None


def relayout(plan: Plan, x: torch.Tensor, to_fast: bool) -> torch.Tensor:
  if torch.is_grad_enabled() and x.requires_grad:
    return _Relayout.apply(x, plan, to_fast)
  return plan.relayout(x, to_fast)


@dataclasses.dataclass(frozen=True)
class FastSphericalHarmonics(CudaSphericalHarmonics):
  """The m-stacked modal layout of FastSphericalHarmonics
  (spherical_harmonic.py:411-621) on one GPU: rows m = 0, 0 (imaginary, always
  zero), 1, -1, 2, -2, ... of shape (2 lw, L).  Transforms and operators run
  in the Real layout; modal arrays are converted at this boundary by
  ``dino_modal_relayout``.  The reference's sharding and einsum-ordering
  options are accepted and have no effect on one GPU.
  """

  spmd_mesh: Any = None
  base_shape_multiple: int | None = None
  reverse_einsum_arg_order: bool | None = None
  stacked_fourier_transforms: bool | None = None
  transform_precision: str = 'tensorfloat32'

  @functools.cached_property
  def modal_axes(self):
    m_pos = np.arange(1, self.longitude_wavenumbers)
    m_pos_neg = np.stack([m_pos, -m_pos], axis=1).ravel()
    return (np.concatenate([[0, 0], m_pos_neg]),
            np.arange(self.total_wavenumbers))

  @property
  def modal_shape(self):
    return (2 * self.longitude_wavenumbers, self.total_wavenumbers)

  @functools.cached_property
  def mask(self):
    m, l = np.meshgrid(*self.modal_axes, indexing='ij')
    rows = np.arange(self.modal_shape[0])[:, None]
    return (abs(m) <= l) & (rows != 1)

  @functools.cached_property
  def basis(self) -> _SphericalHarmonicBasis:
    """f with the zero imaginary m = 0 column, p per m (not repeated)."""
    f = _real_basis(self.longitude_wavenumbers, self.longitude_nodes)
    f = np.insert(f, 1, 0.0, axis=1)
    x = self.nodal_axes[1]
    w = (2 * np.pi / self.longitude_nodes) * self.quadrature_weights_lat
    p = _legendre_host(self.longitude_wavenumbers, self.total_wavenumbers, x)
    return _SphericalHarmonicBasis(f=f, p=p, w=w)

  def to_real(self, x):
    return relayout(self.plan, as_device_tensor(x), False)

  def from_real(self, x):
    return relayout(self.plan, as_device_tensor(x), True)

  def inverse_transform(self, x):
    return super().inverse_transform(self.to_real(x))

  def transform(self, x):
    return self.from_real(super().transform(x))

  def longitudinal_derivative(self, x):
    return self.from_real(super().longitudinal_derivative(self.to_real(x)))


RealSphericalHarmonicsWithZeroImag = FastSphericalHarmonics


def is_fast_layout(grid) -> bool:
  return isinstance(grid.spherical_harmonics, FastSphericalHarmonics)


def to_real_layout(grid, x):
  """Modal array of `grid`'s layout -> the Real layout (identity for Real)."""
  if is_fast_layout(grid):
    return grid.spherical_harmonics.to_real(x)
  return as_device_tensor(x)


def from_real_layout(grid, x):
  """Real-layout modal array -> `grid`'s layout (identity for Real)."""
  if is_fast_layout(grid):
    return grid.spherical_harmonics.from_real(x)
  return x

SphericalHarmonicsImpl = Callable[..., SphericalHarmonics]


# ---------------------------------------------------------------------------
# Grid
# ---------------------------------------------------------------------------


@dataclasses.dataclass(frozen=True)
class Grid:
  """Real-space and spectral grids over the sphere (spherical_harmonic.py:678-1151)."""

  longitude_wavenumbers: int = 0
  total_wavenumbers: int = 0
  longitude_nodes: int = 0
  latitude_nodes: int = 0
  latitude_spacing: str = 'gauss'
  longitude_offset: float = 0.0
  radius: float | None = None
  spherical_harmonics_impl: SphericalHarmonicsImpl = CudaSphericalHarmonics
  spmd_mesh: Any = None

  def __post_init__(self):
    if self.radius is None:
      object.__setattr__(self, 'radius', 1.0)
    if self.latitude_spacing not in LATITUDE_SPACINGS:
      raise ValueError(
          f'Unsupported `latitude_spacing` "{self.latitude_spacing}". '
          f'Supported values are: {list(LATITUDE_SPACINGS)}.')
    if self.spmd_mesh is not None:
      raise NotImplementedError(
          'spmd_mesh model parallelism is not part of this build; '
          'run ensemble members as independent replicas instead')

  @classmethod
  def with_wavenumbers(cls, longitude_wavenumbers: int,
                       dealiasing: str = 'quadratic',
                       latitude_spacing: str = 'gauss',
                       longitude_offset: float = 0.0,
                       spherical_harmonics_impl=CudaSphericalHarmonics,
                       radius: float | None = None, spmd_mesh=None) -> Grid:
    """spherical_harmonic.py:737-770."""
    order = {'linear': 2, 'quadratic': 3, 'cubic': 4}[dealiasing]
    longitude_nodes = order * longitude_wavenumbers + 1
    latitude_nodes = math.ceil(longitude_nodes / 2)
    return cls(longitude_wavenumbers=longitude_wavenumbers,
               total_wavenumbers=longitude_wavenumbers + 1,
               longitude_nodes=longitude_nodes, latitude_nodes=latitude_nodes,
               latitude_spacing=latitude_spacing,
               longitude_offset=longitude_offset,
               spherical_harmonics_impl=spherical_harmonics_impl,
               radius=radius, spmd_mesh=spmd_mesh)

  @classmethod
  def construct(cls, max_wavenumber: int, gaussian_nodes: int,
                latitude_spacing: str = 'gauss', longitude_offset: float = 0.0,
                radius: float | None = None,
                spherical_harmonics_impl=CudaSphericalHarmonics,
                spmd_mesh=None) -> Grid:
    """spherical_harmonic.py:772-813."""
    return cls(longitude_wavenumbers=max_wavenumber + 1,
               total_wavenumbers=max_wavenumber + 2,
               longitude_nodes=4 * gaussian_nodes,
               latitude_nodes=2 * gaussian_nodes,
               latitude_spacing=latitude_spacing,
               longitude_offset=longitude_offset,
               spherical_harmonics_impl=spherical_harmonics_impl,
               radius=radius, spmd_mesh=spmd_mesh)

  # pylint: disable=invalid-name
  @classmethod
  def T21(cls, **kw): return cls.construct(21, 16, **kw)
  @classmethod
  def T31(cls, **kw): return cls.construct(31, 24, **kw)
  @classmethod
  def T42(cls, **kw): return cls.construct(42, 32, **kw)
  @classmethod
  def T85(cls, **kw): return cls.construct(85, 64, **kw)
  @classmethod
  def T106(cls, **kw): return cls.construct(106, 80, **kw)
  @classmethod
  def T119(cls, **kw): return cls.construct(119, 90, **kw)
  @classmethod
  def T170(cls, **kw): return cls.construct(170, 128, **kw)
  @classmethod
  def T213(cls, **kw): return cls.construct(213, 160, **kw)
  @classmethod
  def T340(cls, **kw): return cls.construct(340, 256, **kw)
  @classmethod
  def T425(cls, **kw): return cls.construct(425, 320, **kw)
  @classmethod
  def TL31(cls, **kw): return cls.construct(31, 16, **kw)
  @classmethod
  def TL47(cls, **kw): return cls.construct(47, 24, **kw)
  @classmethod
  def TL63(cls, **kw): return cls.construct(63, 32, **kw)
  @classmethod
  def TL95(cls, **kw): return cls.construct(95, 48, **kw)
  @classmethod
  def TL127(cls, **kw): return cls.construct(127, 64, **kw)
  @classmethod
  def TL159(cls, **kw): return cls.construct(159, 80, **kw)
  @classmethod
  def TL179(cls, **kw): return cls.construct(179, 90, **kw)
  @classmethod
  def TL255(cls, **kw): return cls.construct(255, 128, **kw)
  @classmethod
  def TL639(cls, **kw): return cls.construct(639, 320, **kw)
  @classmethod
  def TL1279(cls, **kw): return cls.construct(1279, 640, **kw)
  # pylint: enable=invalid-name

  def asdict(self) -> dict[str, Any]:
    items = dataclasses.asdict(self)
    impl = self.spherical_harmonics_impl
    items['spherical_harmonics_impl'] = getattr(
        impl, '__name__', getattr(getattr(impl, 'func', None), '__name__', ''))
    items['spmd_mesh'] = ''
    return items

  @functools.cached_property
  def spherical_harmonics(self) -> SphericalHarmonics:
    return self.spherical_harmonics_impl(
        longitude_wavenumbers=self.longitude_wavenumbers,
        total_wavenumbers=self.total_wavenumbers,
        longitude_nodes=self.longitude_nodes,
        latitude_nodes=self.latitude_nodes,
        latitude_spacing=self.latitude_spacing)

  @property
  def plan(self) -> Plan:
    return self.spherical_harmonics.plan

  @property
  def longitudes(self):
    return self.nodal_axes[0]

  @property
  def latitudes(self):
    return np.arcsin(self.nodal_axes[1])

  @functools.cached_property
  def nodal_axes(self):
    lon, sin_lat = self.spherical_harmonics.nodal_axes
    return lon + self.longitude_offset, sin_lat

  @property
  def nodal_shape(self):
    return (self.longitude_nodes, self.latitude_nodes)

  @property
  def nodal_padding(self):
    return (0, 0)

  @functools.cached_property
  def nodal_mesh(self):
    return np.meshgrid(*self.nodal_axes, indexing='ij')

  @functools.cached_property
  def modal_axes(self):
    return self.spherical_harmonics.modal_axes

  @property
  def modal_shape(self):
    return self.spherical_harmonics.modal_shape

  @property
  def modal_padding(self):
    return self.spherical_harmonics.modal_padding

  @functools.cached_property
  def mask(self):
    return self.spherical_harmonics.mask

  @functools.cached_property
  def modal_mesh(self):
    return np.meshgrid(*self.modal_axes, indexing='ij')

  @functools.cached_property
  def cos_lat(self):
    _, sin_lat = self.nodal_axes
    return np.sqrt(1 - sin_lat ** 2)

  @functools.cached_property
  def sec2_lat(self):
    _, sin_lat = self.nodal_axes
    return 1 / (1 - sin_lat ** 2)

  @functools.cached_property
  def laplacian_eigenvalues(self):
    _, l = self.modal_axes
    return -l * (l + 1) / (self.radius ** 2)

  # -- transforms ----------------------------------------------------------
  def to_nodal(self, x):
    """Modal -> nodal over every non-scalar leaf (spherical_harmonic.py:1017-1023)."""
    return pytree.map_over_nonscalars(
        self.spherical_harmonics.inverse_transform, x)

  def to_modal(self, z):
    """Nodal -> modal over every non-scalar leaf (spherical_harmonic.py:1025-1031)."""
    return pytree.map_over_nonscalars(self.spherical_harmonics.transform, z)

  # -- operators -------------------------------------------------------------
  def _op(self, name, x, arg=0):
    from dinosaur_b200 import autograd  # pylint: disable=g-import-not-at-top
    out = autograd.modal_op(self.plan, name, to_real_layout(self, x), arg,
                            radius=1.0)
    return from_real_layout(self, out)

  def laplacian(self, x):
    """x * -l(l+1)/r^2 (spherical_harmonic.py:1033-1036)."""
    out = self._op('laplacian', x)
    return out if self.radius == 1.0 else out / self.radius ** 2

  def inverse_laplacian(self, x):
    """spherical_harmonic.py:1038-1046 (l = 0 maps to 0)."""
    out = self._op('inverse_laplacian', x)
    return out if self.radius == 1.0 else out * self.radius ** 2

  def clip_wavenumbers(self, x, n: int = 1):
    """Zeros the highest n total wavenumbers (spherical_harmonic.py:1048-1061)."""
    if n <= 0:
      raise ValueError(f'`n` must be >= 0; got {n}.')
    return pytree.map_over_nonscalars(lambda y: self._op('clip', y, n), x)

  def d_dlon(self, x):
    """spherical_harmonic.py:1072-1077."""
    return self._op('d_dlon', x)

  def cos_lat_d_dlat(self, x):
    """spherical_harmonic.py:1079-1093."""
    return self._op('cos_lat_d_dlat', x)

  def sec_lat_d_dlat_cos2(self, x):
    """spherical_harmonic.py:1095-1102."""
    return self._op('sec_lat_d_dlat_cos2', x)

  def cos_lat_grad(self, x, clip: bool = True):
    """spherical_harmonic.py:1104-1111."""
    raw = self.d_dlon(x) / self.radius, self.cos_lat_d_dlat(x) / self.radius
    if clip:
      return self.clip_wavenumbers(raw)
    return raw

  def k_cross(self, v):
    """spherical_harmonic.py:1113-1116."""
    return -v[1], v[0]

  def div_cos_lat(self, v, clip: bool = True):
    """spherical_harmonic.py:1118-1128."""
    raw = (self.d_dlon(v[0]) + self.sec_lat_d_dlat_cos2(v[1])) / self.radius
    return self.clip_wavenumbers(raw) if clip else raw

  def curl_cos_lat(self, v, clip: bool = True):
    """spherical_harmonic.py:1130-1140."""
    raw = (self.d_dlon(v[1]) - self.sec_lat_d_dlat_cos2(v[0])) / self.radius
    return self.clip_wavenumbers(raw) if clip else raw

  @property
  def quadrature_weights(self) -> np.ndarray:
    return np.broadcast_to(self.spherical_harmonics.basis.w, self.nodal_shape)

  def integrate(self, z):
    """Quadrature over the sphere (spherical_harmonic.py:1147-1151)."""
    w = torch.as_tensor(
        (2 * np.pi / self.longitude_nodes)
        * self.spherical_harmonics.quadrature_weights_lat * self.radius ** 2,
        device='cuda', dtype=torch.float32)
    z = as_device_tensor(z)
    return torch.einsum('y,...xy->...', w, z)


_CONSTANT_NORMALIZATION_FACTOR = 3.5449077


def add_constant(x, c):
  """Adds c to a modal array (spherical_harmonic.py:1159-1161)."""
  x = as_device_tensor(x).clone()
  x[..., 0, 0] += _CONSTANT_NORMALIZATION_FACTOR * c
  return x


def get_cos_lat_vector(vorticity, divergence, grid: Grid, clip: bool = True):
  """v cos(lat) from vorticity and divergence (spherical_harmonic.py:1164-1178)."""
  stream_function = grid.inverse_laplacian(vorticity)
  velocity_potential = grid.inverse_laplacian(divergence)
  a = grid.cos_lat_grad(velocity_potential, clip=clip)
  b = grid.k_cross(grid.cos_lat_grad(stream_function, clip=clip))
  return a[0] + b[0], a[1] + b[1]


def _cos_lat_tensor(grid: Grid) -> torch.Tensor:
  return torch.as_tensor(grid.cos_lat, device='cuda', dtype=torch.float32)


def uv_nodal_to_vor_div_modal(grid: Grid, u_nodal, v_nodal, clip: bool = True):
  """spherical_harmonic.py:1181-1194."""
  cos = _cos_lat_tensor(grid)
  u = grid.to_modal(as_device_tensor(u_nodal) / cos)
  v = grid.to_modal(as_device_tensor(v_nodal) / cos)
  return (grid.curl_cos_lat((u, v), clip=clip),
          grid.div_cos_lat((u, v), clip=clip))


def vor_div_to_uv_nodal(grid: Grid, vorticity, divergence, clip: bool = True):
  """spherical_harmonic.py:1197-1210."""
  u, v = get_cos_lat_vector(vorticity, divergence, grid, clip=clip)
  cos = _cos_lat_tensor(grid)
  return grid.to_nodal(u) / cos, grid.to_nodal(v) / cos
