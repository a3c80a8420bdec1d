"""ctypes binding of ``libdino_b200.so`` (the C ABI in ``include/dino_b200.h``).

The library is loaded from this package directory.  There is no fallback:
if it is missing, or if no CUDA device is available when a kernel is needed,
calls raise.  Status codes map to the reference's exception types
(``ValueError`` for bad arguments and shapes, ``RuntimeError`` otherwise).
"""

from __future__ import annotations

import ctypes
import functools
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, 'libdino_b200.so')

DINO_OK = 0
DINO_ERR_ARG = 1
DINO_ERR_SHAPE = 2
DINO_ERR_CUDA = 3
DINO_ERR_TIMEOUT = 4
DINO_ERR_NAN = 5
DINO_ERR_UNSUPPORTED = 6

SPACING = {'gauss': 0, 'equiangular': 1, 'equiangular_with_poles': 2}
PRECISION = {'fp32': 0, 'bf16x3': 1, 'tf32x3': 2}
OPS = dict(d_dlon=0, cos_lat_d_dlat=1, sec_lat_d_dlat_cos2=2, laplacian=3,
           inverse_laplacian=4, clip=5)


class DinoError(RuntimeError):
  """A CUDA-side failure reported by libdino_b200."""

  def __init__(self, code: int, message: str):
    super().__init__(f'[dino status {code}] {message}')
    self.code = code


class DinoNonFiniteError(DinoError, AssertionError):
  """DINO_ERR_NAN: a non-finite or singular implicit operator.  Also an
  AssertionError, the exception the reference raises there
  (primitive_equations.py:1296 asserts that the inverse has no NaN)."""


class GridDesc(ctypes.Structure):
  _fields_ = [
      ('longitude_wavenumbers', ctypes.c_int32),
      ('total_wavenumbers', ctypes.c_int32),
      ('longitude_nodes', ctypes.c_int32),
      ('latitude_nodes', ctypes.c_int32),
      ('latitude_spacing', ctypes.c_int32),
      ('reserved', ctypes.c_int32),
      ('radius', ctypes.c_double),
      ('host_nodes', ctypes.POINTER(ctypes.c_double)),
      ('host_weights', ctypes.POINTER(ctypes.c_double)),
  ]


_DP = ctypes.POINTER(ctypes.c_double)


class SWEDesc(ctypes.Structure):
  _fields_ = [
      ('layers', ctypes.c_int32),
      ('members', ctypes.c_int32),
      ('reference_potential', ctypes.POINTER(ctypes.c_double)),
      ('densities', ctypes.POINTER(ctypes.c_double)),
      ('orography_modal', ctypes.POINTER(ctypes.c_float)),
      ('angular_velocity', ctypes.c_double),
  ]


class PEDesc(ctypes.Structure):
  _fields_ = [
      ('layers', ctypes.c_int32),
      ('members', ctypes.c_int32),
      ('n_tracers', ctypes.c_int32),
      ('humidity_tracer', ctypes.c_int32),
      ('include_vertical_advection', ctypes.c_int32),
      ('held_suarez', ctypes.c_int32),
      ('sigma_boundaries', _DP),
      ('sigma_centers', _DP),
      ('layer_thickness', _DP),
      ('inv_center_to_center', _DP),
      ('reference_temperature', _DP),
      ('geopotential_weights', _DP),
      ('temperature_weights', _DP),
      ('sigma_ratios', _DP),
      ('orography_modal', ctypes.POINTER(ctypes.c_float)),
      ('angular_velocity', ctypes.c_double),
      ('gravity', ctypes.c_double),
      ('R', ctypes.c_double),
      ('R_vapor', ctypes.c_double),
      ('Cp_vapor', ctypes.c_double),
      ('kappa', ctypes.c_double),
      ('hs_p0', ctypes.c_double),
      ('hs_sigma_b', ctypes.c_double),
      ('hs_kf', ctypes.c_double),
      ('hs_ka', ctypes.c_double),
      ('hs_ks', ctypes.c_double),
      ('hs_minT', ctypes.c_double),
      ('hs_maxT', ctypes.c_double),
      ('hs_dTy', ctypes.c_double),
      ('hs_dThz', ctypes.c_double),
      ('vertical_scheme', ctypes.c_int32),
      ('hybrid_a_boundaries', _DP),
      ('hybrid_b_boundaries', _DP),
      ('reference_surface_pressure', ctypes.c_double),
      ('implicit_lnps_column', _DP),
      ('implicit_thickness', _DP),
  ]


_vp = ctypes.c_void_p
_i32 = ctypes.c_int32

# name -> (restype, argtypes)
SIGNATURES = {
    'dino_last_error': (ctypes.c_int, [ctypes.c_char_p, ctypes.c_size_t]),
    'dino_version': (ctypes.c_char_p, []),
    'dino_plan_create': (ctypes.c_int, [ctypes.POINTER(GridDesc), _i32, _i32,
                                        ctypes.POINTER(_vp)]),
    'dino_plan_destroy': (ctypes.c_int, [_vp]),
    'dino_plan_nodes': (ctypes.c_int, [_vp, _DP, _DP]),
    'dino_plan_legendre_column': (ctypes.c_int, [_vp, _i32, _i32, _DP]),
    'dino_plan_status': (ctypes.c_int, [_vp]),
    'dino_plan_check_wait_timeout': (ctypes.c_int, [_vp, ctypes.c_int64, _vp]),
    'dino_sht_inverse': (ctypes.c_int, [_vp, _vp, _vp, _i32, _vp]),
    'dino_sht_inverse_noalloc': (ctypes.c_int, [_vp, _vp, _vp, _i32, _vp]),
    'dino_sht_forward': (ctypes.c_int, [_vp, _vp, _vp, _i32, _vp]),
    'dino_sht_inverse_adjoint': (ctypes.c_int, [_vp, _vp, _vp, _i32, _vp]),
    'dino_sht_forward_adjoint': (ctypes.c_int, [_vp, _vp, _vp, _i32, _vp]),
    'dino_modal_op': (ctypes.c_int, [_vp, _i32, _vp, _vp, _i32, _i32, _vp]),
    'dino_sht_phase': (ctypes.c_int, [_vp, _i32, _vp, _vp, _i32, _vp]),
    'dino_pe_create': (ctypes.c_int, [_vp, ctypes.POINTER(PEDesc),
                                      ctypes.POINTER(_vp)]),
    'dino_pe_destroy': (ctypes.c_int, [_vp]),
    'dino_pe_state_size': (ctypes.c_int64, [_vp]),
    'dino_pe_explicit': (ctypes.c_int, [_vp, _vp, _vp, _vp]),
    'dino_pe_implicit': (ctypes.c_int, [_vp, _vp, _vp, _vp]),
    'dino_pe_implicit_inverse': (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_double,
                                                _vp]),
    'dino_pe_step': (ctypes.c_int, [_vp, _vp, ctypes.c_double, _DP, _i32, _vp]),
    'dino_pe_step_graph': (ctypes.c_int, [_vp, _vp, ctypes.c_double, _DP, _i32,
                                          _vp]),
    'dino_modal_relayout': (ctypes.c_int, [_vp, _i32, _vp, _vp, _i32, _vp]),
    'dino_plan_describe': (ctypes.c_int, [_vp, ctypes.c_char_p, ctypes.c_size_t]),
    'dino_swe_create': (ctypes.c_int, [_vp, ctypes.POINTER(SWEDesc),
                                       ctypes.POINTER(_vp)]),
    'dino_swe_destroy': (ctypes.c_int, [_vp]),
    'dino_swe_state_size': (ctypes.c_int64, [_vp]),
    'dino_swe_explicit': (ctypes.c_int, [_vp, _vp, _vp, _vp]),
    'dino_swe_implicit': (ctypes.c_int, [_vp, _vp, _vp, _vp]),
    'dino_swe_implicit_inverse': (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_double,
                                                 _vp]),
    'dino_pe_explicit_vjp': (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp]),
    'dino_pe_implicit_vjp': (ctypes.c_int, [_vp, _vp, _vp, _vp]),
    'dino_pe_implicit_inverse_vjp': (ctypes.c_int, [_vp, _vp, _vp,
                                                    ctypes.c_double, _vp]),
    'dino_pe_counts': (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int32)]),
    'dino_pe_trajectory': (ctypes.c_int, [_vp, _vp, ctypes.c_double, _DP, _i32, _i32,
                                          _i32, _vp, _vp]),
    'dino_pe_step_vjp': (ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_double,
                                        _DP, _vp]),
}


@functools.lru_cache(maxsize=1)
def lib() -> ctypes.CDLL:
  """Loads the library (raises if it has not been built)."""
  if not os.path.exists(LIB_PATH):
    raise ImportError(
        f'{LIB_PATH} is missing: build it with `python -m dinosaur_b200.build`'
        ' (dinosaur_b200 has no CPU fallback).')
  handle = ctypes.CDLL(LIB_PATH)
  for name, (res, args) in SIGNATURES.items():
    fn = getattr(handle, name, None)
    if fn is None:  # reported by the symbol-coverage test
      continue
    fn.restype = res
    fn.argtypes = args
  return handle


def last_error() -> str:
  buf = ctypes.create_string_buffer(2048)
  lib().dino_last_error(buf, len(buf))
  return buf.value.decode(errors='replace')


def check(status: int, what: str = ''):
  """Raises the exception matching a C status code."""
  if status == DINO_OK:
    return
  msg = last_error()
  if what:
    msg = f'{what}: {msg}'
  if status in (DINO_ERR_ARG, DINO_ERR_SHAPE):
    raise ValueError(msg)
  if status == DINO_ERR_UNSUPPORTED:
    raise NotImplementedError(msg)
  if status == DINO_ERR_NAN:
    raise DinoNonFiniteError(status, msg)
  raise DinoError(status, msg)


def dptr(array) -> ctypes.POINTER(ctypes.c_double):
  """Pointer to a contiguous float64 numpy array (caller keeps it alive)."""
  return array.ctypes.data_as(_DP)
