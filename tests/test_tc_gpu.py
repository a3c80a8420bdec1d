"""GPU parity of the tcgen05 split-operand Legendre contractions.

The 'bf16x3' and 'tf32x3' plans run the Legendre GEMMs on tensor cores with
hi*hi + hi*lo + lo*hi products of bf16 or tf32 splits, accumulated in FP32.
Tolerances against the FP64 oracle for one-way transforms and round trips:
split-BF16 relative L2 <= 1e-5 (the target accuracy of the split form) and
max-abs relative <= 5e-5; split-TF32 (11-bit halves, the dropped lo*lo term
~2^-22 relative) relative L2 <= 2e-6 and max-abs relative <= 1e-5.
"""

import numpy as np
import pytest
import torch

from oracle import sht as osht
from oracle import states as ost

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _tensor_cores_only(monkeypatch):
  # These tests exercise the tensor-core kernels themselves: keep them even
  # on grids where the plan's autotuner would pick the FP32 SIMT contraction.
  monkeypatch.setenv('DINO_B200_TENSOR_CORES_ONLY', '1')

from dinosaur_b200 import _lib  # noqa: E402
from dinosaur_b200 import spherical_harmonic as sh  # noqa: E402


FORMS = ['bf16x3', 'tf32x3']
TOL = {'bf16x3': (1e-5, 5e-5), 'tf32x3': (2e-6, 1e-5)}  # (rel L2, max-abs rel)


def tc_grid(name, precision='bf16x3'):
  impl = lambda **kw: sh.CudaSphericalHarmonics(precision=precision, **kw)
  return getattr(sh.Grid, name)(spherical_harmonics_impl=impl)


def l2(a, b):
  a = a.detach().double().cpu().numpy() if torch.is_tensor(a) else a
  return np.linalg.norm(a - b) / np.linalg.norm(b)


def maxrel(a, b):
  a = a.detach().double().cpu().numpy() if torch.is_tensor(a) else a
  return np.abs(a - b).max() / np.abs(b).max()


@pytest.mark.parametrize('precision', FORMS)
@pytest.mark.parametrize('name', ['T21', 'T42', 'T85', 'TL127', 'TL255'])
def test_tc_transforms_match_fp64_oracle(name, precision):
  g = tc_grid(name, precision)
  tl2, tmax = TOL[precision]
  og = getattr(osht.Grid, name)()
  nf = 4 if name != 'TL255' else 3
  x = ost.sht_modal_input(og, nf, seed=3)
  x64 = x.astype(np.float64)
  nodal = g.to_nodal(torch.as_tensor(x, device='cuda'))
  _lib.check(_lib.lib().dino_plan_status(g.plan.handle))
  ref = og.to_nodal(x64)
  assert l2(nodal, ref) < tl2 and maxrel(nodal, ref) < tmax
  z = np.random.default_rng(4).standard_normal((nf,) + og.nodal_shape)
  modal = g.to_modal(torch.as_tensor(z, device='cuda', dtype=torch.float32))
  _lib.check(_lib.lib().dino_plan_status(g.plan.handle))
  refm = og.to_modal(z.astype(np.float32).astype(np.float64))
  assert l2(modal, refm) < tl2 and maxrel(modal, refm) < tmax
  assert np.all(modal.cpu().numpy()[:, ~og.mask] == 0)


@pytest.mark.parametrize('precision', FORMS)
@pytest.mark.parametrize('n,spacing', [(24, 'gauss'), (24, 'equiangular_with_poles'),
                                       (62, 'gauss')])
def test_tc_transforms_on_ragged_latitude_blocks(n, spacing, precision):
  # J = 37 (odd: a self-mirrored middle latitude, 19 latitude pairs) and
  # J = 94 (47 pairs, J not a multiple of 4): partial 16-latitude blocks take
  # the row-store epilogue and the operands the scalar (non-float4) paths.
  tl2, tmax = TOL[precision]
  impl = lambda **kw: sh.CudaSphericalHarmonics(precision=precision, **kw)
  g = sh.Grid.with_wavenumbers(n, latitude_spacing=spacing, spherical_harmonics_impl=impl)
  og = osht.Grid.with_wavenumbers(n, latitude_spacing=spacing)
  x = ost.sht_modal_input(og, 3, seed=9)
  nodal = g.to_nodal(torch.as_tensor(x, device='cuda'))
  _lib.check(_lib.lib().dino_plan_status(g.plan.handle))
  ref = og.to_nodal(x.astype(np.float64))
  assert l2(nodal, ref) < tl2 and maxrel(nodal, ref) < tmax
  z = np.random.default_rng(10).standard_normal((3,) + og.nodal_shape)
  modal = g.to_modal(torch.as_tensor(z, device='cuda', dtype=torch.float32))
  _lib.check(_lib.lib().dino_plan_status(g.plan.handle))
  refm = og.to_modal(z.astype(np.float32).astype(np.float64))
  assert l2(modal, refm) < tl2 and maxrel(modal, refm) < tmax


@pytest.mark.parametrize('precision', FORMS)
def test_tc_matches_fp32_plan_on_large_batch(precision):
  g = tc_grid('TL255', precision)
  f = sh.Grid.TL255()
  og = osht.Grid.TL255()
  x = torch.as_tensor(ost.sht_modal_input(og, 128, seed=0), device='cuda')
  a = g.to_modal(g.to_nodal(x))
  b = f.to_modal(f.to_nodal(x))
  _lib.check(_lib.lib().dino_plan_status(g.plan.handle))
  err_tc = float(torch.linalg.vector_norm(a - x) / torch.linalg.vector_norm(x))
  err_fp = float(torch.linalg.vector_norm(b - x) / torch.linalg.vector_norm(x))
  assert err_tc < TOL[precision][0], err_tc
  assert err_fp < 1e-5, err_fp


@pytest.mark.parametrize('precision', FORMS)
def test_tc_primitive_equations_match_fp64_oracle(precision):
  """Explicit terms, one filtered SIL3 step and the step VJP on a
  split-operand grid (moist, with a passive tracer) against the FP64 oracle.
  A tendency composes several transforms (each <= 5e-5 max-abs, <= 1e-5 L2,
  tested above) with products and derivatives, and small tendencies (the
  vorticity tendency is a difference of curls of large fluxes) carry the
  absolute error of the large fields, so per field: max-abs error relative
  to the field's max <= 1e-4 (explicit terms) or to max(|y_next|, dt |F|)
  (one step); the VJP dot test <= 1e-4."""
  from oracle import dycore as od
  from dinosaur_b200 import coordinate_systems, primitive_equations as pe
  from dinosaur_b200 import sigma_coordinates, time_integration as ti, units
  from pe_cases import KEYS, assert_state, make, to_state, tracers
  og, oeq, st, _, _ = make(tracers=tracers, humidity='specific_humidity')
  g = tc_grid('T21', precision)
  coords = coordinate_systems.CoordinateSystem(
      g, sigma_coordinates.SigmaCoordinates.equidistant(6))
  eq = pe.PrimitiveEquationsSigma(oeq.reference_temperature,
                                  np.asarray(oeq.orography, np.float32), coords,
                                  units.SimUnits(),
                                  humidity_key='specific_humidity')
  def check(got, ref):
    assert_state(got, ref, 1e-4)
  check(eq.explicit_terms(to_state(st)), oeq.explicit_terms(st))
  dt = 0.175008
  step = ti.step_with_filters(ti.imex_rk_sil3(eq, dt),
                              [ti.exponential_step_filter(g, dt)])
  ostep = od.step_with_filters(od.imex_rk_sil3(oeq, dt),
                               [od.exponential_step_filter(og, dt)])
  # One step: a step's error is ~eps * dt * |F|, and the balanced state's
  # divergence is far smaller than dt * its tendency, so each field's error
  # is measured against max(|y_next|, dt |F(y0)|).
  got, ref, f0 = step(to_state(st)), ostep(st), oeq.explicit_terms(st)
  for k in KEYS:
    a = getattr(got, k).double().cpu().numpy()
    scale = max(np.abs(ref[k]).max(), dt * np.abs(f0[k]).max())
    assert np.abs(a - ref[k]).max() <= 1e-4 * scale, k
  _lib.check(_lib.lib().dino_plan_status(g.plan.handle))
  from test_adjoint_gpu import central_dot, gpu_vjp, random_tree, tree_dot
  rng = np.random.default_rng(21)
  w = random_tree(og, st, rng)
  v = random_tree(og, st, rng)
  lhs = tree_dot(gpu_vjp(step, st, w), v)
  rhs = central_dot(ostep, st, w, v)
  assert abs(lhs - rhs) <= 1e-4 * abs(rhs), (lhs, rhs)


@pytest.mark.parametrize('precision,form', [('bf16x3', 'split-BF16'), ('tf32x3', 'split-TF32')])
def test_autotuner_records_its_choice(precision, form):
  """A split-operand plan times its candidate launch shapes at creation and
  keeps the fastest; the choice and its time are reported."""
  g = tc_grid('TL255', precision)
  d = g.plan.describe()
  assert 'autotuned' in d and 'shapes tried per m range' in d, d
  assert form in d
  assert 'FP32 (SIMT)' in sh.Grid.T21().plan.describe()


def test_autotuner_may_pick_fp32_simt_and_stays_accurate(monkeypatch):
  """Without the override the plan times the FP32 SIMT contraction beside
  the tensor-core shapes and runs whichever is faster per direction (on
  small grids often SIMT); either way the result meets the split form's
  bound."""
  monkeypatch.delenv('DINO_B200_TENSOR_CORES_ONLY', raising=False)
  g = tc_grid('T42', 'bf16x3')
  desc = g.plan.describe()
  assert 'FP32 SIMT' in desc, desc
  og = osht.Grid.T42()
  x = ost.sht_modal_input(og, 8, seed=5)
  nodal = g.to_nodal(torch.as_tensor(x, device='cuda'))
  ref = og.to_nodal(x.astype(np.float64))
  assert l2(nodal, ref) < TOL['bf16x3'][0]
  modal = g.to_modal(nodal)
  refm = og.to_modal(ref)
  assert l2(modal, refm) < TOL['bf16x3'][0]


@pytest.mark.parametrize('precision', FORMS)
@pytest.mark.parametrize('name', ['T85', 'TL255'])
def test_two_m_group_launches_match_fp64_oracle(name, precision, monkeypatch):
  """The per-m-range arrangement (low and high zonal wavenumbers launched
  with shapes of their own) gives the same accuracy as one launch."""
  monkeypatch.setenv('DINO_B200_TC_M_GROUPS', '2')
  g = tc_grid(name, precision)
  assert g.plan.describe().count(' m ') >= 4  # two groups in each direction
  tl2, tmax = TOL[precision]
  og = getattr(osht.Grid, name)()
  x = ost.sht_modal_input(og, 5, seed=8)
  nodal = g.to_nodal(torch.as_tensor(x, device='cuda'))
  _lib.check(_lib.lib().dino_plan_status(g.plan.handle))
  ref = og.to_nodal(x.astype(np.float64))
  assert l2(nodal, ref) < tl2 and maxrel(nodal, ref) < tmax
  modal = g.to_modal(nodal)
  refm = og.to_modal(ref)
  assert l2(modal, refm) < tl2 and maxrel(modal, refm) < tmax
