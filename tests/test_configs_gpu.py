"""GPU parity at the benchmark configurations' stated sizes.

Each case runs the CUDA path through the C ABI in FP32 (or a split tensor-core
form) on the configuration's own inputs and compares it with the FP64 oracle,
which runs in spawned worker processes while the GPU works.  Errors are
max-abs differences relative to each field's max-abs FP64 value, per member;
relative L2 norms for the one-day rollout.  Bounds (written per test):

* Held-Suarez ensemble, T42 / 24 levels, 16 members in one batch, 3 filtered
  SIL3 steps: FP32 <= 5e-5 (measured 1.9e-5 in the divergence; with 24
  levels the FP32 rounding of the column sums spreads over the levels, as in
  the 24-level explicit-terms test); split-BF16 <= 2e-4 (measured 7.6e-5:
  its transforms carry ~4e-6 relative error one way).
* Large moist, TL255 / 32 levels, specific humidity and two log-normal
  tracers, 4 members in one batch, one filtered step, FP32 and split-BF16
  against the same FP64 runs: every field <= 2e-5 max-abs and <= 1e-5
  relative L2, except the divergence.  The divergence of the balanced JW
  state is ~4 % of the vorticity's magnitude and its tendency a small
  residual of large cancelling terms, so the transforms' relative error
  reaches it amplified: split-BF16 (~4e-6 one way) measured 1.25e-3 max-abs
  and 9.1e-5 relative L2, bounded by 2.5e-3 and 2e-4; FP32 by 2.5e-4 and
  2e-5.
* The split-BF16 step VJP at that size (one member): the dot test
  <J^T w, v> against <w, J v> from FP64 central differences, <= 1e-4.
* The one-day rollout (T21 / 12 levels, 72 steps) in split-BF16 against FP64:
  relative L2 <= 5e-3 for the divergence (the balanced residual field; FP32
  gives ~8e-5) and <= 1e-4 for the other fields.
"""

import functools

import numpy as np
import pytest
import torch

from oracle import dycore as od
from oracle import states as ost

import config_cases as cc

pytestmark = pytest.mark.gpu

from dinosaur_b200 import coordinate_systems  # noqa: E402
from dinosaur_b200 import held_suarez  # noqa: E402
from dinosaur_b200 import primitive_equations as pe  # noqa: E402
from dinosaur_b200 import sigma_coordinates  # noqa: E402
from dinosaur_b200 import spherical_harmonic as sh  # noqa: E402
from dinosaur_b200 import time_integration as ti  # noqa: E402
from dinosaur_b200 import units  # noqa: E402

from pe_cases import KEYS, make, to_state  # noqa: E402


def gpu_grid(grid_name, precision):
  impl = functools.partial(sh.CudaSphericalHarmonics, precision=precision)
  return getattr(sh.Grid, grid_name)(spherical_harmonics_impl=impl)


def gpu_equation(g, layers, tref, orog, humidity=None, held_suarez_forcing=False):
  coords = coordinate_systems.CoordinateSystem(
      g, sigma_coordinates.SigmaCoordinates.equidistant(layers))
  eq = pe.PrimitiveEquationsSigma(tref, np.asarray(orog, np.float32), coords,
                                  units.SimUnits(), humidity_key=humidity)
  if held_suarez_forcing:
    eq = ti.compose_equations(
        [eq, held_suarez.HeldSuarezForcingSigma(coords, units.SimUnits(), tref)])
  return eq


def stacked_state(members):
  """Members stacked on a leading axis (the engine's batched layout)."""
  t = lambda xs: torch.as_tensor(np.stack(xs), device='cuda', dtype=torch.float32)
  return pe.State(*[t([m[k] for m in members]) for k in KEYS],
                  tracers={n: t([m['tracers'][n] for m in members])
                           for n in members[0]['tracers']})


def member_errors(got, ref, i):
  """Per-field max-abs error relative to the field's max-abs FP64 value."""
  out = {}
  for k in KEYS:
    a = getattr(got, k)[i].double().cpu().numpy()
    out[k] = np.abs(a - ref[k]).max() / max(np.abs(ref[k]).max(), 1e-30)
  for n, r in ref['tracers'].items():
    a = got.tracers[n][i].double().cpu().numpy()
    out[n] = np.abs(a - r).max() / max(np.abs(r).max(), 1e-30)
  return out


def member_l2(got, ref, i):
  out = {}
  for k in KEYS:
    a = getattr(got, k)[i].double().cpu().numpy()
    out[k] = np.linalg.norm(a - ref[k]) / np.linalg.norm(ref[k])
  for n, r in ref['tracers'].items():
    a = got.tracers[n][i].double().cpu().numpy()
    out[n] = np.linalg.norm(a - r) / np.linalg.norm(r)
  return out


@pytest.mark.parametrize('precision,tol', [('fp32', 5e-5), ('bf16x3', 2e-4)])
def test_held_suarez_ensemble_t42_l24_x16(precision, tol):
  """16 Held-Suarez members (rest at 285 K + 0.1 K white noise, seed = member)
  in one batch, 3 filtered SIL3 steps, against 16 FP64 oracle runs."""
  members, layers, n_steps = 16, 24, 3
  with cc.oracle_pool(8) as pool:
    futs = [pool.submit(cc.hs_oracle_rollout, i, n_steps) for i in range(members)]
    inputs = [cc.hs_member(i) for i in range(members)]
    _, _, tref, orog, _ = inputs[0]
    g = gpu_grid('T42', precision)
    eq = gpu_equation(g, layers, tref, orog, held_suarez_forcing=True)
    flt = ti.exponential_step_filter(g, cc.HS_DT, **cc.HS_FILTER)
    step = ti.repeated(ti.step_with_filters(ti.imex_rk_sil3(eq, cc.HS_DT), [flt]),
                       n_steps)
    got = step(stacked_state([x[1] for x in inputs]))
    torch.cuda.synchronize()
    refs = [f.result() for f in futs]
  worst = {}
  for i, ref in enumerate(refs):
    for k, e in member_errors(got, ref, i).items():
      worst[k] = max(worst.get(k, 0.0), e)
  print(f'\nHeld-Suarez T42/24 x16, {precision}, worst member max-abs rel:', worst)
  for k, e in worst.items():
    assert e <= tol, (k, e)


def test_large_moist_tl255_l32_x4():
  """TL255 / 32 levels, humidity + 2 log-normal tracers, 4 members in one
  batch, one filtered step in FP32 and in split-BF16 against FP64 per
  member.  Also covers the largest planes the nodal kernels address with
  32-bit offsets (4 members x 3 tracers at TL255)."""
  members, layers = 4, 32
  bounds = {'fp32': (2.5e-4, 2e-5), 'bf16x3': (2.5e-3, 2e-4)}  # divergence
  with cc.oracle_pool(members) as pool:
    futs = [pool.submit(cc.large_oracle_rollout, i, 1) for i in range(members)]
    inputs = [cc.large_member(i) for i in range(members)]
    _, _, tref, orog, _ = inputs[0]
    outs = {}
    for precision in bounds:
      g = gpu_grid('TL255', precision)
      eq = gpu_equation(g, layers, tref, orog, humidity='specific_humidity')
      step = ti.step_with_filters(ti.imex_rk_sil3(eq, cc.LARGE_DT),
                                  [ti.exponential_step_filter(g, cc.LARGE_DT)])
      outs[precision] = step(stacked_state([x[1] for x in inputs]))
    torch.cuda.synchronize()
    refs = [f.result() for f in futs]
  for precision, got in outs.items():
    worst, worst_l2 = {}, {}
    for i, ref in enumerate(refs):
      for k, e in member_errors(got, ref, i).items():
        worst[k] = max(worst.get(k, 0.0), e)
      for k, e in member_l2(got, ref, i).items():
        worst_l2[k] = max(worst_l2.get(k, 0.0), e)
    print(f'\nTL255/32 moist x4 {precision}, worst member max-abs rel:', worst)
    print(f'TL255/32 moist x4 {precision}, worst member rel L2:', worst_l2)
    div_max, div_l2 = bounds[precision]
    for k, e in worst.items():
      assert e <= (div_max if k == 'divergence' else 2e-5), (precision, k, e)
    for k, e in worst_l2.items():
      assert e <= (div_l2 if k == 'divergence' else 1e-5), (precision, k, e)


def _random_tree(og, like, rng):
  _, l = og.modal_mesh
  noise = lambda a: rng.standard_normal(a.shape) * og.mask / (l + 1.0)
  out = {k: noise(like[k]) for k in KEYS}
  out['tracers'] = {n: noise(a) for n, a in like['tracers'].items()}
  return out


def _tree_dot(a, b):
  return (sum(float(np.sum(a[k] * b[k])) for k in KEYS) +
          sum(float(np.sum(a['tracers'][n] * b['tracers'][n])) for n in a['tracers']))


def test_large_moist_step_vjp_dot_bf16x3():
  """The split-BF16 filtered-step VJP at TL255 / 32 levels with humidity and
  two tracers: <J^T w, v> (hand-written adjoint kernels) against <w, J v>
  (FP64 central differences of the oracle step, eps = 1e-6)."""
  og, st, tref, orog, _ = cc.large_member(0)
  rng = np.random.default_rng(21)
  w = _random_tree(og, st, rng)
  v = _random_tree(og, st, rng)
  with cc.oracle_pool(1) as pool:
    fut = pool.submit(cc.large_oracle_step_jvp, 0, v, 1e-6)
    g = gpu_grid('TL255', 'bf16x3')
    eq = gpu_equation(g, 32, tref, orog, humidity='specific_humidity')
    step = ti.step_with_filters(ti.imex_rk_sil3(eq, cc.LARGE_DT),
                                [ti.exponential_step_filter(g, cc.LARGE_DT)])
    x = to_state(st)
    leaves = [getattr(x, k) for k in KEYS] + [x.tracers[n] for n in x.tracers]
    for t in leaves:
      t.requires_grad_(True)
    y = step(x)
    wt = to_state(w)
    wl = [getattr(wt, k) for k in KEYS] + [wt.tracers[n] for n in wt.tracers]
    yl = [getattr(y, k) for k in KEYS] + [y.tracers[n] for n in y.tracers]
    loss = sum((a.double() * b.double()).sum() for a, b in zip(yl, wl))
    grads = torch.autograd.grad(loss, leaves)
    gd = {k: gr.double().cpu().numpy() for k, gr in zip(KEYS, grads)}
    gd['tracers'] = {n: gr.double().cpu().numpy()
                     for n, gr in zip(st['tracers'], grads[len(KEYS):])}
    jv = fut.result()
  lhs = _tree_dot(gd, v)
  rhs = _tree_dot(w, jv)
  print(f'\nTL255/32 moist bf16x3 step VJP dot: {lhs!r} vs {rhs!r}, '
        f'rel {abs(lhs - rhs) / abs(rhs):.3e}')
  assert abs(lhs - rhs) <= 1e-4 * abs(rhs), (lhs, rhs)


def test_one_day_t21_l12_bf16x3_end_state():
  """The T21 / 12-level day (JW + 1 K bump, dt = 20 min, 72 steps) with the
  split-BF16 Legendre contraction, against the FP64 end state."""
  og, oeq, st, _, _ = make('T21', 12, perturb=False)
  _, tref, orog, _ = ost.baroclinic_config(og, 12)
  dt = 0.175008
  g = gpu_grid('T21', 'bf16x3')
  eq = gpu_equation(g, 12, tref, orog)
  step = ti.repeated(ti.step_with_filters(ti.imex_rk_sil3(eq, dt),
                                          [ti.exponential_step_filter(g, dt)]), 72)
  got = step(to_state(st))
  ostep = od.step_with_filters(od.imex_rk_sil3(oeq, dt),
                               [od.exponential_step_filter(og, dt)])
  ref = od.repeated(ostep, 72)(st)
  errs = {}
  for k in KEYS:
    a = getattr(got, k).double().cpu().numpy()
    errs[k] = np.linalg.norm(a - ref[k]) / np.linalg.norm(ref[k])
  print('\nT21/12 one day bf16x3, rel L2:', errs)
  for k, e in errs.items():
    assert e <= (5e-3 if k == 'divergence' else 1e-4), (k, e)
