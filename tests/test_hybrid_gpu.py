"""GPU parity of the primitive equations on hybrid sigma-pressure levels.

The CUDA engine (hybrid column kernel + the shared transforms, modal passes
and per-wavenumber implicit operators) against the FP64 hybrid oracle
(oracle/hybrid.py), on the same FP32-rounded states.  Tolerances: max-abs
error relative to each field's maximum, 1e-4 for explicit terms (products
of several transforms, as for the sigma equations), 2e-6 for the implicit
terms and inverse (one FP32 matrix per wavenumber), 1e-4 for one filtered
SIL3 step.  The stationarity case follows the reference's
test_stationarity_sigma_like (primitive_equations_test.py:898-962) with its
tolerances.
"""

import numpy as np
import pytest
import torch

from oracle import dycore as od
from oracle import hybrid as oh
from oracle import sht as osht
from oracle import states as ost

pytestmark = pytest.mark.gpu

from dinosaur_b200 import coordinate_systems  # noqa: E402
from dinosaur_b200 import hybrid_coordinates as hc  # noqa: E402
from dinosaur_b200 import primitive_equations as pe  # noqa: E402
from dinosaur_b200 import sigma_coordinates  # noqa: E402
from dinosaur_b200 import spherical_harmonic as sh  # noqa: E402
from dinosaur_b200 import time_integration as ti  # noqa: E402
from dinosaur_b200 import units  # noqa: E402
from pe_cases import KEYS, assert_state, to_state, tracers  # noqa: E402


def make_hybrid(layers=8, levels='analytic', with_tracers=False, humidity=None,
                grid_name='T21'):
  og = getattr(osht.Grid, grid_name)()
  st, tref, orog, vert = ost.baroclinic_config(og, layers, seed=0)
  if with_tracers:
    st['tracers'] = dict(tracers(og, layers))
  rng = np.random.default_rng(7)
  _, l = og.modal_mesh
  noise = lambda n: rng.standard_normal((n,) + og.modal_shape) * og.mask / (l + 1.0) ** 2
  st['vorticity'] = st['vorticity'] + 1e-3 * noise(layers)
  st['divergence'] = st['divergence'] + 1e-3 * noise(layers)
  st['log_surface_pressure'] = st['log_surface_pressure'] + 1e-3 * noise(1)
  st = od.tree_map(lambda x: np.asarray(x, np.float32).astype(np.float64), st)
  if levels == 'analytic':
    olev = oh.HybridCoordinates.analytic_levels(layers)
  elif levels == 'ecmwf_like':
    # pure-pressure layers (b = 0) above 80 hPa, hybrid below
    e = hc.HybridCoordinates.analytic_ecmwf_like(layers)
    olev = oh.HybridCoordinates(np.asarray(e.a_boundaries, np.float64),
                                np.asarray(e.b_boundaries, np.float64))
  else:
    olev = oh.HybridCoordinates.from_sigma_levels(vert)
  oeq = oh.PrimitiveEquationsHybrid(tref, orog, og, olev, od.SimUnits(),
                                    humidity_key=humidity)
  g = getattr(sh.Grid, grid_name)()
  coords = coordinate_systems.CoordinateSystem(
      g, hc.HybridCoordinates(olev.a_boundaries, olev.b_boundaries))
  eq = pe.PrimitiveEquationsHybrid(tref, orog.astype(np.float32), coords,
                                   units.SimUnits(), humidity_key=humidity)
  return og, oeq, st, g, eq


@pytest.mark.parametrize('layers,levels', [(8, 'analytic'), (20, 'analytic'),
                                           (20, 'ecmwf_like')])
def test_explicit_terms_match_oracle(layers, levels):
  og, oeq, st, g, eq = make_hybrid(layers, levels=levels)
  got = eq.explicit_terms(to_state(st))
  assert_state(got, oeq.explicit_terms(st), 1e-4)
  for k in KEYS:
    assert float(getattr(got, k)[..., -1].abs().max()) == 0.0


def test_moist_explicit_terms_with_tracer_match_oracle():
  og, oeq, st, g, eq = make_hybrid(8, with_tracers=True, humidity='specific_humidity')
  assert_state(eq.explicit_terms(to_state(st)), oeq.explicit_terms(st), 1e-4)


def test_implicit_terms_and_inverse_match_oracle():
  og, oeq, st, g, eq = make_hybrid(8)
  s = to_state(st)
  assert_state(eq.implicit_terms(s), oeq.implicit_terms(st), 2e-6)
  for eta in (0.05, 0.175008 / 4):
    assert_state(eq.implicit_inverse(s, eta), oeq.implicit_inverse(st, eta), 2e-6)


def test_one_filtered_sil3_step_matches_oracle():
  og, oeq, st, g, eq = make_hybrid(8)
  dt = 0.175008
  ostep = od.step_with_filters(od.imex_rk_sil3(oeq, dt),
                               [od.exponential_step_filter(og, dt)])
  step = ti.step_with_filters(ti.imex_rk_sil3(eq, dt),
                              [ti.exponential_step_filter(g, dt)])
  assert isinstance(step, ti.FusedSIL3Step)
  assert_state(step(to_state(st)), ostep(st), 1e-4)


def test_sigma_like_levels_match_sigma_engine():
  # On sigma-like hybrid levels the two discretisations agree except where
  # their vertical schemes differ (the T_ref vertical advection is a mass-flux
  # form on hybrid levels, a centred one on sigma levels; ~8e-3 of the
  # temperature tendency on this perturbed state).  The GPU's hybrid - sigma
  # difference must reproduce the FP64 oracles' one.
  og, oeq, st, g, eq = make_hybrid(12, levels='sigma_like')
  coords = coordinate_systems.CoordinateSystem(
      g, sigma_coordinates.SigmaCoordinates.equidistant(12))
  sig = pe.PrimitiveEquationsSigma(eq.reference_temperature, eq.orography, coords,
                                   units.SimUnits())
  osig = od.PrimitiveEquationsSigma(oeq.reference_temperature, oeq.orography, og,
                                    od.SigmaCoordinates.equidistant(12), od.SimUnits())
  s = to_state(st)
  a, b = eq.explicit_terms(s), sig.explicit_terms(s)
  oa, ob = oeq.explicit_terms(st), osig.explicit_terms(st)
  for k in KEYS:
    d_gpu = (getattr(a, k) - getattr(b, k)).double().cpu().numpy()
    d_ref = oa[k] - ob[k]
    assert np.abs(d_gpu - d_ref).max() <= 1e-4 * np.abs(ob[k]).max(), k


def test_jw_steady_state_on_sigma_like_levels_stays_stationary():
  # primitive_equations_test.py:898-962 (T42, 26 levels, dt = 600 s, 24 h).
  g = sh.Grid.with_wavenumbers(42)
  og = osht.Grid.with_wavenumbers(42)
  layers = 26
  vert = od.SigmaCoordinates.equidistant(layers)
  st, aux = ost.steady_state_jw(og, vert, od.SimUnits())
  orog = od.truncated_modal_orography(aux['orography'], og)
  lev = hc.HybridCoordinates.from_sigma_levels(
      sigma_coordinates.SigmaCoordinates.equidistant(layers))
  eq = pe.PrimitiveEquationsHybrid(aux['ref_temperatures'], orog,
                                   coordinate_systems.CoordinateSystem(g, lev),
                                   units.SimUnits())
  dt = units.nondim_time(600.0)
  step = ti.step_with_filters(ti.imex_rk_sil3(eq, dt),
                              [ti.exponential_step_filter(g, dt)])
  s0 = to_state(st)
  s = s0
  for _ in range(6):
    s = ti.repeated(step, 24)(s)
    assert float(s.divergence.abs().max()) < 8e-3
    np.testing.assert_allclose(s.vorticity.cpu().numpy(), s0.vorticity.cpu().numpy(),
                               atol=6e-3)
    np.testing.assert_allclose(s.temperature_variation.cpu().numpy(),
                               s0.temperature_variation.cpu().numpy(), atol=0.2)
    np.testing.assert_allclose(s.log_surface_pressure.cpu().numpy(),
                               s0.log_surface_pressure.cpu().numpy(), atol=5e-4)


def test_reverse_mode_and_held_suarez_are_refused():
  og, oeq, st, g, eq = make_hybrid(8)
  s = to_state(st)
  s = pe.State(s.vorticity.requires_grad_(), s.divergence, s.temperature_variation,
               s.log_surface_pressure)
  with pytest.raises(NotImplementedError):
    eq.explicit_terms(s)
  with pytest.raises(TypeError):
    pe.PrimitiveEquationsHybrid(
        eq.reference_temperature, eq.orography,
        coordinate_systems.CoordinateSystem(
            g, sigma_coordinates.SigmaCoordinates.equidistant(8)),
        units.SimUnits())


def test_members_batch_equals_single_runs():
  # The second member's surface pressure is 1 % higher everywhere: the
  # column kernel reads each member's own l = 0 coefficient of ln p_s.
  og, oeq, st, g, eq = make_hybrid(8)
  st2 = dict(st)
  st2['temperature_variation'] = st['temperature_variation'] * 0.5
  lnps = np.array(st['log_surface_pressure'])
  lnps[0, 0, 0] += np.log(1.01) * 2.0 * np.sqrt(np.pi)
  st2['log_surface_pressure'] = lnps
  s1, s2 = to_state(st), to_state(st2)
  batched = pe.State(*[torch.stack([getattr(s1, k), getattr(s2, k)]) for k in KEYS])
  out = eq.explicit_terms(batched)
  for i, s in enumerate((s1, s2)):
    single = eq.explicit_terms(s)
    for k in KEYS:
      torch.testing.assert_close(getattr(out, k)[i], getattr(single, k), rtol=0, atol=0)
  # and the second member matches the oracle on its own
  assert_state(eq.explicit_terms(s2), oeq.explicit_terms(st2), 1e-4)


def test_graph_replay_equals_eager():
  og, oeq, st, g, eq = make_hybrid(8)
  dt = 0.175008
  s = to_state(st)
  eager = ti.FusedSIL3Step(eq, dt, n_steps=3, use_graph=False)(s)
  graph = ti.FusedSIL3Step(eq, dt, n_steps=3, use_graph=True)(s)
  for k in KEYS:
    assert torch.equal(getattr(eager, k), getattr(graph, k)), k


def test_implicit_vjps_pass_the_dot_test():
  # The implicit terms and their inverse are linear; their VJPs (transposed
  # per-wavenumber operators with the hybrid ln p_s column and thickness row)
  # satisfy <w, A v> = <A^T w, v> to FP32 rounding (<= 1e-5 relative).
  og, oeq, st, g, eq = make_hybrid(8)
  rng = np.random.default_rng(3)
  _, l = og.modal_mesh
  def rand_state():
    f = lambda n: torch.as_tensor(
        (rng.standard_normal((n,) + og.modal_shape) * og.mask / (l + 1.0)).astype(np.float32),
        device='cuda')
    return pe.State(f(8), f(8), f(8), f(1))
  dot = lambda a, b: sum(float((getattr(a, k).double() * getattr(b, k).double()).sum())
                         for k in KEYS)
  for op in (eq.implicit_terms, lambda s: eq.implicit_inverse(s, 0.05)):
    v, w = rand_state(), rand_state()
    x = pe.State(*[getattr(v, k).clone().requires_grad_() for k in KEYS])
    y = op(x)
    loss = sum((getattr(y, k) * getattr(w, k)).sum() for k in KEYS)
    loss.backward()
    lhs = dot(w, op(v))
    rhs = sum(float((getattr(x, k).grad.double() * getattr(v, k).double()).sum()) for k in KEYS)
    assert abs(lhs - rhs) <= 1e-5 * max(abs(lhs), abs(rhs)), (lhs, rhs)


def test_engine_matches_reference_golden_vectors():
  # The reference's own PrimitiveEquationsHybrid, run in float64
  # (tests/golden/pe_hybrid_T21_L6.npz: 6 analytic levels), against the CUDA
  # engine fed the FP32-rounded input state (that rounding alone moves the
  # small ln p_s tendency by 1.1e-5 of its maximum, the rest by <= 4e-7).
  import os
  gdir = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')
  g0 = np.load(os.path.join(gdir, 'pe_T21_L6.npz'))
  g = np.load(os.path.join(gdir, 'pe_hybrid_T21_L6.npz'))
  grid = sh.Grid.T21()
  coords = coordinate_systems.CoordinateSystem(
      grid, hc.HybridCoordinates(g['a_boundaries'], g['b_boundaries']))
  eq = pe.PrimitiveEquationsHybrid(g0['ref_temps'], g0['orography'].astype(np.float32),
                                   coords, units.SimUnits())
  s = pe.State(*[torch.as_tensor(g0['in_' + k], device='cuda', dtype=torch.float32)
                 for k in KEYS])
  ref = lambda prefix: dict({k: g[f'{prefix}_{k}'] for k in KEYS}, tracers={})
  assert_state(eq.explicit_terms(s), ref('explicit'), 1e-4)
  assert_state(eq.implicit_terms(s), ref('implicit'), 1e-5)
  assert_state(eq.implicit_inverse(s, 0.05), ref('inverse'), 1e-5)
  dt = 0.175008
  step = ti.step_with_filters(ti.imex_rk_sil3(eq, dt), [ti.exponential_step_filter(grid, dt)])
  assert_state(step(s), ref('step1'), 1e-4)
