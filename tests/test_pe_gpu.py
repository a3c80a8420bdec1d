"""GPU parity of the primitive-equation step against the FP64 oracle.

All CUDA results go through the C ABI (``libdino_b200.so``) in FP32 and are
compared with the oracle on the same inputs.  Tolerances (written per test):
single evaluations <= 2e-5 max-abs error relative to each field's max-abs
FP64 value; one full filtered SIL3 step <= 2e-5; reference identities use
the reference test's own tolerances.
"""

import numpy as np
import pytest
import torch

from oracle import dycore as od
from oracle import sht as osht
from oracle import states as ost

pytestmark = pytest.mark.gpu

from dinosaur_b200 import coordinate_systems  # noqa: E402
from dinosaur_b200 import held_suarez  # noqa: E402
from dinosaur_b200 import primitive_equations as pe  # noqa: E402
from dinosaur_b200 import sigma_coordinates  # noqa: E402
from dinosaur_b200 import spherical_harmonic as sh  # noqa: E402
from dinosaur_b200 import time_integration as ti  # noqa: E402
from dinosaur_b200 import units  # noqa: E402

from pe_cases import KEYS, assert_state, make, rel, to_state  # noqa: E402
from pe_cases import tracers as _tracers  # noqa: E402


def test_constants_match_oracle():
  ps, ops = units.SimUnits(), od.SimUnits()
  for k in ('angular_velocity', 'g', 'R', 'R_vapor', 'Cp_vapor', 'kappa'):
    assert getattr(ps, k) == pytest.approx(getattr(ops, k), rel=1e-15)
  vert = sigma_coordinates.SigmaCoordinates.equidistant(12)
  overt = od.SigmaCoordinates.equidistant(12)
  np.testing.assert_array_equal(vert.centers, overt.centers)
  np.testing.assert_allclose(
      pe.get_temperature_implicit_weights_sigma(vert, np.linspace(200, 290, 12),
                                                0.28),
      od.get_temperature_implicit_weights(overt, np.linspace(200, 290, 12), 0.28))


def test_explicit_terms_match_oracle():
  og, oeq, st, g, eq = make()
  got = eq.explicit_terms(to_state(st))
  ref = oeq.explicit_terms(st)
  assert_state(got, ref, 2e-5)
  # The top total wavenumber is clipped exactly.
  for k in KEYS:
    assert float(getattr(got, k)[..., -1].abs().max()) == 0.0


def test_implicit_terms_and_inverse_match_oracle():
  og, oeq, st, g, eq = make()
  s = to_state(st)
  assert_state(eq.implicit_terms(s), oeq.implicit_terms(st), 2e-6)
  for eta in (0.05, 0.175008 / 4):
    assert_state(eq.implicit_inverse(s, eta), oeq.implicit_inverse(st, eta),
                 2e-6)


@pytest.mark.parametrize('params', [
    dict(lw=16, layers=5, tref=np.linspace(100, 200, 5), kappa=1.4, R=33.0,
         eta=0.3, seed=0),
    dict(lw=128, layers=23, tref=np.linspace(250, 300, 23), kappa=111.0,
         R=1.0, eta=0.1, seed=1),
])
def test_reference_primitive_inverse_identity(params):
  # primitive_equations_test.py:578-658: inverse(x - eta G(x)) == x, atol 1e-5.
  g = sh.Grid.with_wavenumbers(params['lw'])
  vert = sigma_coordinates.SigmaCoordinates.equidistant(params['layers'])
  coords = coordinate_systems.CoordinateSystem(g, vert)
  ps = units.SimUnits.from_si(ideal_gas_constant_si=params['R'],
                              kappa_si=params['kappa'])
  rng = np.random.default_rng(params['seed'])
  scale = (g.total_wavenumbers + 1) ** -2
  shp = coords.modal_shape
  t = lambda a: torch.as_tensor(a, device='cuda', dtype=torch.float32)
  state = pe.State(t(scale * rng.standard_normal(shp)),
                   t(scale * rng.standard_normal(shp)),
                   t(scale * rng.standard_normal(shp)),
                   t(scale * rng.standard_normal(coords.surface_modal_shape)))
  eq = pe.PrimitiveEquationsSigma(params['tref'], np.zeros(g.modal_shape),
                                  coords, ps)
  x = state - params['eta'] * eq.implicit_terms(state)
  back = eq.implicit_inverse(x, params['eta'])
  for k in KEYS:
    np.testing.assert_allclose(getattr(back, k).cpu().numpy(),
                               getattr(state, k).cpu().numpy(), atol=1e-5)
  with pytest.raises(TypeError):
    eq.implicit_inverse(x, torch.tensor(0.3))


def test_one_filtered_sil3_step_matches_oracle():
  og, oeq, st, g, eq = make()
  dt = 0.175008
  ostep = od.step_with_filters(od.imex_rk_sil3(oeq, dt),
                               [od.exponential_step_filter(og, dt)])
  step = ti.step_with_filters(ti.imex_rk_sil3(eq, dt),
                              [ti.exponential_step_filter(g, dt)])
  assert isinstance(step, ti.FusedSIL3Step)
  got = step(to_state(st))
  ref = ostep(st)
  assert_state(got, ref, 5e-5)


def test_generic_imex_path_matches_fused():
  og, oeq, st, g, eq = make()
  dt = 0.175008
  generic = ti.imex_runge_kutta(ti.SIL3_TABLEAU, eq, dt)
  fused = ti.imex_rk_sil3(eq, dt)
  s = to_state(st)
  a = generic(s)
  b = fused(s)
  for k in KEYS:
    assert rel(getattr(a, k), getattr(b, k).double().cpu().numpy()) < 1e-5


def test_graph_replay_equals_eager():
  og, oeq, st, g, eq = make()
  dt = 0.175008
  s = to_state(st)
  eager = ti.FusedSIL3Step(eq, dt, n_steps=3, use_graph=False)(s)
  graph = ti.FusedSIL3Step(eq, dt, n_steps=3, use_graph=True)(s)
  for k in KEYS:
    assert torch.equal(getattr(eager, k), getattr(graph, k)), k


@pytest.mark.parametrize('start_with_input', [False, True])
def test_trajectory_frames_equal_repeated_steps(start_with_input):
  """trajectory_from_step (time_integration.py:523-564) on the fused step:
  the native rollout's frames equal the states of repeated graph steps
  bit for bit; sim_time advances per frame; post_process_fn maps frames."""
  og, oeq, st, g, eq = make(tracers=_tracers, humidity='specific_humidity')
  dt = 0.175008
  step = ti.step_with_filters(ti.imex_rk_sil3(eq, dt),
                              [ti.exponential_step_filter(g, dt)])
  outer, inner = 3, 2
  x = to_state(st)
  x = pe.State(x.vorticity, x.divergence, x.temperature_variation,
               x.log_surface_pressure, tracers=x.tracers, sim_time=1.5)
  final, frames = ti.trajectory_from_step(
      step, outer, inner, start_with_input=start_with_input)(x)
  assert frames.vorticity.shape == (outer,) + tuple(x.vorticity.shape)
  assert frames.tracers['tracer_a'].shape[0] == outer
  ref = x
  expected = []
  for _ in range(outer):
    nxt = ti.repeated(step, inner)(ref)
    expected.append(ref if start_with_input else nxt)
    ref = nxt
  for i, e in enumerate(expected):
    for k in KEYS:
      assert torch.equal(getattr(frames, k)[i], getattr(e, k)), (i, k)
    assert torch.equal(frames.tracers['specific_humidity'][i],
                       e.tracers['specific_humidity'])
  for k in KEYS:
    assert torch.equal(getattr(final, k), getattr(ref, k)), k
  first = 0 if start_with_input else 1
  np.testing.assert_allclose(
      frames.sim_time.numpy(), 1.5 + dt * inner * (np.arange(outer) + first))
  assert final.sim_time == pytest.approx(1.5 + dt * inner * outer)
  _, vort = ti.trajectory_from_step(step, outer, inner,
                                    post_process_fn=lambda s: s.vorticity)(x)
  assert torch.equal(vort, frames.vorticity if not start_with_input else
                     torch.stack([e.vorticity for e in expected[1:]] +
                                 [final.vorticity]))


def test_members_batch_equals_single_runs():
  og, oeq, st, g, eq = make()
  st2 = dict(st)
  st2['temperature_variation'] = st['temperature_variation'] * 0.5
  s1, s2 = to_state(st), to_state(st2)
  batched = pe.State(*[torch.stack([getattr(s1, k), getattr(s2, k)])
                       for k in KEYS])
  out = eq.explicit_terms(batched)
  o1 = eq.explicit_terms(s1)
  o2 = eq.explicit_terms(s2)
  for k in KEYS:
    torch.testing.assert_close(getattr(out, k)[0], getattr(o1, k), rtol=0,
                               atol=0)
    torch.testing.assert_close(getattr(out, k)[1], getattr(o2, k), rtol=0,
                               atol=0)


def test_moist_explicit_terms_with_tracers_match_oracle():
  og, oeq, st, g, eq = make(tracers=_tracers, humidity='specific_humidity')
  got = eq.explicit_terms(to_state(st))
  ref = oeq.explicit_terms(st)
  assert_state(got, ref, 2e-5)


@pytest.mark.parametrize('moist', [False, True])
def test_explicit_terms_24_levels_match_oracle(moist):
  # With 24 levels the nodal column kernel splits every column into four
  # level chunks whose column totals and sigma-dot prefix sums are exchanged
  # through shared memory (two columns per thread dry, one with tracers).
  # The FP32 error of the vorticity tendency is spread evenly over the levels
  # (measured 0.5-2.6e-5 relative to its maximum, no peak at the chunk
  # boundaries 6, 12, 18), hence 5e-5 here against 2e-5 at 6 levels.
  kw = dict(tracers=_tracers, humidity='specific_humidity') if moist else {}
  og, oeq, st, g, eq = make(layers=24, **kw)
  got = eq.explicit_terms(to_state(st))
  ref = oeq.explicit_terms(st)
  assert_state(got, ref, 5e-5)


def test_level_chunks_agree_across_batch_sizes():
  # T42 / 24 levels: one member runs four level chunks per column, a batch of
  # sixteen two (the chunk count follows the available parallelism); the
  # chunked prefix sums may differ from each other only by FP32 rounding.
  og, oeq, st, g, eq = make('T42', layers=24)
  s1 = to_state(st)
  batch = pe.State(*[torch.stack([getattr(s1, k)] * 16) for k in KEYS])
  ob = eq.explicit_terms(batch)
  o1 = eq.explicit_terms(s1)
  for k in KEYS:
    a, b = getattr(ob, k)[5].double(), getattr(o1, k).double()
    err = float((a - b).abs().max() / b.abs().max())
    assert err < 1e-6, (k, err)


def test_dry_tracer_advection_matches_oracle():
  og, oeq, st, g, eq = make(tracers=_tracers)
  got = eq.explicit_terms(to_state(st))
  ref = oeq.explicit_terms(st)
  assert_state(got, ref, 2e-5)


def test_held_suarez_composed_step_matches_oracle():
  og = osht.Grid.T21()
  layers = 6
  ost_, tref, orog, vert = ost.held_suarez_config(og, layers, member=3)
  ops = od.SimUnits()
  ohs = od.HeldSuarezForcingSigma(og, vert, ops, tref)
  opeq = od.PrimitiveEquationsSigma(tref, orog, og, vert, ops)
  ocomp = od.ComposedEquation([opeq, ohs])
  g = sh.Grid.T21()
  coords = coordinate_systems.CoordinateSystem(
      g, sigma_coordinates.SigmaCoordinates.equidistant(layers))
  peq = pe.PrimitiveEquationsSigma(tref, orog, coords, units.SimUnits())
  hs = held_suarez.HeldSuarezForcingSigma(coords, units.SimUnits(), tref)
  comp = ti.compose_equations([peq, hs])
  st = od.tree_map(lambda x: np.asarray(x, np.float32).astype(np.float64), ost_)
  # small flow so that the drag terms are exercised
  rng = np.random.default_rng(5)
  noise = rng.standard_normal((layers,) + og.modal_shape) * og.mask / 1e3
  st['vorticity'] = (st['vorticity'] + noise).astype(np.float32).astype(np.float64)
  st['divergence'] = (st['divergence'] + noise[::-1]).astype(np.float32).astype(np.float64)
  got = comp.explicit_terms(to_state(st))
  assert_state(got, ocomp.explicit_terms(st), 2e-5)
  dt = 0.131256
  oflt = od.exponential_step_filter(og, dt, tau=0.0087504, order=1.5, cutoff=0.8)
  flt = ti.exponential_step_filter(g, dt, tau=0.0087504, order=1.5, cutoff=0.8)
  ref = od.step_with_filters(od.imex_rk_sil3(ocomp, dt), [oflt])(st)
  out = ti.step_with_filters(ti.imex_rk_sil3(comp, dt), [flt])(to_state(st))
  assert_state(out, ref, 2e-5)


def test_held_suarez_forcing_standalone_matches_oracle():
  """HeldSuarezForcingSigma evaluated on its own (held_suarez.py:105-167):
  kt, equilibrium_temperature and explicit_terms against the oracle, and the
  fused composition equal to the primitive equations' tendencies plus the
  standalone forcing."""
  og = osht.Grid.T21()
  layers = 6
  ost_, tref, orog, vert = ost.held_suarez_config(og, layers, member=2)
  ops = od.SimUnits()
  ohs = od.HeldSuarezForcingSigma(og, vert, ops, tref)
  g = sh.Grid.T21()
  coords = coordinate_systems.CoordinateSystem(
      g, sigma_coordinates.SigmaCoordinates.equidistant(layers))
  hs = held_suarez.HeldSuarezForcingSigma(coords, units.SimUnits(), tref)
  np.testing.assert_allclose(hs.kv(), ohs.kv(), rtol=1e-12)
  np.testing.assert_allclose(hs.kt(), ohs.kt(), rtol=1e-12)
  ps = np.exp(og.to_nodal(ost_['log_surface_pressure']))
  np.testing.assert_allclose(hs.equilibrium_temperature(ps),
                             ohs.equilibrium_temperature(ps), rtol=1e-12)
  t_dev = hs.equilibrium_temperature(torch.as_tensor(ps, device='cuda',
                                                     dtype=torch.float32))
  np.testing.assert_allclose(t_dev.cpu().numpy(), ohs.equilibrium_temperature(ps),
                             rtol=2e-6)
  st = od.tree_map(lambda x: np.asarray(x, np.float32).astype(np.float64), ost_)
  rng = np.random.default_rng(6)
  noise = rng.standard_normal((layers,) + og.modal_shape) * og.mask / 1e3
  st['vorticity'] = (st['vorticity'] + noise).astype(np.float32).astype(np.float64)
  st['divergence'] = (st['divergence'] + noise[::-1]).astype(np.float32).astype(np.float64)
  got = hs.explicit_terms(to_state(st))
  assert_state(got, ohs.explicit_terms(st), 2e-5)
  peq = pe.PrimitiveEquationsSigma(tref, orog, coords, units.SimUnits())
  fused = ti.compose_equations([peq, hs]).explicit_terms(to_state(st))
  dyn = peq.explicit_terms(to_state(st))
  for k in KEYS:
    a = getattr(fused, k).double()
    b = getattr(dyn, k).double() + getattr(got, k).double()
    assert float((a - b).abs().max() / b.abs().max()) < 2e-5, k


def test_config0_t21_day_matches_fp64_oracle():
  """T21, 12 levels, JW + 1 K bump, dt = 20 min, 72 steps (one day)."""
  og, oeq, st, g, eq = make('T21', 12, perturb=False)
  dt = 0.175008
  step = ti.repeated(ti.step_with_filters(
      ti.imex_rk_sil3(eq, dt), [ti.exponential_step_filter(g, dt)]), 72)
  got = step(to_state(st))
  ostep = od.step_with_filters(od.imex_rk_sil3(oeq, dt),
                               [od.exponential_step_filter(og, dt)])
  ref = od.repeated(ostep, 72)(st)
  for k in KEYS:
    a = getattr(got, k).double().cpu().numpy()
    err = np.linalg.norm(a - ref[k]) / np.linalg.norm(ref[k])
    assert err < 1e-4, (k, err)


def test_jw_steady_state_stays_stationary():
  # primitive_equations_test.py:186-276 (T42, 26 levels, dt = 600 s, 24 h).
  g = sh.Grid.with_wavenumbers(42)
  og = osht.Grid.with_wavenumbers(42)
  layers = 26
  vert = od.SigmaCoordinates.equidistant(layers)
  st, aux = ost.steady_state_jw(og, vert, od.SimUnits())
  orog = od.truncated_modal_orography(aux['orography'], og)
  coords = coordinate_systems.CoordinateSystem(
      g, sigma_coordinates.SigmaCoordinates.equidistant(layers))
  eq = pe.PrimitiveEquationsSigma(aux['ref_temperatures'], orog, coords,
                                  units.SimUnits())
  dt = units.nondim_time(600.0)
  step = ti.step_with_filters(ti.imex_rk_sil3(eq, dt),
                              [ti.exponential_step_filter(g, dt)])
  s0 = to_state(st)
  s = s0
  for _ in range(6):
    s = ti.repeated(step, 24)(s)
    assert float(s.divergence.abs().max()) < 1e-3
    np.testing.assert_allclose(s.vorticity.cpu().numpy(),
                               s0.vorticity.cpu().numpy(), atol=5e-4)
    np.testing.assert_allclose(s.temperature_variation.cpu().numpy(),
                               s0.temperature_variation.cpu().numpy(), atol=5e-2)
    np.testing.assert_allclose(s.log_surface_pressure.cpu().numpy(),
                               s0.log_surface_pressure.cpu().numpy(), atol=5e-4)


def test_bad_state_shapes_raise():
  og, oeq, st, g, eq = make()
  s = to_state(st)
  bad = pe.State(s.vorticity[:, :-1], s.divergence, s.temperature_variation,
                 s.log_surface_pressure)
  with pytest.raises(pe.StateShapeError):
    eq.explicit_terms(bad)


def test_time_reversed_step_and_digital_filter_initialization():
  """TimeReversedImExODE and digital_filter_initialization
  (time_integration.py:117-138, :645-716) against the FP64 oracle: one
  reversed step <= 5e-5, the DFI state (8 steps each way) <= 5e-5 max-abs
  relative; the fused reversed step (the SIL3 step at -dt) equals the generic
  tableau on the reversed ODE to FP32 round-off."""
  og, oeq, st, g, eq = make()
  dt = 0.175008
  rev = ti.TimeReversedImExODE(eq)
  fused = ti.imex_rk_sil3(rev, dt)
  assert isinstance(fused, ti.FusedSIL3Step) and fused.dt == -dt
  ref = od.imex_rk_sil3(od.TimeReversedImExODE(oeq), dt)(st)
  got = fused(to_state(st))
  assert_state(got, ref, 5e-5)
  generic = ti.imex_runge_kutta(ti.SIL3_TABLEAU, rev, dt)(to_state(st))
  for k in KEYS:
    assert rel(getattr(generic, k), getattr(got, k).double().cpu().numpy()) < 1e-5
  flt = [ti.exponential_step_filter(g, dt)]
  oflt = [od.exponential_step_filter(og, dt)]
  dfi = ti.digital_filter_initialization(eq, ti.imex_rk_sil3, flt, 8 * dt, 8 * dt, dt)
  odfi = od.digital_filter_initialization(oeq, od.imex_rk_sil3, oflt, 8 * dt,
                                          8 * dt, dt)
  assert_state(dfi(to_state(st)), odfi(st), 5e-5)
