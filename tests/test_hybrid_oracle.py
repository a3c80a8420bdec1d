"""The FP64 hybrid-coordinate oracle (oracle/hybrid.py) against the pins
that the reference's own tests give it (primitive_equations_test.py:739-905):

* on sigma-like hybrid levels (a = 0, b = sigma) the explicit and implicit
  terms equal the sigma equations' to atol 1e-3 (test_equivalence_sigma_like,
  :785-848; the sigma oracle is pinned to golden vectors of the reference);
* implicit_inverse inverts (1 - eta implicit_terms) to atol 1e-5
  (test_implicit_inverse_sigma_like, :850-896), here also on analytic
  (non-sigma) levels;
* the package's HybridCoordinates constructors give the oracle's levels;
* the package's PrimitiveEquationsHybrid host checks (level scaling and
  refusals) run without a GPU.
"""

import numpy as np
import pytest

from oracle import dycore as od
from oracle import hybrid as oh
from oracle import sht as osht
from oracle import states as ost


def jw_case(layers, amplitude=0.0):
  og = osht.Grid.with_wavenumbers(21)
  st, tref, orog, vert = ost.baroclinic_config(og, layers, seed=0, amplitude=amplitude)
  return og, st, tref, orog, vert


def assert_close(a, b, atol):
  for k in od.STATE_KEYS:
    np.testing.assert_allclose(a[k], b[k], atol=atol, rtol=0, err_msg=k)


@pytest.mark.parametrize('layers', [20, 40])
def test_sigma_like_levels_match_sigma_equations(layers):
  # The explicit terms agree to ~1e-11; the implicit divergence differs by
  # the top level's geopotential coefficient (alpha_0 = 1 on hybrid levels),
  # 5.5e-4 at 20 layers and 9e-5 at the reference test's 40.
  og, st, tref, orog, vert = jw_case(layers)
  sig = od.PrimitiveEquationsSigma(tref, orog, og, vert, od.SimUnits())
  hyb = oh.PrimitiveEquationsHybrid(tref, orog, og,
                                    oh.HybridCoordinates.from_sigma_levels(vert),
                                    od.SimUnits())
  assert_close(hyb.explicit_terms(st), sig.explicit_terms(st), 1e-3)
  assert_close(hyb.implicit_terms(st), sig.implicit_terms(st), 1e-3)


def random_state(og, layers, seed):
  rng = np.random.default_rng(seed)
  _, l = og.modal_mesh
  f = lambda n: rng.standard_normal((n,) + og.modal_shape) * og.mask / (l + 1.0)
  return od.make_state(f(layers), f(layers), f(layers), f(1))


@pytest.mark.parametrize('levels', ['sigma_like', 'analytic'])
def test_implicit_inverse_inverts(levels):
  og = osht.Grid.with_wavenumbers(16)
  layers = 5
  vert = od.SigmaCoordinates.equidistant(layers)
  lev = (oh.HybridCoordinates.from_sigma_levels(vert) if levels == 'sigma_like'
         else oh.HybridCoordinates.analytic_levels(layers))
  eq = oh.PrimitiveEquationsHybrid(280 * np.ones(layers), np.zeros(og.modal_shape),
                                   og, lev, od.SimUnits())
  st = random_state(og, layers, 0)
  eta = 0.1
  rhs = od.tree_axpy((1.0, st), (-eta, eq.implicit_terms(st)))
  assert_close(eq.implicit_inverse(rhs, eta), st, 1e-5)


def test_package_levels_match_oracle():
  from dinosaur_b200 import hybrid_coordinates as hc
  from dinosaur_b200 import sigma_coordinates as sc
  a = hc.HybridCoordinates.analytic_levels(17)
  b = oh.HybridCoordinates.analytic_levels(17)
  np.testing.assert_array_equal(a.a_boundaries, b.a_boundaries)
  np.testing.assert_array_equal(a.b_boundaries, b.b_boundaries)
  s = hc.HybridCoordinates.from_sigma_levels(sc.SigmaCoordinates.equidistant(8))
  assert s.layers == 8 and np.all(s.a_boundaries == 0)
  np.testing.assert_allclose(s.layer_thickness(2.0), 2.0 / 8)
  with pytest.raises(ValueError):
    hc.HybridCoordinates(np.zeros(3), np.zeros(4))


def test_package_level_pressures_broadcast_like_the_reference():
  # hybrid_coordinates.py:443-462: one new axis per non-singleton axis of the
  # surface pressure, so a (1, lon, lat) surface pressure gives
  # (levels, lon, lat) boundaries, centres and thicknesses.
  from dinosaur_b200 import hybrid_coordinates as hc
  lev = hc.HybridCoordinates.analytic_levels(6)
  ps = np.random.default_rng(3).uniform(90.0, 110.0, (1, 8, 4))
  bounds = lev.pressure_boundaries(ps)
  assert bounds.shape == (7, 8, 4)
  np.testing.assert_allclose(
      bounds, lev.a_boundaries[:, None, None] + lev.b_boundaries[:, None, None] * ps[0])
  assert lev.pressure_centers(ps).shape == (6, 8, 4)
  np.testing.assert_allclose(lev.layer_thickness(ps), np.diff(bounds, axis=0))
  assert lev.pressure_boundaries(100.0).shape == (7,)
  assert lev.layer_thickness(ps[0]).shape == (6, 8, 4)


@pytest.mark.parametrize('levels', ['analytic', 'sigma_like', 'ecmwf_like'])
def test_package_hybrid_matrices_match_oracle(levels):
  """The FP64 host matrices that the CUDA engine's implicit operators are
  built from (geopotential G, temperature H, the ln p_s column) equal the
  oracle's restatement."""
  from dinosaur_b200 import hybrid_coordinates as hc
  from dinosaur_b200 import primitive_equations as pe
  from dinosaur_b200 import sigma_coordinates as sc
  from dinosaur_b200 import units
  k = 12
  lev = {'analytic': lambda: hc.HybridCoordinates.analytic_levels(k),
         'sigma_like': lambda: hc.HybridCoordinates.from_sigma_levels(
             sc.SigmaCoordinates.equidistant(k)),
         'ecmwf_like': lambda: hc.HybridCoordinates.analytic_ecmwf_like(k)}[levels]()
  # FP64 levels on both sides: the formulas are compared, not dtype rules
  # (sigma levels are float32, and NumPy keeps b * p_s float32 then, as the
  # reference does).
  nd = hc.HybridCoordinates(
      units.nondim_pressure(np.asarray(lev.a_boundaries, np.float64) * 100.0),
      np.asarray(lev.b_boundaries, np.float64))
  olev = oh.HybridCoordinates(nd.a_boundaries, nd.b_boundaries)
  psr = units.nondim_pressure(101325.0)
  tref = np.linspace(210.0, 290.0, k)
  R, kappa = 0.5, 2 / 7
  np.testing.assert_allclose(pe.get_geopotential_weights_hybrid(nd, R, psr),
                             oh.geopotential_weights(olev, R, psr), rtol=1e-12, atol=0)
  np.testing.assert_allclose(pe.get_temperature_implicit_weights_hybrid(nd, tref, kappa, psr),
                             oh.temperature_implicit_weights(olev, tref, kappa, psr),
                             rtol=1e-12, atol=1e-12)
  np.testing.assert_allclose(pe.pgf_lps_coefficient_hybrid(tref, psr, nd, R),
                             oh.pgf_coefficient(tref, psr, olev, R), rtol=1e-12, atol=0)


def test_package_hybrid_equations_host_checks():
  """Construction of PrimitiveEquationsHybrid is host logic: it accepts
  hybrid levels, scales a_boundaries from hPa to nondimensional pressure,
  and refuses sigma levels, a non-positive reference surface pressure and
  Held-Suarez forcing (defined on sigma levels only) before any GPU work."""
  from dinosaur_b200 import coordinate_systems
  from dinosaur_b200 import held_suarez
  from dinosaur_b200 import hybrid_coordinates as hc
  from dinosaur_b200 import primitive_equations as pe
  from dinosaur_b200 import sigma_coordinates as sc
  from dinosaur_b200 import spherical_harmonic as sh
  from dinosaur_b200 import time_integration
  from dinosaur_b200 import units
  g = sh.Grid.T21()
  k = 6
  lev = hc.HybridCoordinates.analytic_levels(k)
  coords = coordinate_systems.CoordinateSystem(g, lev)
  tref = np.full((k, 1, 1), 288.0)
  orog = np.zeros(g.nodal_shape, np.float32)
  eq = pe.PrimitiveEquationsHybrid(tref, orog, coords, units.SimUnits())
  assert eq.p_s_ref == pytest.approx(units.nondim_pressure(101325.0))
  np.testing.assert_allclose(
      eq.nondim_levels.a_boundaries,
      units.nondim_pressure(np.asarray(lev.a_boundaries, np.float64) * 100.0))
  np.testing.assert_array_equal(eq.nondim_levels.b_boundaries, lev.b_boundaries)
  with pytest.raises(ValueError):
    pe.PrimitiveEquationsHybrid(tref, orog, coords, units.SimUnits(),
                                reference_surface_pressure=0.0)
  sigma_coords = coordinate_systems.CoordinateSystem(
      g, sc.SigmaCoordinates.equidistant(k))
  with pytest.raises(TypeError):
    pe.PrimitiveEquationsHybrid(tref, orog, sigma_coords, units.SimUnits())
  hs = held_suarez.HeldSuarezForcingSigma(sigma_coords, units.SimUnits(), tref)
  with pytest.raises(NotImplementedError):
    time_integration.compose_equations([eq, hs])
