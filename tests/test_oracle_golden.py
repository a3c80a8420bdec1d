"""Pins the FP64 oracle against outputs of the reference's own code.

The fixtures were written by ``tests/golden/make_golden.py``, which imports
neuralgcm/dinosaur's modules and runs them in float64.  Tolerances are FP64
round-off tolerances (the two sides evaluate the same formulas with different
summation order).
"""

import os

import numpy as np
import pytest

from oracle import dycore, sht, states

GOLDEN = os.path.join(os.path.dirname(__file__), 'golden')


def load(name):
  return np.load(os.path.join(GOLDEN, name))


def close(a, b, rtol=1e-10, atol=1e-12):
  np.testing.assert_allclose(np.asarray(a, np.float64),
                             np.asarray(b, np.float64), rtol=rtol, atol=atol)


def test_basis_matches_reference():
  g = load('basis.npz')
  x, w = sht.gauss_legendre_nodes(32)
  close(x, g['gauss_x'], atol=0)
  close(w, g['gauss_w'], atol=0)
  close(sht.legendre_table(22, 23, x), g['legendre_T21'], atol=1e-13)
  xe, we = sht.equiangular_nodes(13)
  close(xe, g['equi_x'])
  close(we, g['equi_w'])
  close(sht.real_fourier_basis(22, 64), g['fourier_T21'], atol=1e-14)
  close(sht.real_basis_derivative(g['deriv_in']), g['deriv_out'], atol=0)


GRIDS = {
    'T21': sht.Grid.T21(),
    'TL31': sht.Grid.TL31(),
    'W16': sht.Grid.with_wavenumbers(16),
}


@pytest.mark.parametrize('name', sorted(GRIDS))
def test_sht_and_operators_match_reference(name):
  g = load(f'sht_{name}.npz')
  grid = GRIDS[name]
  modal = g['modal_in']
  close(grid.to_nodal(modal), g['nodal_out'])
  close(grid.to_modal(g['nodal_in']), g['modal_out'])
  close(grid.d_dlon(modal), g['d_dlon'], atol=0)
  close(grid.cos_lat_d_dlat(modal), g['cos_lat_d_dlat'])
  close(grid.sec_lat_d_dlat_cos2(modal), g['sec_lat_d_dlat_cos2'])
  close(grid.laplacian(modal), g['laplacian'])
  close(grid.inverse_laplacian(modal), g['inverse_laplacian'])
  close(grid.clip_wavenumbers(modal), g['clip'], atol=0)
  close(grid.div_cos_lat((modal[0], modal[1])), g['div_cos_lat'])
  close(grid.curl_cos_lat((modal[0], modal[1]), clip=False), g['curl_cos_lat'])
  u, v = sht.get_cos_lat_vector(g['vort'], g['div'], grid, clip=False)
  close(u, g['u_cos'])
  close(v, g['v_cos'])
  u, v = sht.get_cos_lat_vector(g['vort'], g['div'], grid)
  close(u, g['u_cos_clip'])
  close(v, g['v_cos_clip'])
  un, vn = sht.vor_div_to_uv_nodal(grid, g['vort'], g['div'])
  close(un, g['u_nodal'])
  close(vn, g['v_nodal'])
  close(grid.integrate(g['nodal_in']), g['integrate'])
  close(sht.exponential_filter_scaling(grid) * np.ones(grid.modal_shape),
        g['filter_default'], rtol=1e-12)
  close(sht.exponential_filter_scaling(grid, 0.131256 / 0.0087504, 1.5, 0.8)
        * np.ones(grid.modal_shape), g['filter_hs'], rtol=1e-12)


def test_sigma_coordinates_match_reference():
  g = load('sigma.npz')
  sig = dycore.SigmaCoordinates.equidistant(6)
  close(sig.centers, g['centers'], atol=0)
  close(sig.layer_thickness, g['thickness'], atol=0)
  close(dycore.cumulative_sigma_integral(g['x'], sig), g['cumulative'])
  close(dycore.cumulative_sigma_integral(g['x'], sig, downward=False),
        g['cumulative_up'])
  close(dycore.sigma_integral(g['x'], sig), g['integral'])
  close(dycore.centered_vertical_advection(g['w'], g['x'], sig),
        g['advection'])


def test_units_match_reference():
  g = load('units.npz')
  ps = dycore.SimUnits()
  for k in ('radius', 'angular_velocity', 'g', 'R', 'R_vapor', 'Cp_vapor',
            'kappa'):
    close(getattr(ps, k), g[k], rtol=1e-14)
  hs = dycore.HeldSuarezForcingSigma(sht.Grid.T21(),
                                     dycore.SigmaCoordinates.equidistant(6),
                                     ps, np.full(6, 285.0))
  for k in ('kf', 'ka', 'ks', 'p0'):
    close(getattr(hs, k), g[k], rtol=1e-14)


STATE_KEYS = ('vorticity', 'divergence', 'temperature_variation',
              'log_surface_pressure')


def unpack(g, prefix, tracers=None):
  return dycore.make_state(*[g[f'{prefix}_{k}'] for k in STATE_KEYS],
                           tracers=tracers)


def assert_state_close(a, b, **kw):
  for k in STATE_KEYS:
    scale = max(np.abs(b[k]).max(), 1e-300)
    close(a[k] / scale, b[k] / scale, **kw)


@pytest.fixture(scope='module')
def pe_setup():
  g = load('pe_T21_L6.npz')
  grid = sht.Grid.T21()
  vertical = dycore.SigmaCoordinates.equidistant(6)
  eq = dycore.PrimitiveEquationsSigma(g['ref_temps'], g['orography'], grid,
                                      vertical, dycore.SimUnits())
  return g, grid, vertical, eq


def test_initial_states_match_reference(pe_setup):
  g, grid, vertical, _ = pe_setup
  st, aux = states.steady_state_jw(grid, vertical, dycore.SimUnits())
  close(st['vorticity'], g['jw_vorticity'], atol=1e-13)
  close(st['temperature_variation'], g['jw_temperature'], rtol=1e-9,
        atol=1e-9)
  close(st['log_surface_pressure'], g['jw_log_ps'], rtol=1e-12)
  close(aux['ref_temperatures'], g['ref_temps'], rtol=1e-12)
  close(aux['orography'], g['orography_nodal'], rtol=1e-9, atol=1e-12)
  close(dycore.truncated_modal_orography(aux['orography'], grid),
        g['orography'], rtol=1e-9, atol=1e-12)
  bump = states.gaussian_scalar(grid, 6, lon_location=1.0, lat_location=0.3,
                                perturbation_radius=0.1, amplitude=1.0)
  close(bump, g['bump'], atol=1e-13)


def test_primitive_terms_match_reference(pe_setup):
  g, _, _, eq = pe_setup
  s = unpack(g, 'in')
  assert_state_close(eq.explicit_terms(s), unpack(g, 'explicit'), atol=1e-9)
  assert_state_close(eq.implicit_terms(s), unpack(g, 'implicit'), atol=1e-11)
  assert_state_close(eq.implicit_inverse(s, 0.05), unpack(g, 'inverse'),
                     atol=1e-11)


def test_sil3_steps_match_reference(pe_setup):
  g, grid, _, eq = pe_setup
  dt = 0.175008
  step = dycore.step_with_filters(dycore.imex_rk_sil3(eq, dt),
                                  [dycore.exponential_step_filter(grid, dt)])
  s1 = step(unpack(g, 'in'))
  assert_state_close(s1, unpack(g, 'step1'), atol=1e-10)
  s2 = step(s1)
  assert_state_close(s2, unpack(g, 'step2'), atol=1e-10)


def test_moist_terms_match_reference(pe_setup):
  g, grid, vertical, _ = pe_setup
  gm = load('pe_moist_T21_L6.npz')
  eq = dycore.PrimitiveEquationsSigma(
      g['ref_temps'], g['orography'], grid, vertical, dycore.SimUnits(),
      humidity_key='specific_humidity')
  s = unpack(g, 'in', tracers={'specific_humidity': gm['humidity'],
                               'tracer': gm['tracer']})
  out = eq.explicit_terms(s)
  assert_state_close(out, unpack(gm, 'explicit'), atol=1e-9)
  for k, ref in (('specific_humidity', gm['explicit_humidity']),
                 ('tracer', gm['explicit_tracer'])):
    scale = np.abs(ref).max()
    close(out['tracers'][k] / scale, ref / scale, atol=1e-9)


def test_held_suarez_matches_reference():
  g = load('hs_T21_L6.npz')
  grid = sht.Grid.T21()
  vertical = dycore.SigmaCoordinates.equidistant(6)
  ps = dycore.SimUnits()
  ref = np.full(6, 285.0)
  hs = dycore.HeldSuarezForcingSigma(grid, vertical, ps, ref)
  s = unpack(g, 'in')
  assert_state_close(hs.explicit_terms(s), unpack(g, 'forcing'), atol=1e-10)
  pe = dycore.PrimitiveEquationsSigma(ref, np.zeros(grid.modal_shape), grid,
                                      vertical, ps)
  eq = dycore.ComposedEquation([pe, hs])
  dt = 0.131256
  step = dycore.step_with_filters(
      dycore.imex_rk_sil3(eq, dt),
      [dycore.exponential_step_filter(grid, dt, tau=0.0087504, order=1.5,
                                      cutoff=0.8)])
  assert_state_close(step(s), unpack(g, 'step1'), atol=1e-10)


SWE_KEYS = ('vorticity', 'divergence', 'potential')


def test_shallow_water_matches_reference():
  from oracle import swe
  g = load('swe_T21_L2.npz')
  grid = sht.Grid.T21()
  steady = swe.multi_layer(g['u_layers'], g['densities'], grid)
  for k in SWE_KEYS:
    scale = max(np.abs(g[f'steady_{k}']).max(), 1e-300)
    close(steady[k] / scale, g[f'steady_{k}'] / scale, atol=1e-11)
  eq = swe.ShallowWaterEquations(grid, dycore.SimUnits(), g['orography'],
                                 g['ref_potential'], g['densities'])
  s = {k: g[f'in_{k}'] for k in SWE_KEYS}

  def check(got, prefix, atol):
    for k in SWE_KEYS:
      ref = g[f'{prefix}_{k}']
      scale = max(np.abs(ref).max(), 1e-300)
      close(got[k] / scale, ref / scale, atol=atol)

  check(eq.explicit_terms(s), 'explicit', 1e-10)
  check(eq.implicit_terms(s), 'implicit', 1e-12)
  check(eq.implicit_inverse(s, 0.03), 'inverse', 1e-12)
  dt = float(g['dt'])
  step = swe.filtered_step(swe.imex_rk_sil3(eq, dt),
                           sht.exponential_filter_scaling(grid, dt / 0.010938, 18, 0))
  s1 = step(s)
  check(s1, 'step1', 1e-10)
  check(step(s1), 'step2', 1e-10)


def test_fast_layout_is_the_real_layout_with_a_zero_row():
  g = load('fast_T21.npz')
  grid = sht.Grid.T21()
  m = g['modal_axes_m']
  np.testing.assert_array_equal(m[:2], [0, 0])
  np.testing.assert_array_equal(np.delete(m, 1), grid.modal_axes[0])
  np.testing.assert_array_equal(g['modal_axes_l'], grid.modal_axes[1])
  assert not g['mask'][1].any()
  np.testing.assert_array_equal(sht.fast_to_real(g['mask']), grid.mask)
  x = sht.fast_to_real(g['modal_in'])
  close(grid.to_nodal(x), g['nodal_out'])
  close(sht.real_to_fast(grid.to_modal(g['nodal_in'])), g['modal_out'])
  for name in ('d_dlon', 'laplacian', 'cos_lat_d_dlat', 'sec_lat_d_dlat_cos2'):
    close(sht.real_to_fast(getattr(grid, name)(x)), g[name], atol=1e-12)
  close(sht.real_to_fast(grid.clip_wavenumbers(x)), g['clip'], atol=0)


def test_digital_filter_initialization_matches_reference(pe_setup):
  g, grid, _, eq = pe_setup
  d = load('dfi_T21_L6.npz')
  dt = float(d['dt'])
  close(dycore.dfi_lanczos_weights(8 * dt, 8 * dt, dt), d['weights'], atol=0)
  s = unpack(g, 'in')
  rev = dycore.imex_rk_sil3(dycore.TimeReversedImExODE(eq), dt)(s)
  assert_state_close(rev, unpack(d, 'reversed_step'), atol=1e-10)
  dfi = dycore.digital_filter_initialization(
      eq, dycore.imex_rk_sil3, [dycore.exponential_step_filter(grid, dt)],
      8 * dt, 8 * dt, dt)
  assert_state_close(dfi(s), unpack(d, 'dfi'), atol=1e-10)


@pytest.mark.parametrize('fixture', ['pe_hybrid_T21_L6.npz',
                                     'pe_hybrid_ecmwf_like_T21_L6.npz'])
def test_hybrid_terms_and_step_match_reference(pe_setup, fixture):
  """PrimitiveEquationsHybrid on 6 hybrid levels, same input state: the
  analytic levels (pe_hybrid_T21_L6.npz) and ECMWF-like levels whose top two
  layers are pure pressure, b = 0 (pe_hybrid_ecmwf_like_T21_L6.npz).  The
  reference differences its float32 reference temperatures in float32
  (get_temperature_implicit_weights_hybrid's np.diff), 1.1e-7 of the
  implicit temperature term; hence 1e-6 for the implicit terms, 1e-8
  elsewhere (the step measures 1e-9)."""
  from oracle import hybrid
  g0, grid, _, _ = pe_setup
  g = load(fixture)
  eq = hybrid.PrimitiveEquationsHybrid(
      g0['ref_temps'], g0['orography'], grid,
      hybrid.HybridCoordinates(g['a_boundaries'], g['b_boundaries']), dycore.SimUnits())
  s = unpack(g0, 'in')
  assert_state_close(eq.explicit_terms(s), unpack(g, 'explicit'), atol=1e-8)
  assert_state_close(eq.implicit_terms(s), unpack(g, 'implicit'), atol=1e-6)
  assert_state_close(eq.implicit_inverse(s, 0.05), unpack(g, 'inverse'), atol=1e-8)
  dt = 0.175008
  step = dycore.step_with_filters(dycore.imex_rk_sil3(eq, dt),
                                  [dycore.exponential_step_filter(grid, dt)])
  assert_state_close(step(s), unpack(g, 'step1'), atol=1e-8)


def test_moist_hybrid_terms_match_reference(pe_setup):
  """Moist PrimitiveEquationsHybrid with a passive tracer on the 6 analytic
  levels (pe_hybrid_moist_T21_L6.npz; inputs of pe_moist_T21_L6.npz)."""
  from oracle import hybrid
  g0, grid, _, _ = pe_setup
  g = load('pe_hybrid_T21_L6.npz')
  gm = load('pe_moist_T21_L6.npz')
  ghm = load('pe_hybrid_moist_T21_L6.npz')
  eq = hybrid.PrimitiveEquationsHybrid(
      g0['ref_temps'], g0['orography'], grid,
      hybrid.HybridCoordinates(g['a_boundaries'], g['b_boundaries']), dycore.SimUnits(),
      humidity_key='specific_humidity')
  s = unpack(g0, 'in', tracers={'specific_humidity': gm['humidity'],
                                'tracer': gm['tracer']})
  out = eq.explicit_terms(s)
  assert_state_close(out, unpack(ghm, 'explicit'), atol=1e-8)
  for k, ref in (('specific_humidity', ghm['explicit_humidity']),
                 ('tracer', ghm['explicit_tracer'])):
    scale = np.abs(ref).max()
    close(out['tracers'][k] / scale, ref / scale, atol=1e-8)


def test_package_hybrid_levels_match_reference():
  """dinosaur_b200.hybrid_coordinates' constructors and pressure helpers
  give the reference's levels (hybrid_levels.npz)."""
  from dinosaur_b200 import hybrid_coordinates as hc
  from dinosaur_b200 import sigma_coordinates as sc
  g = load('hybrid_levels.npz')
  cases = {'analytic': hc.HybridCoordinates.analytic_levels(17),
           'ecmwf_like': hc.HybridCoordinates.analytic_ecmwf_like(20),
           'sigma': hc.HybridCoordinates.from_sigma_levels(
               sc.SigmaCoordinates.equidistant(8)),
           'coeffs': hc.HybridCoordinates.from_coefficients(
               [0.0, 0.1, 0.05, 0.0], [0.0, 0.2, 0.6, 1.0], p0=1013.25)}
  for name, lev in cases.items():
    close(lev.a_boundaries, g[f'{name}_a'], rtol=1e-15, atol=0)
    close(lev.b_boundaries, g[f'{name}_b'], rtol=1e-15, atol=0)
  lev = cases['analytic']
  close(lev.layer_thickness(900.0), g['analytic_thickness_at_900'], rtol=1e-15, atol=1e-13)
  close(lev.pressure_centers(900.0), g['analytic_centers_at_900'], rtol=1e-15, atol=1e-13)
