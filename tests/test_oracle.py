"""The reference test suite's analytic identities, applied to the FP64 oracle.

Each test names the reference test it restates and keeps its tolerance.
"""

import numpy as np
import pytest

from oracle import dycore, sht


def random_modal_state(grid, seed=0):
  """spherical_harmonic_test.py:37-44."""
  _, l = grid.modal_mesh
  rs = np.random.RandomState(seed)
  return rs.normal(size=grid.mask.shape) * grid.mask / (l + 1) ** 2


@pytest.mark.parametrize('lw,tw,spacing', [(32, 32, 'gauss'), (45, 123, 'gauss'),
                                           (64, 64, 'gauss')])
def test_round_trip(lw, tw, spacing):
  # spherical_harmonic_test.py:187-219
  g = sht.Grid(lw, tw, 4 * lw, 2 * tw, spacing)
  modal = random_modal_state(g)
  modal[0, 0] = 0
  np.testing.assert_allclose(g.to_modal(g.to_nodal(modal)), modal, atol=1e-5)


def test_laplacian_round_trip():
  # spherical_harmonic_test.py:221-240
  g = sht.Grid.with_wavenumbers(32)
  x = random_modal_state(g)
  x[0, 0] = 0
  np.testing.assert_allclose(g.inverse_laplacian(g.laplacian(x)), x)


@pytest.mark.parametrize('wavenumbers', [64, 128])
def test_analytic_derivatives(wavenumbers):
  # spherical_harmonic_test.py:242-287 with the test functions' derivatives
  # written out (f = cos^4(lat) sin(3 lon)).
  g = sht.Grid.with_wavenumbers(wavenumbers)
  lon, sin_lat = g.nodal_mesh
  lat = np.arcsin(sin_lat)
  f = np.cos(lat) ** 4 * np.sin(3 * lon)
  fm = g.to_modal(f)
  np.testing.assert_allclose(g.to_nodal(g.d_dlon(fm)),
                             3 * np.cos(lat) ** 4 * np.cos(3 * lon), atol=1e-5)
  df_dlat = -4 * np.cos(lat) ** 3 * np.sin(lat) * np.sin(3 * lon)
  np.testing.assert_allclose(g.to_nodal(g.cos_lat_d_dlat(fm)),
                             df_dlat * np.cos(lat), atol=1e-5)
  dcos2f = -6 * np.cos(lat) ** 5 * np.sin(lat) * np.sin(3 * lon)
  np.testing.assert_allclose(g.to_nodal(g.sec_lat_d_dlat_cos2(fm)),
                             dcos2f / np.cos(lat), atol=1e-5)


def test_orthonormality_and_area():
  # spherical_harmonic_test.py:497-529
  g = sht.Grid.T21()
  np.testing.assert_allclose(g.integrate(np.ones(g.nodal_shape)), 4 * np.pi)
  m, l = g.modal_mesh
  for row, col in [(0, 0), (1, 3), (6, 10), (20, 21)]:
    e = np.zeros(g.modal_shape)
    e[row, col] = 1
    y = g.to_nodal(e)
    np.testing.assert_allclose(g.integrate(y * y), 1.0, atol=1e-10)


def test_modal_axes_and_shapes():
  # spherical_harmonic_test.py:117-155
  g = sht.Grid.T21()
  assert g.nodal_shape == (64, 32) and g.modal_shape == (43, 23)
  assert sht.Grid.TL31().modal_shape == (63, 33)
  np.testing.assert_array_equal(g.modal_axes[0][:5], [0, 1, -1, 2, -2])


def test_constant_normalization():
  # spherical_harmonic.py:1154-1161
  g = sht.Grid.T21()
  assert g.to_modal(np.ones(g.nodal_shape))[0, 0] == pytest.approx(3.5449077,
                                                                    rel=1e-7)


def test_exponential_filter_value():
  # filtering_test.py:38-43
  g = sht.Grid.TL127()
  s = sht.exponential_filter_scaling(g, attenuation=16)
  assert s[0] == pytest.approx(1.0)
  assert s[-1] == pytest.approx(1.125e-7, abs=1e-9)


def test_legendre_matches_scipy_lpmv():
  # associated_legendre_test.py:41-55 (up to the normalisation)
  import scipy.special as sps
  x = np.linspace(-0.9, 0.9, 7)
  p = sht.legendre_table(6, 8, x)
  for m in range(6):
    for l in range(m, 8):
      ref = sps.lpmv(m, l, x)
      ratio = p[m, :, l] / ref
      np.testing.assert_allclose(ratio, ratio[0], rtol=1e-10)


@pytest.mark.parametrize('eta', [0.3, 0.05])
def test_primitive_inverse_identity(eta):
  # primitive_equations_test.py:578-658
  g = sht.Grid.with_wavenumbers(16)
  vert = dycore.SigmaCoordinates.equidistant(5)
  ps = dycore.SimUnits.from_si(ideal_gas_constant_si=33.0, kappa_si=1.4)
  rng = np.random.default_rng(0)
  scale = (g.total_wavenumbers + 1) ** -2
  shp = (5,) + g.modal_shape
  st = dycore.make_state(*(scale * rng.standard_normal(s) for s in
                           (shp, shp, shp, (1,) + g.modal_shape)))
  eq = dycore.PrimitiveEquationsSigma(np.linspace(100, 200, 5),
                                      np.zeros(g.modal_shape), g, vert, ps)
  x = dycore.tree_axpy((1.0, st), (-eta, eq.implicit_terms(st)))
  back = eq.implicit_inverse(x, eta)
  for k in dycore.STATE_KEYS:
    np.testing.assert_allclose(back[k], st[k], atol=1e-5)


class _LinearODE:
  """dx/dt = a x (explicit) + b x (implicit): exact solution exp((a+b) t)."""

  def __init__(self, a, b):
    self.a, self.b = a, b

  def explicit_terms(self, s):
    return dycore.tree_map(lambda x: self.a * x, s)

  def implicit_terms(self, s):
    return dycore.tree_map(lambda x: self.b * x, s)

  def implicit_inverse(self, s, eta):
    return dycore.tree_map(lambda x: x / (1 - eta * self.b), s)


def test_sil3_converges_on_linear_ode():
  # time_integration_test.py:60-149 (imex_rk_sil3 column): second order.
  a, b, t_end = -0.3, -1.0, 1.0
  errs = []
  for n in (20, 40):
    dt = t_end / n
    eq = _LinearODE(a, b)
    s = dycore.make_state(*(np.ones((1, 1, 1)) for _ in range(4)))
    step = dycore.imex_rk_sil3(eq, dt)
    for _ in range(n):
      s = step(s)
    errs.append(abs(s['vorticity'].item() - np.exp((a + b) * t_end)))
  assert errs[1] < errs[0] / 3.5
