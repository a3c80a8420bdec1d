"""The package's own host tables against outputs of the reference's code.

``dinosaur_b200.spherical_harmonic`` builds the equiangular latitudes'
quadrature weights (handed to the CUDA plan) and the FP64 ``basis`` matrices
on the host, with formulations of its own: closed-form Fejer / Clenshaw-Curtis
weights instead of the reference's linear solve (associated_legendre.py:160-175),
and a Legendre recurrence that advances every order m at once.  These tests
pin them directly to the golden vectors that ``tests/golden/make_golden.py``
produced from the reference (``basis.npz``), so the GPU tests that feed them
to the plan do not rest on the oracle's copy of the same formulas, and they
check the defining property of the weights (exact for P_k, k < n) at sizes
the fixtures do not cover.
"""

import os

import numpy as np
import pytest

from dinosaur_b200 import spherical_harmonic as sh
from oracle import sht as osht

GOLDEN = os.path.join(os.path.dirname(__file__), 'golden')


def golden():
  return np.load(os.path.join(GOLDEN, 'basis.npz'))


def test_legendre_table_matches_reference():
  g = golden()
  np.testing.assert_allclose(sh._legendre_host(22, 23, g['gauss_x']),
                             g['legendre_T21'], rtol=0, atol=1e-13)


def test_equiangular_nodes_and_weights_match_reference():
  g = golden()
  x, w = sh._equiangular(13, with_poles=False)
  np.testing.assert_allclose(x, g['equi_x'], rtol=0, atol=1e-15)
  np.testing.assert_allclose(w, g['equi_w'], rtol=0, atol=1e-14)


def test_fourier_basis_matches_reference():
  np.testing.assert_allclose(sh._real_basis(22, 64), golden()['fourier_T21'],
                             rtol=0, atol=1e-14)


@pytest.mark.parametrize('with_poles', [False, True])
@pytest.mark.parametrize('n', [2, 3, 8, 13, 31, 64, 129, 256])
def test_closed_form_weights_integrate_legendre_polynomials(n, with_poles):
  """sum_j w_j P_k(x_j) = 2 delta_k0 for k < n: the property the reference's
  solve imposes, which makes the n-point rule unique."""
  x, w = sh._equiangular(n, with_poles)
  p0 = osht.legendre_table(1, n, x)[0]          # unit-norm P_k, shape (n, k)
  moments = w @ p0 * np.sqrt(2.0)               # P_0 = 1 / sqrt 2
  expected = np.zeros(n)
  expected[0] = 2.0
  np.testing.assert_allclose(moments, expected, rtol=0, atol=1e-12)
  ox, ow = (osht.equiangular_nodes_with_poles if with_poles
            else osht.equiangular_nodes)(n)
  np.testing.assert_allclose(w, ow, rtol=0, atol=1e-14)
  np.testing.assert_array_equal(x, ox)


def test_legendre_recurrence_matches_oracle_at_tl255_size():
  x = np.sort(np.cos(np.linspace(0.005, np.pi - 0.005, 256)))
  np.testing.assert_allclose(sh._legendre_host(256, 257, x),
                             osht.legendre_table(256, 257, x), rtol=0, atol=1e-12)


@pytest.mark.parametrize('spacing', ['equiangular', 'equiangular_with_poles'])
def test_grid_basis_on_equiangular_latitudes(spacing):
  """Grid.basis needs no GPU on equiangular latitudes; it equals the
  oracle's (f, p, w) on the same grid."""
  grid = sh.Grid.with_wavenumbers(16, latitude_spacing=spacing)
  basis = grid.spherical_harmonics.basis
  og = osht.Grid.with_wavenumbers(16, latitude_spacing=spacing)
  f, p, w = og.basis
  np.testing.assert_allclose(basis.f, f, rtol=0, atol=1e-14)
  np.testing.assert_allclose(basis.p, p, rtol=0, atol=1e-13)
  np.testing.assert_allclose(basis.w, w, rtol=0, atol=1e-14)
