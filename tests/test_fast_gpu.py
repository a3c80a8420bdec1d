"""GPU parity of the FastSphericalHarmonics modal layout.

Against the reference's own outputs (tests/golden/fast_T21.npz, written by
make_golden.py from dinosaur.spherical_harmonic.FastSphericalHarmonics in
float64): modal axes and mask exactly; transforms and spectral operators
<= 2e-6 max-abs relative.  A primitive-equation step on a Fast-layout grid
equals the Real-layout step exactly (the engine runs in the Real layout), and
the layout conversion's autograd transpose matches <J^T w, v> = <w, J v>.
"""

import functools
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

from dinosaur_b200 import coordinate_systems  # noqa: E402
from dinosaur_b200 import primitive_equations as pe  # noqa: E402
from dinosaur_b200 import sigma_coordinates  # noqa: E402
from dinosaur_b200 import spherical_harmonic as sh  # noqa: E402
from dinosaur_b200 import time_integration as ti  # noqa: E402
from dinosaur_b200 import units  # noqa: E402

GOLDEN = os.path.join(os.path.dirname(__file__), 'golden')


def fast_grid(**kw):
  return sh.Grid.T21(spherical_harmonics_impl=functools.partial(
      sh.FastSphericalHarmonics, **kw))


def rel(a, b):
  a = a.detach().double().cpu().numpy()
  return np.abs(a - b).max() / max(np.abs(b).max(), 1e-30)


def test_fast_layout_matches_reference():
  g = np.load(os.path.join(GOLDEN, 'fast_T21.npz'))
  grid = fast_grid()
  assert grid.modal_shape == (44, 23)
  np.testing.assert_array_equal(grid.modal_axes[0], g['modal_axes_m'])
  np.testing.assert_array_equal(grid.modal_axes[1], g['modal_axes_l'])
  np.testing.assert_array_equal(grid.mask, g['mask'])
  x = torch.as_tensor(g['modal_in'], device='cuda', dtype=torch.float32)
  assert rel(grid.to_nodal(x), g['nodal_out']) < 2e-6
  z = torch.as_tensor(g['nodal_in'], device='cuda', dtype=torch.float32)
  assert rel(grid.to_modal(z), g['modal_out']) < 2e-6
  for name in ('d_dlon', 'laplacian', 'cos_lat_d_dlat', 'sec_lat_d_dlat_cos2'):
    assert rel(getattr(grid, name)(x), g[name]) < 2e-6, name
  # The input is the FP32 rounding of the FP64 fixture.
  assert rel(grid.clip_wavenumbers(x), g['clip']) < 1e-7


def test_fast_layout_step_equals_real_layout_step():
  from pe_cases import make, to_state
  og, oeq, st, g, eq = make()
  fg = fast_grid()
  coords = coordinate_systems.CoordinateSystem(
      fg, sigma_coordinates.SigmaCoordinates.equidistant(6))
  orog = np.insert(np.asarray(oeq.orography, np.float32), 1, 0.0, axis=-2)
  feq = pe.PrimitiveEquationsSigma(oeq.reference_temperature, orog, coords,
                                   units.SimUnits())
  dt = 0.175008
  real = ti.step_with_filters(ti.imex_rk_sil3(eq, dt),
                              [ti.exponential_step_filter(g, dt)])(to_state(st))
  fs = to_state(st)
  fs = pe.State(*[sh.from_real_layout(fg, getattr(fs, k)) for k in
                  ('vorticity', 'divergence', 'temperature_variation',
                   'log_surface_pressure')])
  fast = ti.step_with_filters(ti.imex_rk_sil3(feq, dt),
                              [ti.exponential_step_filter(fg, dt)])(fs)
  for k in ('vorticity', 'divergence', 'temperature_variation',
            'log_surface_pressure'):
    a = getattr(fast, k)
    assert tuple(a.shape[-2:]) == (44, 23)
    assert float(a[..., 1, :].abs().max()) == 0.0
    torch.testing.assert_close(sh.to_real_layout(fg, a), getattr(real, k),
                               rtol=0, atol=0)


def test_fast_layout_autograd_is_the_transpose():
  grid = fast_grid()
  rng = np.random.default_rng(3)
  mask = torch.as_tensor(grid.mask, device='cuda', dtype=torch.float32)
  v = torch.as_tensor(rng.standard_normal((2,) + grid.modal_shape), device='cuda',
                      dtype=torch.float32) * mask
  w = torch.as_tensor(rng.standard_normal((2,) + grid.nodal_shape), device='cuda',
                      dtype=torch.float32)
  x = v.clone().requires_grad_(True)
  (grid.to_nodal(x) * w).sum().backward()
  lhs = float((x.grad.double() * v.double()).sum())
  rhs = float((grid.to_nodal(v).double() * w.double()).sum())
  assert abs(lhs - rhs) <= 1e-5 * abs(rhs)
