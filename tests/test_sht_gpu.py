"""GPU parity of the spherical-harmonic transform pair and operators.

CUDA (FP32, through the C ABI) against the FP64 oracle on seeded inputs.
Tolerances: FP32 transforms are compared by the max-abs error relative to the
max-abs of the FP64 result (<= 2e-6 for one-way transforms at these sizes) and
by the reference's own round-trip identity (atol 1e-5,
dinosaur/spherical_harmonic_test.py:187-219).
"""

import numpy as np
import pytest
import torch

from oracle import sht as osht
from oracle import states as ostates

pytestmark = pytest.mark.gpu

from dinosaur_b200 import spherical_harmonic as sh  # noqa: E402


def rel_err(actual, expected):
  actual = actual.detach().cpu().double().numpy() if torch.is_tensor(actual) else actual
  return np.abs(actual - expected).max() / max(np.abs(expected).max(), 1e-30)


def grid_pair(name):
  if name.startswith('W'):
    kw = {}
    spacing = 'gauss'
    if name.endswith('e'):
      spacing = 'equiangular'
      name = name[:-1]
    n = int(name[1:])
    return (sh.Grid.with_wavenumbers(n, latitude_spacing=spacing),
            osht.Grid.with_wavenumbers(n, latitude_spacing=spacing))
  return getattr(sh.Grid, name)(), getattr(osht.Grid, name)()


GRIDS = ['T21', 'TL31', 'T42', 'T85', 'TL127', 'W16', 'W16e']


@pytest.mark.parametrize('name', ['T21', 'T42', 'TL255'])
def test_gauss_nodes_and_legendre_table(name):
  g, o = grid_pair(name)
  x, w = g.plan.nodes
  xo, wo = osht.gauss_legendre_nodes(g.latitude_nodes)
  np.testing.assert_allclose(x, xo, atol=2e-15)
  # Near the poles 1 - x^2 is small, so FP64 weights agree to ~1e-10 relative.
  np.testing.assert_allclose(w, wo, rtol=1e-9, atol=1e-16)
  p = osht.legendre_table(g.longitude_wavenumbers, g.total_wavenumbers, xo)
  import ctypes
  from dinosaur_b200 import _lib
  col = np.zeros(g.latitude_nodes)
  for m in (0, 1, g.longitude_wavenumbers // 2, g.longitude_wavenumbers - 1):
    for l in (m, min(m + 1, g.total_wavenumbers - 1), g.total_wavenumbers - 1):
      _lib.check(_lib.lib().dino_plan_legendre_column(
          g.plan.handle, m, l, _lib.dptr(col)))
      np.testing.assert_allclose(col, p[m, :, l], rtol=1e-6, atol=1e-6)


@pytest.mark.parametrize('name', GRIDS)
def test_transforms_match_oracle(name):
  g, o = grid_pair(name)
  x = ostates.sht_modal_input(o, 6, seed=1).astype(np.float64)
  nodal = g.to_nodal(x)
  assert nodal.shape == (6,) + g.nodal_shape
  ref_nodal = o.to_nodal(x.astype(np.float32).astype(np.float64))
  assert rel_err(nodal, ref_nodal) < 2e-6
  z = np.random.default_rng(2).standard_normal((5,) + g.nodal_shape)
  modal = g.to_modal(z)
  assert modal.shape == (5,) + g.modal_shape
  ref_modal = o.to_modal(z.astype(np.float32).astype(np.float64))
  assert rel_err(modal, ref_modal) < 2e-6
  # Structural zeros of the forward transform are exact.
  assert np.all(modal.cpu().numpy()[:, ~o.mask] == 0)


@pytest.mark.parametrize('lw', [16, 64])
def test_reference_round_trip_identity(lw):
  # spherical_harmonic_test.py:187-219 (gauss, Real layout)
  g = sh.Grid(longitude_nodes=4 * lw, latitude_nodes=2 * lw,
              longitude_wavenumbers=lw, total_wavenumbers=lw)
  _, l = g.modal_mesh
  rs = np.random.RandomState(0)
  modal = rs.normal(size=g.mask.shape) * g.mask / (l + 1) ** 2
  modal[0, 0] = 0
  back = g.to_modal(g.to_nodal(modal)).cpu().numpy()
  np.testing.assert_allclose(back, modal, atol=1e-5)


def test_tl255_batch_round_trip_and_one_way():
  g, o = grid_pair('TL255')
  x = ostates.sht_modal_input(o, 16, seed=0)
  xt = torch.as_tensor(x, device='cuda')
  nodal = g.to_nodal(xt)
  back = g.to_modal(nodal)
  err = torch.linalg.vector_norm(back - xt) / torch.linalg.vector_norm(xt)
  assert float(err) < 1e-5
  ref = o.to_nodal(x[:2].astype(np.float64))
  assert rel_err(nodal[:2], ref) < 3e-6


@pytest.mark.parametrize('name', ['T21', 'TL31', 'W16'])
def test_operators_match_oracle(name):
  g, o = grid_pair(name)
  x = ostates.sht_modal_input(o, 3, seed=4).astype(np.float64)
  xt = torch.as_tensor(x, device='cuda', dtype=torch.float32)
  for op in ('d_dlon', 'cos_lat_d_dlat', 'sec_lat_d_dlat_cos2', 'laplacian',
             'inverse_laplacian', 'clip_wavenumbers'):
    got = getattr(g, op)(xt)
    ref = getattr(o, op)(x)
    assert rel_err(got, ref) < 2e-6, op
  u, v = sh.get_cos_lat_vector(xt[0], xt[1], g, clip=False)
  uo, vo = osht.get_cos_lat_vector(x[0], x[1], o, clip=False)
  assert rel_err(u, uo) < 2e-6 and rel_err(v, vo) < 2e-6
  un, vn = sh.vor_div_to_uv_nodal(g, xt[0], xt[1])
  uno, vno = osht.vor_div_to_uv_nodal(o, x[0], x[1])
  assert rel_err(un, uno) < 1e-5 and rel_err(vn, vno) < 1e-5


@pytest.mark.parametrize('name', ['T21', 'W16', 'TL127'])
def test_adjoints_are_transposes(name):
  g, _ = grid_pair(name)
  gen = torch.Generator(device='cuda').manual_seed(0)
  x = torch.randn((3,) + g.modal_shape, device='cuda', generator=gen)
  y = torch.randn((3,) + g.nodal_shape, device='cuda', generator=gen)
  p = g.plan
  lhs = torch.sum(p.inverse(x).double() * y.double())
  rhs = torch.sum(x.double() * p.inverse_adjoint(y).double())
  assert abs(float(lhs - rhs)) <= 1e-5 * float(abs(lhs) + abs(rhs))
  lhs = torch.sum(p.forward(y).double() * x.double())
  rhs = torch.sum(y.double() * p.forward_adjoint(x).double())
  assert abs(float(lhs - rhs)) <= 1e-5 * float(abs(lhs) + abs(rhs))
  for op in ('d_dlon', 'cos_lat_d_dlat', 'sec_lat_d_dlat_cos2', 'laplacian'):
    a = p.modal_op(op, x)
    b = p.modal_op(op, x[[1, 2, 0]], transpose=True)
    lhs = torch.sum(a.double() * x[[1, 2, 0]].double())
    rhs = torch.sum(x.double() * b.double())
    assert abs(float(lhs - rhs)) <= 1e-5 * float(abs(lhs) + abs(rhs) + 1e-30), op


def test_autograd_through_transforms():
  # A quadratic loss, so the central difference is exact up to FP32 rounding.
  g, _ = grid_pair('T21')
  gen = torch.Generator(device='cuda').manual_seed(0)
  x = torch.randn((2,) + g.modal_shape, device='cuda', generator=gen)
  w = torch.randn((2,) + g.modal_shape, device='cuda', generator=gen)
  x.requires_grad_(True)
  loss = (w * g.to_modal(g.to_nodal(x) ** 2)).sum()
  loss.backward()
  gx = x.grad.clone()
  d = torch.randn(x.shape, device='cuda', generator=gen)
  eps = 0.1
  with torch.no_grad():
    lp = (w * g.to_modal(g.to_nodal(x + eps * d) ** 2)).double().sum()
    lm = (w * g.to_modal(g.to_nodal(x - eps * d) ** 2)).double().sum()
  fd = (lp - lm) / (2 * eps)
  assert abs(float(fd - (gx.double() * d).sum())) <= 1e-3 * abs(float(fd))


def test_shape_and_argument_errors():
  g, _ = grid_pair('T21')
  with pytest.raises(ValueError):
    g.clip_wavenumbers(torch.zeros(g.modal_shape, device='cuda'), n=0)
  with pytest.raises(ValueError):
    sh.Grid(longitude_wavenumbers=10, total_wavenumbers=5, longitude_nodes=64,
            latitude_nodes=32).plan
