"""Edge cases of the transform path (CUDA through the C ABI).

* empty batches return empty results without a launch error;
* a field's result does not depend on the batch around it: ragged batch
  sizes that split into L2-sized chunks (TL255: 64 fields per chunk) and
  batches larger than a plan's workspace give bit-identical results to
  single-field calls, in every Legendre form;
* grids with nodes at the poles ('equiangular_with_poles') match the FP64
  oracle (<= 2e-6 max-abs relative, as the other one-way transforms).
"""

import functools

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


def grid(name, precision='fp32', **kw):
  impl = functools.partial(sh.CudaSphericalHarmonics, precision=precision)
  return getattr(sh.Grid, name)(spherical_harmonics_impl=impl, **kw)


@pytest.mark.parametrize('precision', ['fp32', 'bf16x3', 'tf32x3'])
def test_empty_batches(precision):
  g = grid('T42', precision)
  x = torch.empty((0,) + g.modal_shape, device='cuda')
  y = g.to_nodal(x)
  assert tuple(y.shape) == (0,) + g.nodal_shape
  z = g.to_modal(torch.empty((0,) + g.nodal_shape, device='cuda'))
  assert tuple(z.shape) == (0,) + g.modal_shape
  _lib.check(_lib.lib().dino_plan_status(g.plan.handle))


@pytest.mark.parametrize('precision', ['fp32', 'bf16x3', 'tf32x3'])
def test_fields_do_not_depend_on_their_batch(precision):
  g = grid('TL255', precision)
  og = osht.Grid.TL255()
  n = 67  # one full 64-field chunk plus a ragged remainder of 3
  x = torch.as_tensor(ost.sht_modal_input(og, n, seed=5), device='cuda')
  nodal = g.to_nodal(x)
  modal = g.to_modal(nodal)
  for i in (0, 37, 63, 64, 66):
    torch.testing.assert_close(g.to_nodal(x[i:i + 1])[0], nodal[i], rtol=0, atol=0)
    torch.testing.assert_close(g.to_modal(nodal[i:i + 1])[0], modal[i], rtol=0,
                               atol=0)
  _lib.check(_lib.lib().dino_plan_status(g.plan.handle))


def test_batches_larger_than_the_workspace():
  og = osht.Grid.T42()
  small = sh.Plan(43, 44, 128, 64, 'gauss', max_fields=5)
  big = sh.Grid.T42().plan
  x = torch.as_tensor(ost.sht_modal_input(og, 23, seed=6), device='cuda')
  a = small.inverse(x)
  torch.testing.assert_close(a, big.inverse(x), rtol=0, atol=0)
  torch.testing.assert_close(small.forward(a), big.forward(a), rtol=0, atol=0)


def test_equiangular_with_poles_matches_oracle():
  g = sh.Grid.with_wavenumbers(16, latitude_spacing='equiangular_with_poles')
  og = osht.Grid.with_wavenumbers(16, latitude_spacing='equiangular_with_poles')
  x = ost.sht_modal_input(og, 3, seed=7).astype(np.float64)
  got = g.to_nodal(torch.as_tensor(x, device='cuda', dtype=torch.float32))
  ref = og.to_nodal(x)
  err = np.abs(got.double().cpu().numpy() - ref).max() / np.abs(ref).max()
  assert err < 2e-6, err
  z = np.random.default_rng(8).standard_normal((3,) + og.nodal_shape)
  got = g.to_modal(torch.as_tensor(z, device='cuda', dtype=torch.float32))
  ref = og.to_modal(z.astype(np.float32).astype(np.float64))
  err = np.abs(got.double().cpu().numpy() - ref).max() / np.abs(ref).max()
  assert err < 2e-6, err
