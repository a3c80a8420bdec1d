"""The allocation-free inverse transform, checked against dino_sht_inverse.

dino_sht_inverse_noalloc is for callers that may not allocate device memory
when they call in (a handler inside a framework that owns the GPU memory pool,
or a loop that cannot pay for cudaMalloc's device synchronisation).  It keeps
its intermediate coefficients in a fixed array inside the library.  Here it
is called twice in a row through the C ABI, with different inputs, and each
result must match the regular entry point (same FP32 kernels) within the
transform tests' tolerance (max-abs error <= 2e-6 of the max-abs value).
This file is collected last so that a run stopping at the first failure has
already run every other test.
"""

import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

from dinosaur_b200 import _lib  # noqa: E402
from dinosaur_b200 import spherical_harmonic as sh  # noqa: E402


def _noalloc(plan, x, out):
  return _lib.lib().dino_sht_inverse_noalloc(
      plan.handle, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(out.data_ptr()),
      x.shape[0], sh.stream_handle())


@pytest.mark.parametrize('name,fields', [('T42', 64), ('TL255', 24)])
def test_noalloc_matches_regular_inverse_on_two_calls(name, fields):
  grid = getattr(sh.Grid, name)()
  plan = grid.plan
  gen = torch.Generator(device='cuda').manual_seed(11)
  mask = torch.as_tensor(grid.mask, device='cuda', dtype=torch.float32)
  for call in range(2):
    x = torch.randn((fields,) + grid.modal_shape, device='cuda',
                    generator=gen) * mask
    expected = plan.inverse(x)
    out = torch.full((fields,) + grid.nodal_shape, float('nan'), device='cuda')
    _lib.check(_noalloc(plan, x, out), 'dino_sht_inverse_noalloc')
    torch.cuda.synchronize()
    err = float((out - expected).abs().max() / expected.abs().max())
    assert err <= 2e-6, (call, err)


def test_noalloc_rejects_batches_beyond_the_fixed_scratch():
  grid = sh.Grid.TL255()
  plan = grid.plan
  m, j = grid.modal_shape[0], grid.nodal_shape[1]
  too_many = (4 * 1024 * 1024) // (m * j) + 1
  x = torch.zeros((too_many,) + grid.modal_shape, device='cuda')
  out = torch.zeros((too_many,) + grid.nodal_shape, device='cuda')
  rc = _noalloc(plan, x, out)
  assert rc == _lib.DINO_ERR_SHAPE
  assert 'exceeds the fixed scratch' in _lib.last_error()


def test_noalloc_empty_batch_is_a_no_op_with_null_buffers():
  plan = sh.Grid.T21().plan
  rc = _lib.lib().dino_sht_inverse_noalloc(plan.handle, None, None, 0,
                                           sh.stream_handle())
  assert rc == _lib.DINO_OK
  rc = _lib.lib().dino_sht_inverse_noalloc(plan.handle, None, None, 1,
                                           sh.stream_handle())
  assert rc == _lib.DINO_ERR_ARG
