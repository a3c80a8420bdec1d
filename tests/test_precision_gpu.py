"""The three Legendre forms on the SHT microbenchmark's inputs, against the
FP64 oracle.

Grids T85 and TL255, a batch of 128 fields of seeded complex Gaussians
scaled by (l+1)^-1.5 with the top total wavenumber zeroed
(``oracle.states.sht_modal_input``, seed 0).  Per form:

* inverse (modal -> nodal) one way against the oracle's FP64 transform of the
  same FP32 input;
* forward (nodal -> modal) one way against the oracle's FP64 transform of the
  FP32-rounded oracle nodal field;
* round trip to_modal(to_nodal(x)) against x.

Errors are relative L2 over the batch and max-abs relative (to the largest
reference magnitude).  Bounds: 'fp32' (SIMT FMA) and 'tf32x3' (11-bit tf32
halves, dropped lo*lo term ~2^-22 relative) relative L2 <= 2e-6, max-abs
<= 1e-5; 'bf16x3' (8-bit bf16 halves, dropped term ~2^-16) relative L2 <= 1e-5,
max-abs <= 5e-5.

``python tests/test_precision_gpu.py`` prints the table of measured errors.
"""

import functools
import os
import sys

import numpy as np
import pytest
import torch

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

from oracle import sht as osht  # noqa: E402
from oracle import states as ost  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _tensor_cores_only(monkeypatch):
  # These tests exercise the tensor-core kernels themselves: keep them even
  # on grids where the plan's autotuner would pick the FP32 SIMT contraction.
  monkeypatch.setenv('DINO_B200_TENSOR_CORES_ONLY', '1')

FORMS = ['fp32', 'bf16x3', 'tf32x3']
BOUNDS = {'fp32': (2e-6, 1e-5), 'bf16x3': (1e-5, 5e-5), 'tf32x3': (2e-6, 1e-5)}
FIELDS = 128

_REF = {}


def _reference(name):
  """FP32 modal input, the FP64 oracle's nodal field of it, the FP32-rounded
  nodal field and the oracle's FP64 modal transform of that (cached)."""
  if name not in _REF:
    og = getattr(osht.Grid, name)()
    x = ost.sht_modal_input(og, FIELDS, seed=0)
    nodal = og.to_nodal(x.astype(np.float64))
    z = nodal.astype(np.float32)
    modal = og.to_modal(z.astype(np.float64))
    _REF[name] = (x, nodal, z, modal)
  return _REF[name]


def _errs(got, ref):
  got = got.detach().double().cpu().numpy()
  return (float(np.linalg.norm(got - ref) / np.linalg.norm(ref)),
          float(np.abs(got - ref).max() / np.abs(ref).max()))


def form_errors(name, precision):
  """{'inverse': (l2, max), 'forward': (l2, max), 'round_trip': (l2, max)}."""
  from dinosaur_b200 import _lib
  from dinosaur_b200 import spherical_harmonic as sh
  impl = functools.partial(sh.CudaSphericalHarmonics, precision=precision)
  g = getattr(sh.Grid, name)(spherical_harmonics_impl=impl)
  x, nodal, z, modal = _reference(name)
  xd = torch.as_tensor(x, device='cuda')
  y = g.to_nodal(xd)
  out = {'inverse': _errs(y, nodal),
         'forward': _errs(g.to_modal(torch.as_tensor(z, device='cuda')), modal),
         'round_trip': _errs(g.to_modal(y), x.astype(np.float64))}
  _lib.check(_lib.lib().dino_plan_status(g.plan.handle))
  return out


@pytest.mark.parametrize('precision', FORMS)
@pytest.mark.parametrize('name', ['T85', 'TL255'])
def test_forms_against_fp64_oracle(name, precision):
  tl2, tmax = BOUNDS[precision]
  for what, (l2, mx) in form_errors(name, precision).items():
    assert l2 < tl2 and mx < tmax, (what, l2, mx)


if __name__ == '__main__':
  print('| grid | form | inverse L2 / max | forward L2 / max | round trip L2 / max |')
  print('|---|---|---|---|---|')
  for name in ['T85', 'TL255']:
    for precision in FORMS:
      e = form_errors(name, precision)
      cells = ['%.2e / %.2e' % e[k] for k in ('inverse', 'forward', 'round_trip')]
      print('| %s | %s | %s |' % (name, precision, ' | '.join(cells)), flush=True)
