"""Failure paths on the GPU, made to happen without a fault.

* A bounded device wait that runs out: dino_plan_check_wait_timeout runs the
  tensor-core pipelines' own wait routine on an mbarrier that nothing ever
  completes, with a 50 ms limit.  The wait gives up and records a code;
  dino_plan_status reports DINO_ERR_TIMEOUT once (the flag is cleared by the
  read), and the context still runs transforms correctly afterwards.
* A non-finite implicit operator (the reference asserts that the inverse
  has no NaN, primitive_equations.py:1296): a NaN step size is refused on the
  host (ValueError); an infinite reference temperature makes the GPU
  factorisation's pivot check fail, so the call returns DINO_ERR_NAN, raised
  as an AssertionError; no bad operator is cached and valid calls still work.
"""

import functools

import numpy as np
import pytest
import torch

from oracle import sht as osht
from oracle import states as ost

pytestmark = pytest.mark.gpu

from dinosaur_b200 import _lib  # noqa: E402
from dinosaur_b200 import coordinate_systems  # noqa: E402
from dinosaur_b200 import primitive_equations as pe  # noqa: E402
from dinosaur_b200 import sigma_coordinates  # noqa: E402
from dinosaur_b200 import spherical_harmonic as sh  # noqa: E402
from dinosaur_b200 import units  # noqa: E402

from pe_cases import make, to_state  # noqa: E402


def test_bounded_wait_gives_up_and_reports_timeout():
  impl = functools.partial(sh.CudaSphericalHarmonics, precision='bf16x3')
  g = sh.Grid.T21(spherical_harmonics_impl=impl)
  plan = g.plan
  lib = _lib.lib()
  assert lib.dino_plan_status(plan.handle) == _lib.DINO_OK
  rc = lib.dino_plan_check_wait_timeout(plan.handle, 50_000_000, sh.stream_handle())
  assert rc == _lib.DINO_OK
  assert lib.dino_plan_status(plan.handle) == _lib.DINO_ERR_TIMEOUT
  assert 'gave up' in _lib.last_error()
  assert lib.dino_plan_status(plan.handle) == _lib.DINO_OK  # cleared by the read
  # Limits outside 1 ms .. 10 s are refused on the host.
  assert (lib.dino_plan_check_wait_timeout(plan.handle, 10, sh.stream_handle())
          == _lib.DINO_ERR_ARG)
  # The context is intact: a transform pair still matches the FP64 oracle.
  og = osht.Grid.T21()
  x = ost.sht_modal_input(og, 4)
  nodal = g.to_nodal(torch.as_tensor(x, device='cuda'))
  ref = og.to_nodal(x.astype(np.float64))
  err = float(np.abs(nodal.double().cpu().numpy() - ref).max() / np.abs(ref).max())
  assert err < 5e-5, err
  assert lib.dino_plan_status(plan.handle) == _lib.DINO_OK


def test_fp32_plan_has_no_tensor_core_wait():
  plan = sh.Grid.T21().plan
  assert (_lib.lib().dino_plan_check_wait_timeout(plan.handle, 50_000_000,
                                                  sh.stream_handle())
          == _lib.DINO_ERR_UNSUPPORTED)


@pytest.mark.filterwarnings('ignore:invalid value:RuntimeWarning')
def test_nonfinite_implicit_operator_is_refused():
  og, oeq, st, g, eq = make()
  s = to_state(st)
  # A NaN step size is refused on the host.
  with pytest.raises(ValueError):
    eq.implicit_inverse(s, float('nan'))
  # An infinite reference temperature makes the operators non-finite: the
  # GPU factorisation flags it.
  layers = 6
  coords = coordinate_systems.CoordinateSystem(
      g, sigma_coordinates.SigmaCoordinates.equidistant(layers))
  tref = np.linspace(220.0, 288.0, layers)
  tref[2] = np.inf
  bad = pe.PrimitiveEquationsSigma(tref, np.zeros(g.modal_shape, np.float32), coords,
                                   units.SimUnits())
  with pytest.raises(AssertionError) as info:
    bad.implicit_inverse(s, 0.05)
  assert isinstance(info.value, _lib.DinoError)
  assert info.value.code == _lib.DINO_ERR_NAN
  # Nothing was cached: the same call fails again, and valid equations work.
  with pytest.raises(AssertionError):
    bad.implicit_inverse(s, 0.05)
  good = eq.implicit_inverse(s, 0.05)
  assert all(bool(torch.isfinite(t).all()) for t in
             (good.vorticity, good.divergence, good.temperature_variation,
              good.log_surface_pressure))
