"""FP64 NumPy oracle for the spectral dynamical-core step.

TEST INFRASTRUCTURE ONLY. This package restates, in double precision NumPy,
the algorithm of neuralgcm/dinosaur 1.3.6 for the hot path that
``dinosaur_b200`` implements in CUDA: the spherical-harmonic transform pair,
the spectral operators, the sigma-coordinate and hybrid-coordinate primitive
equations (explicit terms, implicit terms, implicit inverse), the
``imex_rk_sil3`` integrator with
its exponential step filter, Held-Suarez forcing and the initial states used
as fixtures.  Every function cites the reference file and line range it
follows.

Only the test suite, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py`` may import this package, and only as
the reference values a result is compared with, or as the timed CPU baseline.  The product path (``dinosaur_b200``)
never imports it and fails loudly when its CUDA library is missing.

Parity pins: ``tests/golden/make_golden.py`` imports the reference's own
modules (with small NumPy stand-ins for ``jax``, ``tree_math`` and ``pint``,
none of which are installed here) and records their outputs; the oracle is
checked against those fixtures in ``tests/test_oracle_golden.py`` and against
the reference test suite's analytic identities in ``tests/test_oracle.py``.
"""

from oracle import sht, dycore, states  # noqa: F401
