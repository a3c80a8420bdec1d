"""dinosaur_b200: a B200-native spectral dynamical-core step.

Drop-in for the hot path of neuralgcm/dinosaur (``Grid.to_nodal/to_modal``,
the spectral operators, ``PrimitiveEquationsSigma`` explicit/implicit/inverse
terms and ``imex_rk_sil3`` with step filters), implemented as hand-written
sm_100a CUDA kernels behind the C ABI in ``include/dino_b200.h``.
"""

__version__ = '0.1.0'
