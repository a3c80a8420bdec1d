"""Sigma levels (host FP64/float32 constants), mirroring
``SigmaCoordinates`` (dinosaur/sigma_coordinates.py:59-153).

The vertical integrals and advection of sigma_coordinates.py:161-405 run
inside the fused nodal kernel of ``libdino_b200``; this module keeps the
coordinate object and the constants the kernels consume, computed with the
reference's dtype rules (properties are returned in the dtype of the
boundaries, float32 for ``equidistant``).
"""

from __future__ import annotations

import dataclasses

import numpy as np


def _with_f64_math(f):
  return lambda x: f(x.astype(np.float64)).astype(x.dtype)


@dataclasses.dataclass(frozen=True, eq=False)
class SigmaCoordinates:
  boundaries: np.ndarray

  def __init__(self, boundaries):
    b = np.asarray(boundaries)
    if not (np.isclose(b[0], 0) and np.isclose(b[-1], 1)):
      raise ValueError('Expected boundaries[0] = 0, boundaries[-1] = 1, '
                       f'got boundaries = {b}')
    if not all(np.diff(b) > 0):
      raise ValueError('Expected `boundaries` to be monotonically increasing, '
                       f'got boundaries = {b}')
    object.__setattr__(self, 'boundaries', b)

  @property
  def internal_boundaries(self):
    return self.boundaries[1:-1]

  @property
  def centers(self):
    return _with_f64_math(lambda x: (x[1:] + x[:-1]) / 2)(self.boundaries)

  @property
  def layer_thickness(self):
    return _with_f64_math(np.diff)(self.boundaries)

  @property
  def center_to_center(self):
    return _with_f64_math(np.diff)(self.centers)

  @property
  def layers(self):
    return len(self.boundaries) - 1

  @classmethod
  def equidistant(cls, layers: int, dtype=np.float32) -> SigmaCoordinates:
    return cls(np.linspace(0, 1, layers + 1, dtype=dtype))

  @classmethod
  def from_centers(cls, centers):
    def centers_to_boundaries(c):
      n = len(c)
      m = 0.5 * (np.eye(n) + np.eye(n, k=-1))
      return np.pad(np.linalg.solve(m, c), [(1, 0)])
    return cls(_with_f64_math(centers_to_boundaries)(np.asarray(centers)))

  def asdict(self):
    return {'boundaries': self.boundaries.tolist()}

  def __hash__(self):
    return hash(tuple(self.centers.tolist()))

  def __eq__(self, other):
    return isinstance(other, SigmaCoordinates) and np.array_equal(
        self.centers, other.centers)
