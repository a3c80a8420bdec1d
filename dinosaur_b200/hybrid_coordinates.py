"""Hybrid sigma-pressure vertical coordinates (hybrid_coordinates.py:239-596).

The pressure at the boundary between layers is ``a + b * p_s``: ``a`` is a
pressure offset (hPa in the constructors below) and ``b`` the terrain-
following (sigma) part, both listed from the top of the atmosphere down.
``PrimitiveEquationsHybrid`` (``dinosaur_b200.primitive_equations``) solves
the primitive equations on these levels with the Simmons & Burridge (1981)
vertical discretisation.
"""

from __future__ import annotations

import dataclasses

import numpy as np

from dinosaur_b200 import sigma_coordinates


@dataclasses.dataclass(frozen=True)
class HybridCoordinates:
  """Hybrid levels; ``a_boundaries`` in pressure units, ``b_boundaries``
  dimensionless, both of length ``layers + 1`` (hybrid_coordinates.py:239-266)."""

  a_boundaries: np.ndarray
  b_boundaries: np.ndarray

  def __post_init__(self):
    object.__setattr__(self, 'a_boundaries', np.asarray(self.a_boundaries))
    object.__setattr__(self, 'b_boundaries', np.asarray(self.b_boundaries))
    if len(self.a_boundaries) != len(self.b_boundaries):
      raise ValueError(
          'Expected `a_boundaries` and `b_boundaries` to have the same length, '
          f'got {len(self.a_boundaries)} and {len(self.b_boundaries)}.')

  @classmethod
  def from_coefficients(cls, a_coeffs, b_coeffs, p0: float = 1000.0):
    """P = A p0 + B p_s with dimensionless A, B (:268-288)."""
    return cls(a_boundaries=np.array(a_coeffs) * p0,
               b_boundaries=np.array(b_coeffs))

  @classmethod
  def analytic_levels(cls, n_levels: int, p_top: float = 0.0, p0: float = 1000.0,
                      sigma_exponent: float = 3.0, stretch_exponent: float = 2.0):
    """Power-law blend from pressure aloft to sigma at the surface (:290-346):
    eta = (k / n)^stretch, B = eta^sigma_exponent, A = P(eta) / p0 - B."""
    eta = np.linspace(0, 1, n_levels + 1) ** stretch_exponent
    p_profile = p_top + eta * (p0 - p_top)
    b = eta ** sigma_exponent
    a = p_profile / p0 - b
    a[0] = p_top / p0
    b[0] = 0.0
    a[-1] = 0.0
    b[-1] = 1.0
    return cls.from_coefficients(a, b, p0)

  @classmethod
  def analytic_ecmwf_like(cls, n_levels: int = 137, p0: float = 1013.25,
                          p_top: float = 0.0, p_transition: float = 80.0,
                          alpha_strat: float = 4.2, alpha_surf: float = 0.25,
                          b_exponent: float = 1.3):
    """Pure pressure above p_transition, hybrid below (:348-411)."""
    k = np.linspace(0, 1, n_levels + 1)
    p_target = p_top + k ** np.linspace(alpha_strat, alpha_surf, n_levels + 1) * (
        p0 - p_top)
    a = np.zeros_like(p_target)
    b = np.zeros_like(p_target)
    for i, p in enumerate(p_target):
      if p <= p_transition:
        a[i] = p
      else:
        bv = 1.0 if i == n_levels else ((p - p_transition) / (p0 - p_transition)) ** b_exponent
        b[i] = bv
        a[i] = max(0.0, p - bv * p0)
    a[0] = 0.0
    b[0] = 0.0
    return cls(a_boundaries=a, b_boundaries=b)

  @classmethod
  def from_sigma_levels(cls, sigma_levels: sigma_coordinates.SigmaCoordinates):
    """a = 0, b = sigma: hybrid levels that are sigma levels (:464-471)."""
    b = np.array(sigma_levels.boundaries)
    return cls(a_boundaries=np.zeros_like(b), b_boundaries=b)

  @classmethod
  def ECMWF137(cls):  # pylint: disable=invalid-name
    raise NotImplementedError(
        'the ECMWF 137-level coefficient table is not bundled; build the levels '
        'with HybridCoordinates(a_boundaries, b_boundaries)')

  @classmethod
  def UFS127(cls):  # pylint: disable=invalid-name
    raise NotImplementedError(
        'the UFS 127-level coefficient table is not bundled; build the levels '
        'with HybridCoordinates(a_boundaries, b_boundaries)')

  def get_eta(self, p_surface: float) -> np.ndarray:
    return self.a_centers / p_surface + self.b_centers

  @property
  def pressure_thickness(self) -> np.ndarray:
    return np.diff(self.a_boundaries)

  @property
  def sigma_thickness(self) -> np.ndarray:
    return np.diff(self.b_boundaries)

  @property
  def a_centers(self) -> np.ndarray:
    return (self.a_boundaries[1:] + self.a_boundaries[:-1]) / 2

  @property
  def b_centers(self) -> np.ndarray:
    return (self.b_boundaries[1:] + self.b_boundaries[:-1]) / 2

  @property
  def center_to_center(self) -> np.ndarray:
    return np.diff(self.b_centers)

  @property
  def layers(self) -> int:
    return len(self.a_boundaries) - 1

  def _expand(self, x, surface_pressure):
    # One trailing axis per non-singleton axis of the surface pressure, as the
    # reference does (hybrid_coordinates.py:443-462): a (1, lon, lat) surface
    # pressure gives (levels, lon, lat) results.
    nd = sum(1 for s in np.shape(surface_pressure) if s > 1)
    return np.reshape(x, x.shape + (1,) * nd)

  def pressure_boundaries(self, surface_pressure):
    return (self._expand(self.a_boundaries, surface_pressure)
            + self._expand(self.b_boundaries, surface_pressure) * surface_pressure)

  def pressure_centers(self, surface_pressure):
    b = self.pressure_boundaries(surface_pressure)
    return (b[1:] + b[:-1]) / 2

  def layer_thickness(self, surface_pressure):
    return (self._expand(self.pressure_thickness, surface_pressure)
            + self._expand(self.sigma_thickness, surface_pressure) * surface_pressure)

  def get_sigma_boundaries(self, surface_pressure):
    return self.pressure_boundaries(surface_pressure) / surface_pressure

  def get_sigma_centers(self, surface_pressure):
    return self.pressure_centers(surface_pressure) / surface_pressure

  def __hash__(self):
    return hash((tuple(self.a_boundaries.tolist()), tuple(self.b_boundaries.tolist())))

  def __eq__(self, other):
    return (isinstance(other, HybridCoordinates)
            and np.array_equal(self.a_boundaries, other.a_boundaries)
            and np.array_equal(self.b_boundaries, other.b_boundaries))
