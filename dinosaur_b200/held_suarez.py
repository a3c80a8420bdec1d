"""Held-Suarez forcing on sigma levels (dinosaur/held_suarez.py:47-167).

Constants are given in SI units (the reference takes pint quantities) and are
nondimensionalised with the default scale.  The forcing runs fused with the
primitive equations: ``time_integration.compose_equations([pe, hs])`` returns
a primitive-equation object whose explicit-terms kernel adds Rayleigh drag
and Newtonian cooling from the same diagnostic state (the reference
recomputes that state, held_suarez.py:126-128).
"""

from __future__ import annotations

import numpy as np

from dinosaur_b200 import time_integration
from dinosaur_b200 import units


class HeldSuarezForcingSigma(time_integration.ExplicitODE):

  def __init__(self, coords, physics_specs, reference_temperature,
               p0: float = 1e5, sigma_b: float = 0.7,
               kf: float = 1 / units.SECONDS_PER_DAY,
               ka: float = 1 / (40 * units.SECONDS_PER_DAY),
               ks: float = 1 / (4 * units.SECONDS_PER_DAY),
               minT: float = 200.0, maxT: float = 315.0, dTy: float = 60.0,
               dThz: float = 10.0):
    self.coords = coords
    self.physics_specs = physics_specs
    self.reference_temperature = np.asarray(reference_temperature)
    self.p0 = units.nondim_pressure(p0)
    self.sigma_b = sigma_b
    # Rates in 1/s -> nondimensional rates.
    self.kf = kf * units.TIME_SCALE
    self.ka = ka * units.TIME_SCALE
    self.ks = ks * units.TIME_SCALE
    self.minT, self.maxT, self.dTy, self.dThz = minT, maxT, dTy, dThz
    self.sigma = coords.vertical.centers

  def kv(self):
    """held_suarez.py:99-103."""
    coeff = self.kf * np.maximum(0, (self.sigma - self.sigma_b)
                                 / (1 - self.sigma_b))
    return coeff[:, None, None]

  def explicit_terms(self, state):
    raise NotImplementedError(
        'Held-Suarez forcing runs fused with the primitive equations: use '
        'time_integration.compose_equations([primitive, held_suarez])')
