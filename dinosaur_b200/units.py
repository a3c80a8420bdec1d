"""Nondimensional physical constants (plain floats).

Mirrors ``SimUnits`` (dinosaur/units.py:92-199) with the default scale of
dinosaur/scales.py:206-228 (length = Earth radius, time = 1/(2 Omega),
mass = 1 kg, temperature = 1 K).  Values are plain floats; the reference's
pint quantities are not needed on this path.
"""

from __future__ import annotations

import dataclasses

RADIUS_SI = 6.37122e6            # m (scales.py:37-44)
OMEGA_SI = 7.292e-5              # 1/s
GRAVITY_SI = 9.80616             # m/s^2
CP_SI = 1004.0                   # J/kg/K
KAPPA = 2 / 7
R_SI = CP_SI * KAPPA             # J/kg/K
R_VAPOR_SI = 461.0               # J/kg/K
CP_VAPOR_SI = 1859.0             # J/kg/K

LENGTH_SCALE = RADIUS_SI
TIME_SCALE = 1 / 2 / OMEGA_SI
MASS_SCALE = 1.0
SECONDS_PER_DAY = 86400.0


def nondim_time(seconds: float) -> float:
  return seconds / TIME_SCALE


def nondim_pressure(pascal: float) -> float:
  return pascal * LENGTH_SCALE * TIME_SCALE ** 2 / MASS_SCALE


def nondim_velocity(m_per_s: float) -> float:
  return m_per_s * TIME_SCALE / LENGTH_SCALE


def nondim_specific_gas(j_per_kg_k: float) -> float:
  return j_per_kg_k * TIME_SCALE ** 2 / LENGTH_SCALE ** 2


@dataclasses.dataclass(frozen=True)
class SimUnits:
  """Nondimensional constants with the reference's attribute names."""

  radius: float = 1.0
  angular_velocity: float = OMEGA_SI * TIME_SCALE
  gravity_acceleration: float = GRAVITY_SI * TIME_SCALE ** 2 / LENGTH_SCALE
  ideal_gas_constant: float = nondim_specific_gas(R_SI)
  water_vapor_gas_constant: float = nondim_specific_gas(R_VAPOR_SI)
  water_vapor_isobaric_heat_capacity: float = nondim_specific_gas(CP_VAPOR_SI)
  kappa: float = KAPPA

  @classmethod
  def from_si(cls, ideal_gas_constant_si: float = R_SI,
              kappa_si: float = KAPPA, **kw) -> SimUnits:
    return cls(ideal_gas_constant=nondim_specific_gas(ideal_gas_constant_si),
               kappa=kappa_si, **kw)

  @property
  def R(self): return self.ideal_gas_constant
  @property
  def R_vapor(self): return self.water_vapor_gas_constant
  @property
  def g(self): return self.gravity_acceleration
  @property
  def Cp(self): return self.ideal_gas_constant / self.kappa
  @property
  def Cp_vapor(self): return self.water_vapor_isobaric_heat_capacity

  def nondimensionalize_seconds(self, seconds: float) -> float:
    return nondim_time(seconds)
