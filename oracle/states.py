"""FP64 initial states and the benchmark configurations' inputs.

Test infrastructure (see ``oracle/__init__.py``).  Follows
``dinosaur/primitive_equations_states.py`` (reference v1.3.6) for the
Jablonowski-Williamson steady state (:196-387), the Gaussian scalar (:504-544)
and the isothermal rest atmosphere (:37-160, deterministic part only: the
reference draws its optional surface-pressure bump with ``jax.random`` and the
configurations here use amplitude p1 = 0).
"""

from __future__ import annotations

import numpy as np

from oracle import dycore, sht


def steady_state_jw(grid: sht.Grid, vertical: dycore.SigmaCoordinates,
                    physics_specs: dycore.SimUnits, u0_si=35.0, p0_si=1e5,
                    t0=288.0, delta_t=4.8e5, gamma_si=0.005, eta_tropo=0.2,
                    eta0=0.252):
  """Returns (state, aux) with aux = {orography, ref_temperatures, geopotential}.

  primitive_equations_states.py:196-387 (sigma levels: eta = sigma centres).
  """
  u0 = dycore.nondim_velocity(u0_si)
  p0 = dycore.nondim_pressure(p0_si)
  gamma = gamma_si * dycore.LENGTH_SCALE  # K/m -> K per nondim length
  a = physics_specs.radius
  g = physics_specs.g
  r_gas = physics_specs.R
  omega = physics_specs.angular_velocity

  def ref_temperature(eta):
    top = t0 * eta ** (r_gas * gamma / g)
    if eta < eta_tropo:
      return top + delta_t * (eta_tropo - eta) ** 5
    return top

  def ref_geopotential(eta):
    top = (t0 * g / gamma) * (1 - eta ** (r_gas * gamma / g))
    if eta < eta_tropo:
      return top - r_gas * delta_t * (
          (np.log(eta / eta_tropo) + 137 / 60) * eta_tropo ** 5
          - 5 * eta * eta_tropo ** 4 + 5 * (eta ** 2) * (eta_tropo ** 3)
          - (10 / 3) * (eta_tropo ** 2) * eta ** 3
          + (5 / 4) * eta_tropo * eta ** 4 - (eta ** 5) / 5)
    return top

  def geopotential(lat, eta):
    eta_nu = (eta - eta0) * np.pi / 2
    return ref_geopotential(eta) + u0 * np.cos(eta_nu) ** 1.5 * (
        ((-2 * np.sin(lat) ** 6 * (np.cos(lat) ** 2 + 1 / 3) + 10 / 63)
         * u0 * np.cos(eta_nu) ** (3 / 2))
        + ((1.6 * (np.cos(lat) ** 3) * (np.sin(lat) ** 2 + 2 / 3) - np.pi / 4)
           * a * omega))

  def temperature_variation(lat, eta):
    eta_nu = (eta - eta0) * np.pi / 2
    c, s = np.cos(eta_nu), np.sin(eta_nu)
    return (0.75 * (eta * np.pi * u0 / r_gas) * s * np.sqrt(c) * (
        ((-2 * (np.cos(lat) ** 2 + 1 / 3) * np.sin(lat) ** 6 + 10 / 63)
         * 2 * u0 * c ** (3 / 2))
        + ((1.6 * (np.cos(lat) ** 3) * (np.sin(lat) ** 2 + 2 / 3) - np.pi / 4)
           * a * omega)))

  def vorticity(lat, eta):
    eta_nu = (eta - eta0) * np.pi / 2
    return ((-4 * u0 / a) * (np.cos(eta_nu) ** (3 / 2)) * np.sin(lat)
            * np.cos(lat) * (2 - 5 * np.sin(lat) ** 2))

  _, sin_lat = grid.nodal_mesh
  lat = np.arcsin(sin_lat)
  etas = vertical.centers
  nodal_vorticity = np.stack([vorticity(lat, eta) for eta in etas])
  nodal_temperature = np.stack([temperature_variation(lat, eta) for eta in etas])
  log_ps = np.log(p0 * np.ones(lat.shape)[None])
  state = dycore.make_state(
      vorticity=grid.to_modal(nodal_vorticity),
      divergence=np.zeros(grid.modal_shape)[None].repeat(len(etas), 0),
      temperature_variation=grid.to_modal(nodal_temperature),
      log_surface_pressure=grid.to_modal(log_ps))
  aux = dict(
      orography=geopotential(lat, 1.0) / g,
      geopotential=np.stack([geopotential(lat, eta) for eta in etas]),
      ref_temperatures=np.stack([ref_temperature(eta) for eta in etas]))
  return state, aux


def gaussian_scalar_nodal(grid: sht.Grid, layers: int, lon_location=np.pi / 9,
                          lat_location=2 * np.pi / 9, perturbation_radius=0.2,
                          amplitude=1.0, radius=1.0):
  """Nodal values of gaussian_scalar (primitive_equations_states.py:504-544)."""
  lon, sin_lat = grid.nodal_mesh
  lat = np.arcsin(sin_lat)
  x = (np.sin(lat_location) * np.sin(lat)
       + np.cos(lat_location) * np.cos(lat) * np.cos(lon - lon_location))
  r = radius * np.arccos(np.clip(x, -1, 1))
  big_r = radius * perturbation_radius
  field = amplitude * np.exp(-((r / big_r) ** 2))
  return np.stack([field] * layers)


def gaussian_scalar(grid: sht.Grid, layers: int, **kw):
  return grid.to_modal(gaussian_scalar_nodal(grid, layers, **kw))


def isothermal_rest_atmosphere(grid: sht.Grid, vertical, tref=288.0,
                               p0_si=1e5):
  """Flat rest state (primitive_equations_states.py:37-160 with p1 = 0)."""
  k = vertical.layers
  p0 = dycore.nondim_pressure(p0_si)
  zeros = np.zeros((k,) + grid.modal_shape)
  log_ps = grid.to_modal(np.log(p0 * np.ones((1,) + grid.nodal_shape)))
  state = dycore.make_state(zeros, zeros.copy(), zeros.copy(), log_ps)
  aux = dict(orography=np.zeros(grid.nodal_shape),
             ref_temperatures=np.full((k,), tref))
  return state, aux


# ---------------------------------------------------------------------------
# Benchmark-configuration inputs (seeded synthetic data).
# ---------------------------------------------------------------------------

def sht_modal_input(grid: sht.Grid, batch: int, seed: int = 0,
                    dtype=np.float32) -> np.ndarray:
  """Seeded modal coefficients for the SHT microbenchmark.

  Complex Gaussians (Re -> cos row, Im -> sin row, m = 0 real only) scaled by
  (l+1)^-1.5, masked to |m| <= l, with the top total wavenumber zeroed.
  """
  rng = np.random.default_rng(seed)
  m_axis, l_axis = grid.modal_axes
  lw = grid.longitude_wavenumbers
  re = rng.standard_normal((batch, lw, grid.total_wavenumbers))
  im = rng.standard_normal((batch, lw, grid.total_wavenumbers))
  out = np.zeros((batch,) + grid.modal_shape)
  out[:, 0] = re[:, 0]
  out[:, 1::2] = re[:, 1:]
  out[:, 2::2] = im[:, 1:]
  out *= grid.mask / (l_axis + 1.0) ** 1.5
  out[..., -1] = 0
  return out.astype(dtype)


def baroclinic_config(grid: sht.Grid, layers: int, seed: int = 0,
                      physics_specs=None, amplitude=1.0,
                      radius_km=500.0):
  """JW steady state plus a seeded Gaussian temperature bump on all levels.

  Returns (state, ref_temperatures, modal_orography, vertical).
  """
  physics_specs = physics_specs or dycore.SimUnits()
  vertical = dycore.SigmaCoordinates.equidistant(layers)
  state, aux = steady_state_jw(grid, vertical, physics_specs)
  rng = np.random.default_rng(seed)
  lon0 = rng.uniform(0, 2 * np.pi)
  lat0 = rng.uniform(-np.pi / 3, np.pi / 3)
  bump = gaussian_scalar(grid, layers, lon_location=lon0, lat_location=lat0,
                         perturbation_radius=radius_km / 6371.22,
                         amplitude=amplitude)
  state['temperature_variation'] = state['temperature_variation'] + bump
  orography = dycore.truncated_modal_orography(aux['orography'], grid)
  return state, aux['ref_temperatures'], orography, vertical


def held_suarez_config(grid: sht.Grid, layers: int, member: int = 0,
                       tref=285.0, noise_k=0.1):
  """Rest state at tref plus seeded white noise (sigma = noise_k) in T'."""
  vertical = dycore.SigmaCoordinates.equidistant(layers)
  state, aux = isothermal_rest_atmosphere(grid, vertical, tref=tref)
  rng = np.random.default_rng(member)
  noise = noise_k * rng.standard_normal((layers,) + grid.nodal_shape)
  state['temperature_variation'] = grid.to_modal(noise)
  return state, aux['ref_temperatures'], np.zeros(grid.modal_shape), vertical
