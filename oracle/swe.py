"""FP64 restatement of the reference's shallow-water equations.

Test infrastructure only (the checker for the CUDA path).  States are dicts
with 'vorticity', 'divergence', 'potential' arrays of shape [layers, M, L].
Follows dinosaur/shallow_water.py and dinosaur/shallow_water_states.py.
"""

from __future__ import annotations

import numpy as np

from oracle import sht

SWE_KEYS = ('vorticity', 'divergence', 'potential')


def make_state(vorticity, divergence, potential):
  return dict(vorticity=vorticity, divergence=divergence, potential=potential)


def tree_map(fn, *states):
  return {k: fn(*[s[k] for s in states]) for k in SWE_KEYS}


def tree_axpy(*terms):
  coeffs = [c for c, _ in terms]
  states = [s for _, s in terms]
  return tree_map(lambda *xs: sum(c * x for c, x in zip(coeffs, xs)), *states)


def get_density_ratios(density) -> np.ndarray:
  """shallow_water.py:71-86: D[i, j] = rho_i / rho_j (i < j), 0 (i = j),
  1 (i > j), for densities ordered from the top."""
  density = np.asarray(density, np.float64)
  ratios = np.minimum(density / density[..., np.newaxis], 1)
  np.fill_diagonal(ratios, 0)
  return ratios


def get_coriolis(grid: sht.Grid) -> np.ndarray:
  """shallow_water.py:89-92 (sin(lat) on the nodal mesh)."""
  _, sin_lat = grid.nodal_mesh
  return sin_lat


class ShallowWaterEquations:
  """shallow_water.py:121-230."""

  def __init__(self, grid: sht.Grid, physics_specs, orography,
               reference_potential, densities=np.ones((1,))):
    self.grid = grid
    self.physics_specs = physics_specs
    self.orography = orography
    self.reference_potential = np.asarray(reference_potential, np.float64)
    self.densities = np.asarray(densities, np.float64)

  @property
  def coriolis_parameter(self):
    """shallow_water.py:142-146: 2 Omega sin(lat)."""
    _, sin_lat = self.grid.nodal_mesh
    return 2 * self.physics_specs.angular_velocity * sin_lat

  @property
  def density_ratios(self):
    return get_density_ratios(self.densities)

  @property
  def ref_potential(self):
    return self.reference_potential[..., np.newaxis, np.newaxis]

  def explicit_terms(self, state):
    """shallow_water.py:158-205."""
    grid = self.grid
    u = np.stack(sht.get_cos_lat_vector(state['vorticity'],
                                        state['divergence'], grid))
    nodal_u = grid.to_nodal(u)
    nodal_vorticity = grid.to_nodal(grid.clip_wavenumbers(state['vorticity']))
    nodal_potential = grid.to_nodal(grid.clip_wavenumbers(state['potential']))
    total_vorticity = nodal_vorticity + self.coriolis_parameter
    sec2 = grid.sec2_lat
    nodal_b = nodal_u * total_vorticity * sec2
    nodal_g = nodal_u * nodal_potential * sec2
    nodal_e = (nodal_u * nodal_u).sum(0) * sec2 / 2
    b = grid.to_modal(nodal_b)
    g = grid.to_modal(nodal_g)
    e = grid.to_modal(nodal_e)
    p = np.einsum('ab,...bml->...aml', self.density_ratios, state['potential'])
    if self.orography is not None:
      p = p + self.orography
    vort = grid.clip_wavenumbers(-grid.div_cos_lat(b))
    div = grid.clip_wavenumbers(-grid.laplacian(p + e) + grid.curl_cos_lat(b))
    pot = grid.clip_wavenumbers(-grid.div_cos_lat(g))
    return make_state(vort, div, pot)

  def implicit_terms(self, state):
    """shallow_water.py:207-213."""
    return make_state(np.zeros_like(state['vorticity']),
                      -self.grid.laplacian(state['potential']),
                      -self.ref_potential * state['divergence'])

  def implicit_inverse(self, state, step_size):
    """shallow_water.py:215-230 (closed-form Schur complement per l)."""
    grid = self.grid
    inv = 1 / (1 - step_size ** 2 * self.ref_potential *
               grid.laplacian_eigenvalues)
    return make_state(
        state['vorticity'],
        inv * (state['divergence'] - step_size * grid.laplacian(state['potential'])),
        inv * (-step_size * self.ref_potential * state['divergence'] +
               state['potential']))


def imex_rk_sil3(equation, dt):
  """time_integration.py:329-405 on SWE states (SIL3 tableau)."""
  a_ex = [[1 / 3], [1 / 6, 1 / 2], [1 / 2, -1 / 2, 1]]
  a_im = [[1 / 6, 1 / 6], [1 / 3, 0, 1 / 3], [3 / 8, 0, 3 / 8, 1 / 4]]
  b_ex = [1 / 2, -1 / 2, 1, 0]
  b_im = [3 / 8, 0, 3 / 8, 1 / 4]
  F, G, Ginv = (equation.explicit_terms, equation.implicit_terms,
                equation.implicit_inverse)

  def step(y0):
    f = [F(y0)] + [None] * 3
    g = [G(y0)] + [None] * 3
    for i in range(1, 4):
      terms = [(1.0, y0)]
      terms += [(dt * a_ex[i - 1][j], f[j]) for j in range(i) if a_ex[i - 1][j]]
      terms += [(dt * a_im[i - 1][j], g[j]) for j in range(i) if a_im[i - 1][j]]
      y = Ginv(tree_axpy(*terms), dt * a_im[i - 1][i])
      if i < 3 or b_ex[i]:
        f[i] = F(y)
      g[i] = G(y)
    terms = [(1.0, y0)]
    terms += [(dt * b_ex[j], f[j]) for j in range(4) if b_ex[j]]
    terms += [(dt * b_im[j], g[j]) for j in range(4) if b_im[j]]
    return tree_axpy(*terms)

  return step


def filtered_step(step, scaling):
  """step_with_filters with a per-l spectral scaling (time_integration.py:494-505)."""
  return lambda y: tree_map(lambda x: x * scaling, step(y))


def one_layer(u, grid: sht.Grid):
  """shallow_water_states.py:50-85: steady zonal flow of one layer."""
  sec_lat = 1 / grid.cos_lat
  lon, _ = grid.nodal_axes
  u = np.ones_like(lon)[..., np.newaxis] * u
  sec_lat_u = u * sec_lat
  vorticity = -grid.sec_lat_d_dlat_cos2(grid.to_modal(sec_lat_u))
  f = get_coriolis(grid)
  total_vorticity = grid.to_nodal(vorticity) + f
  potential_plus_energy = -grid.inverse_laplacian(
      grid.sec_lat_d_dlat_cos2(grid.to_modal(sec_lat_u * total_vorticity)))
  potential = potential_plus_energy - grid.to_modal(u ** 2 / 2)
  potential = np.array(potential)
  potential[0, 0] = 0
  return make_state(vorticity, np.zeros_like(vorticity), potential)


def multi_layer(u, density, grid: sht.Grid):
  """shallow_water_states.py:88-119: u is [layers, lat]; potentials solve
  (D + I) phi = phi_one_layer across layers."""
  layers = [one_layer(ui, grid) for ui in u]
  s = {k: np.stack([st[k] for st in layers]) for k in SWE_KEYS}
  n = len(layers)
  ratios = get_density_ratios(density) + np.eye(n)
  potential = s['potential']
  if n > 1:
    flat = potential.reshape(n, -1)
    potential = np.linalg.solve(ratios, flat).reshape(potential.shape)
  return make_state(s['vorticity'], s['divergence'], potential)
