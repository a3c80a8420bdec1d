"""FP64 restatement of dinosaur's sigma-coordinate primitive-equation step.

Test infrastructure (see ``oracle/__init__.py``).  Follows reference v1.3.6:
``dinosaur/scales.py`` + ``dinosaur/units.py`` (nondimensional constants),
``dinosaur/sigma_coordinates.py`` (vertical integrals and advection),
``dinosaur/primitive_equations.py`` (``PrimitiveEquationsSigma``),
``dinosaur/held_suarez.py`` (``HeldSuarezForcingSigma``),
``dinosaur/time_integration.py`` (``imex_rk_sil3``, step filters) and
``dinosaur/filtering.py``.

States are plain dicts with the reference ``State`` field names
(``vorticity``, ``divergence``, ``temperature_variation``,
``log_surface_pressure``, ``tracers``); modal arrays are ``[levels, m, l]``.
"""

from __future__ import annotations

import dataclasses
import functools

import numpy as np

from oracle import sht


# ---------------------------------------------------------------------------
# Units (scales.py:37-77, :206-228; units.py:92-199)
# ---------------------------------------------------------------------------

RADIUS_SI = 6.37122e6            # m
OMEGA_SI = 7.292e-5              # 1/s
GRAVITY_SI = 9.80616             # m/s^2
CP_SI = 1004.0                   # J/kg/K
KAPPA = 2 / 7
R_SI = CP_SI * KAPPA             # J/kg/K
R_VAPOR_SI = 461.0               # J/kg/K
CP_VAPOR_SI = 1859.0             # J/kg/K

# NEURALGCM_V1_SCALE: length = radius, time = 1/(2 omega), mass = 1 kg, 1 K.
LENGTH_SCALE = RADIUS_SI
TIME_SCALE = 1 / 2 / OMEGA_SI
MASS_SCALE = 1.0


def nondim_time(seconds):
  return seconds / TIME_SCALE


def nondim_pressure(pascal):
  # Pa = kg m^-1 s^-2
  return pascal * LENGTH_SCALE * TIME_SCALE ** 2 / MASS_SCALE


def nondim_velocity(m_per_s):
  return m_per_s * TIME_SCALE / LENGTH_SCALE


def nondim_length(m):
  return m / LENGTH_SCALE


def nondim_specific_gas(j_per_kg_k):
  return j_per_kg_k * TIME_SCALE ** 2 / LENGTH_SCALE ** 2


@dataclasses.dataclass(frozen=True)
class SimUnits:
  """Nondimensional physical constants (units.py:92-199)."""

  radius: float = 1.0
  angular_velocity: float = OMEGA_SI * TIME_SCALE
  gravity_acceleration: float = GRAVITY_SI * TIME_SCALE ** 2 / LENGTH_SCALE
  ideal_gas_constant: float = nondim_specific_gas(R_SI)
  water_vapor_gas_constant: float = nondim_specific_gas(R_VAPOR_SI)
  water_vapor_isobaric_heat_capacity: float = nondim_specific_gas(CP_VAPOR_SI)
  kappa: float = KAPPA

  @classmethod
  def from_si(cls, ideal_gas_constant_si=R_SI, kappa_si=KAPPA) -> SimUnits:
    return cls(ideal_gas_constant=nondim_specific_gas(ideal_gas_constant_si),
               kappa=kappa_si)

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


# ---------------------------------------------------------------------------
# Sigma coordinates (sigma_coordinates.py:59-405)
# ---------------------------------------------------------------------------

def _with_f64_math(f):
  """sigma_coordinates.py:51-52: compute in f64, return in the input dtype."""
  return lambda x: f(x.astype(np.float64)).astype(x.dtype)


@dataclasses.dataclass(frozen=True, eq=False)
class SigmaCoordinates:
  """Sigma levels; properties keep the dtype of ``boundaries``."""

  boundaries: np.ndarray

  def __post_init__(self):
    b = np.asarray(self.boundaries)
    if not (np.isclose(b[0], 0) and np.isclose(b[-1], 1)):
      raise ValueError('Expected boundaries[0] = 0, boundaries[-1] = 1, '
                       f'got boundaries = {b}')
    if not all(np.diff(b) > 0):
      raise ValueError('Expected `boundaries` to be monotonically increasing, '
                       f'got boundaries = {b}')
    object.__setattr__(self, 'boundaries', b)

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


def cumulative_sigma_integral(x, coords: SigmaCoordinates, downward=True):
  """Midpoint rule cumulative integral over sigma (:201-258)."""
  xds = x * coords.layer_thickness[:, None, None]
  if downward:
    return np.cumsum(xds, axis=-3)
  return np.flip(np.cumsum(np.flip(xds, -3), axis=-3), -3)


def sigma_integral(x, coords: SigmaCoordinates, keepdims=True):
  """:261-278."""
  xds = x * coords.layer_thickness[:, None, None]
  return xds.sum(axis=-3, keepdims=keepdims)


def centered_difference(x, coords: SigmaCoordinates):
  """(x[n+1] - x[n]) / (sigma[n+1] - sigma[n]) (:161-198).

  Like the reference, the reciprocal spacing is formed in the dtype of the
  sigma boundaries (float32 for ``equidistant``) before it multiplies x.
  """
  inv_dsigma = 1 / coords.center_to_center
  return np.diff(x, axis=-3) * inv_dsigma[:, None, None]


def centered_vertical_advection(w, x, coords: SigmaCoordinates):
  """-(w dx/dsigma) at centres, zero boundary values (:344-405).

  ``w`` holds K-1 values at internal boundaries; ``x`` holds K centre values
  (x may be a (K, 1, 1) column that broadcasts against w).
  """
  zeros_w = np.zeros((1,) + w.shape[1:])
  wp = np.concatenate([zeros_w, w, zeros_w], axis=-3)
  xd = centered_difference(x, coords)
  zeros_x = np.zeros((1,) + xd.shape[1:])
  xdp = np.concatenate([zeros_x, xd, zeros_x], axis=-3)
  prod = wp * xdp
  return -0.5 * (prod[1:] + prod[:-1])


# ---------------------------------------------------------------------------
# Vertical weight matrices (primitive_equations.py:283-598)
# ---------------------------------------------------------------------------

def get_sigma_ratios(coords: SigmaCoordinates):
  """:283-303."""
  alpha = np.diff(np.log(coords.centers), append=0) / 2
  alpha[-1] = -np.log(coords.centers[-1])
  return alpha


def get_geopotential_weights(coords: SigmaCoordinates, ideal_gas_constant):
  """G matrix (:306-338)."""
  alpha = get_sigma_ratios(coords)
  k = coords.layers
  weights = np.zeros([k, k])
  for j in range(k):
    weights[j, j] = alpha[j]
    for kk in range(j + 1, k):
      weights[j, kk] = alpha[kk] + alpha[kk - 1]
  return ideal_gas_constant * weights


def get_temperature_implicit_weights(coords: SigmaCoordinates,
                                     reference_temperature, kappa):
  """H matrix (:419-502)."""
  reference_temperature = np.asarray(reference_temperature)
  k = coords.layers
  p = np.tril(np.ones([k, k]))
  alpha = get_sigma_ratios(coords)[..., None]
  p_alpha = p * alpha
  p_alpha_shifted = np.roll(p_alpha, 1, axis=0)
  p_alpha_shifted[0] = 0
  h0 = (kappa * reference_temperature[..., None] * (p_alpha + p_alpha_shifted)
        / coords.layer_thickness[..., None])
  temp_diff = np.diff(reference_temperature)
  thickness_sum = coords.layer_thickness[:-1] + coords.layer_thickness[1:]
  k0 = np.concatenate((temp_diff / thickness_sum, [0]), axis=0)[..., None]
  thickness_cumulative = np.cumsum(coords.layer_thickness)[..., None]
  k1 = p - thickness_cumulative
  kk = k0 * k1
  k_shifted = np.roll(kk, 1, axis=0)
  k_shifted[0] = 0
  return (h0 - kk - k_shifted) * coords.layer_thickness


def implicit_term_matrix(eta, grid: sht.Grid, coords: SigmaCoordinates,
                         reference_temperature, kappa, ideal_gas_constant):
  """Per-l (2K+1)^2 matrix of (1 - eta * implicit_terms) (:544-598)."""
  k = coords.layers
  eye = np.eye(k)[None]
  lam = grid.laplacian_eigenvalues
  g = get_geopotential_weights(coords, ideal_gas_constant)
  r = ideal_gas_constant
  h = get_temperature_implicit_weights(coords, reference_temperature, kappa)
  t = np.asarray(reference_temperature)[:, None]
  thickness = coords.layer_thickness[None, None, :]
  nl = grid.total_wavenumbers
  row0 = np.concatenate([
      np.broadcast_to(eye, [nl, k, k]),
      eta * np.einsum('l,jk->ljk', lam, g),
      eta * r * np.einsum('l,jo->ljo', lam, t)], axis=2)
  row1 = np.concatenate([
      eta * np.broadcast_to(h[None], [nl, k, k]),
      np.broadcast_to(eye, [nl, k, k]),
      np.zeros([nl, k, 1])], axis=2)
  row2 = np.concatenate([
      np.broadcast_to(eta * thickness, [nl, 1, k]),
      np.zeros([nl, 1, k]),
      np.ones([nl, 1, 1])], axis=2)
  return np.concatenate((row0, row1, row2), axis=1)


def _vertical_matvec(a, x):
  """'gh,...hml->...gml' (:122-125)."""
  return np.einsum('gh,...hml->...gml', a, x)


def _vertical_matvec_per_wavenumber(a, x):
  """'lgh,...hml->...gml' (:127-130)."""
  return np.einsum('lgh,...hml->...gml', a, x)


# ---------------------------------------------------------------------------
# State helpers
# ---------------------------------------------------------------------------

STATE_KEYS = ('vorticity', 'divergence', 'temperature_variation',
              'log_surface_pressure')


def make_state(vorticity, divergence, temperature_variation,
               log_surface_pressure, tracers=None):
  return dict(vorticity=vorticity, divergence=divergence,
              temperature_variation=temperature_variation,
              log_surface_pressure=log_surface_pressure,
              tracers=dict(tracers or {}))


def tree_map(fn, *states):
  out = {k: fn(*[s[k] for s in states]) for k in STATE_KEYS}
  out['tracers'] = {name: fn(*[s['tracers'][name] for s in states])
                    for name in states[0]['tracers']}
  return out


def tree_axpy(*terms):
  """sum_i c_i * state_i for (c_i, state_i) pairs (tree_math vector ops)."""
  coeffs = [c for c, _ in terms]
  states = [s for _, s in terms]
  return tree_map(lambda *xs: sum(c * x for c, x in zip(coeffs, xs)), *states)


# ---------------------------------------------------------------------------
# Primitive equations on sigma levels (primitive_equations.py:670-1458)
# ---------------------------------------------------------------------------

@dataclasses.dataclass
class DiagnosticState:
  vorticity: np.ndarray
  divergence: np.ndarray
  temperature_variation: np.ndarray
  cos_lat_u: tuple
  sigma_dot_explicit: np.ndarray
  sigma_dot_full: np.ndarray
  cos_lat_grad_log_sp: tuple
  u_dot_grad_log_sp: np.ndarray
  tracers: dict


def compute_diagnostic_state(state, grid: sht.Grid, vertical: SigmaCoordinates):
  """Nodal diagnostics (primitive_equations.py:168-225)."""
  nodal_vorticity = grid.to_nodal(state['vorticity'])
  nodal_divergence = grid.to_nodal(state['divergence'])
  nodal_temperature = grid.to_nodal(state['temperature_variation'])
  tracers = {k: grid.to_nodal(v) for k, v in state['tracers'].items()}
  cos_lat_u = tuple(grid.to_nodal(c) for c in sht.get_cos_lat_vector(
      state['vorticity'], state['divergence'], grid, clip=False))
  grad = grid.cos_lat_grad(state['log_surface_pressure'], clip=False)
  nodal_grad = tuple(grid.to_nodal(g) for g in grad)
  u_dot_grad = sum(x * y * grid.sec2_lat for x, y in zip(cos_lat_u, nodal_grad))
  f_explicit = cumulative_sigma_integral(u_dot_grad, vertical)
  f_full = cumulative_sigma_integral(nodal_divergence + u_dot_grad, vertical)
  sum_sigma = np.cumsum(vertical.layer_thickness)[:, None, None]
  sigma_dot_explicit = (sum_sigma * f_explicit[-1:] - f_explicit)[:-1]
  sigma_dot_full = (sum_sigma * f_full[-1:] - f_full)[:-1]
  return DiagnosticState(nodal_vorticity, nodal_divergence, nodal_temperature,
                         cos_lat_u, sigma_dot_explicit, sigma_dot_full,
                         nodal_grad, u_dot_grad, tracers)


def truncated_modal_orography(orography, grid: sht.Grid, wavenumbers_to_clip=1):
  """primitive_equations.py:626-636."""
  return grid.clip_wavenumbers(grid.to_modal(orography), n=wavenumbers_to_clip)


@dataclasses.dataclass
class PrimitiveEquationsSigma:
  """FP64 oracle of PrimitiveEquationsSigma (primitive_equations.py:835-1458)."""

  reference_temperature: np.ndarray
  orography: np.ndarray
  grid: sht.Grid
  vertical: SigmaCoordinates
  physics_specs: SimUnits
  include_vertical_advection: bool = True
  humidity_key: str | None = None
  cloud_keys: tuple | None = None

  @property
  def T_ref(self):
    return np.asarray(self.reference_temperature)[:, None, None]

  @functools.cached_property
  def coriolis_parameter(self):
    """:726-730."""
    _, sin_lat = self.grid.nodal_mesh
    return 2 * self.physics_specs.angular_velocity * sin_lat

  def _vertical_tendency(self, w, x):
    return centered_vertical_advection(w, x, self.vertical)

  def _virtual_temperature_adjustment(self, aux):
    """:690-703."""
    if self.humidity_key is None:
      return 1.0
    q = aux.tracers[self.humidity_key]
    ratio = self.physics_specs.R_vapor / self.physics_specs.R
    adjustment = 1 + (ratio - 1) * q
    if self.cloud_keys is not None:
      for key in self.cloud_keys:
        adjustment = adjustment - aux.tracers[key]
    return adjustment

  def kinetic_energy_tendency(self, aux):
    """:778-785."""
    u2 = aux.cos_lat_u[0] ** 2 + aux.cos_lat_u[1] ** 2
    kinetic = u2 * self.grid.sec2_lat / 2
    return -self.grid.laplacian(self.grid.to_modal(kinetic))

  def orography_tendency(self):
    """:787-793."""
    return -self.physics_specs.g * self.grid.laplacian(self.orography)

  def div_sec_lat(self, m_component, n_component):
    """:601-623."""
    m = self.grid.to_modal(m_component * self.grid.sec2_lat)
    n = self.grid.to_modal(n_component * self.grid.sec2_lat)
    return self.grid.div_cos_lat((m, n), clip=False)

  def horizontal_scalar_advection(self, scalar, aux):
    """:795-805."""
    u, v = aux.cos_lat_u
    return scalar * aux.divergence, -self.div_sec_lat(u * scalar, v * scalar)

  def _t_omega_over_sigma_sp(self, temperature_field, g_term, v_dot_grad_log_sp):
    """:965-999."""
    f = cumulative_sigma_integral(g_term, self.vertical)
    alpha = get_sigma_ratios(self.vertical)[:, None, None]
    del_sigma = self.vertical.layer_thickness[:, None, None]
    af = alpha * f
    af_shift = np.concatenate([np.zeros_like(af[:1]), af[:-1]], axis=0)
    g_part = (af + af_shift) / del_sigma
    return temperature_field * (v_dot_grad_log_sp - g_part)

  def curl_and_div_tendencies(self, aux):
    """:1001-1059."""
    sec2 = self.grid.sec2_lat
    u, v = aux.cos_lat_u
    total_vorticity = aux.vorticity + self.coriolis_parameter
    nodal_vorticity_u = -v * total_vorticity * sec2
    nodal_vorticity_v = u * total_vorticity * sec2
    dsdt = aux.sigma_dot_full
    if self.include_vertical_advection:
      sigma_dot_u = -self._vertical_tendency(dsdt, u)
      sigma_dot_v = -self._vertical_tendency(dsdt, v)
    else:
      sigma_dot_u = sigma_dot_v = 0
    adjustment = self._virtual_temperature_adjustment(aux)
    rt = self.physics_specs.R * aux.temperature_variation * adjustment
    gx, gy = aux.cos_lat_grad_log_sp
    vertical_term_u = (sigma_dot_u + rt * gx) * sec2
    vertical_term_v = (sigma_dot_v + rt * gy) * sec2
    cu = self.grid.to_modal(nodal_vorticity_u + vertical_term_u)
    cv = self.grid.to_modal(nodal_vorticity_v + vertical_term_v)
    return (-self.grid.curl_cos_lat((cu, cv), clip=False),
            -self.grid.div_cos_lat((cu, cv), clip=False))

  def nodal_temperature_vertical_tendency(self, aux):
    """:1061-1079."""
    if self.include_vertical_advection:
      tendency = self._vertical_tendency(aux.sigma_dot_full,
                                         aux.temperature_variation)
    else:
      tendency = 0
    if np.unique(self.T_ref.ravel()).size > 1:
      tendency = tendency + self._vertical_tendency(aux.sigma_dot_explicit,
                                                    self.T_ref)
    return tendency

  def nodal_temperature_adiabatic_tendency(self, aux):
    """:1081-1115."""
    g_explicit = aux.u_dot_grad_log_sp
    g_full = g_explicit + aux.divergence
    mean_t_part = self._t_omega_over_sigma_sp(self.T_ref, g_explicit,
                                              aux.u_dot_grad_log_sp)
    ps = self.physics_specs
    if self.humidity_key is None:
      variation_t_part = self._t_omega_over_sigma_sp(
          aux.temperature_variation, g_full, aux.u_dot_grad_log_sp)
      return ps.kappa * (mean_t_part + variation_t_part)
    ratio = ps.R_vapor / ps.R
    hc_ratio = ps.Cp_vapor / ps.Cp
    q = aux.tracers[self.humidity_key]
    variation = aux.temperature_variation * (
        (1 + (ratio - 1) * q) / (1 + (hc_ratio - 1) * q))
    humidity_ref = self.T_ref * (((ratio - hc_ratio) * q)
                                 / (1 + (hc_ratio - 1) * q))
    part = self._t_omega_over_sigma_sp(variation + humidity_ref, g_full,
                                       aux.u_dot_grad_log_sp)
    return ps.kappa * (mean_t_part + part)

  def nodal_log_pressure_tendency(self, aux):
    """:1117-1124."""
    return -sigma_integral(aux.u_dot_grad_log_sp, self.vertical)

  def vorticity_tendency_due_to_humidity(self, state, aux):
    """:937-963."""
    ps = self.physics_specs
    q_modal = state['tracers'][self.humidity_key]
    gq = [self.grid.to_nodal(c) for c in
          self.grid.cos_lat_grad(q_modal, clip=False)]
    gl = aux.cos_lat_grad_log_sp
    coefficient = self.T_ref * (ps.R_vapor - ps.R)
    curl_term = coefficient * self.grid.sec2_lat * (gl[0] * gq[1]
                                                    - gl[1] * gq[0])
    return self.grid.to_modal(curl_term)

  def divergence_tendency_due_to_humidity(self, state, aux):
    """:861-935 (dense vertical matmul)."""
    ps = self.physics_specs
    q = aux.tracers[self.humidity_key]
    nodal_lap_lsp = self.grid.to_nodal(
        self.grid.laplacian(state['log_surface_pressure']))
    correction = q * nodal_lap_lsp * self.T_ref * (ps.R_vapor - ps.R)
    q_modal = state['tracers'][self.humidity_key]
    gq = [self.grid.to_nodal(c) for c in
          self.grid.cos_lat_grad(q_modal, clip=False)]
    coefficient = self.T_ref * (ps.R_vapor - ps.R)
    gl = aux.cos_lat_grad_log_sp
    dot_term = coefficient * self.grid.sec2_lat * (gq[0] * gl[0]
                                                   + gq[1] * gl[1])
    temperature = aux.temperature_variation + self.T_ref
    temperature_diff = q * temperature * (ps.R_vapor / ps.R - 1)
    g = get_geopotential_weights(self.vertical, ps.R)
    geopotential_diff = _vertical_matvec(g, temperature_diff)
    return (-self.grid.laplacian(self.grid.to_modal(geopotential_diff))
            - self.grid.to_modal(dot_term + correction))

  def explicit_terms(self, state):
    """:1126-1194."""
    aux = compute_diagnostic_state(state, self.grid, self.vertical)
    vort_dot, div_dot = self.curl_and_div_tendencies(aux)
    ke = self.kinetic_energy_tendency(aux)
    orog = self.orography_tendency()
    if self.humidity_key is not None:
      vort_dot = vort_dot + self.vorticity_tendency_due_to_humidity(state, aux)
      div_dot = div_dot + self.divergence_tendency_due_to_humidity(state, aux)
    dT_h_nodal, dT_h_modal = self.horizontal_scalar_advection(
        aux.temperature_variation, aux)
    tracer_terms = {k: self.horizontal_scalar_advection(v, aux)
                    for k, v in aux.tracers.items()}
    dT_vertical = self.nodal_temperature_vertical_tendency(aux)
    dT_adiabatic = self.nodal_temperature_adiabatic_tendency(aux)
    lsp = self.nodal_log_pressure_tendency(aux)
    if self.include_vertical_advection:
      vert = lambda x: self._vertical_tendency(aux.sigma_dot_full, x)
    else:
      vert = lambda x: 0
    to_modal = self.grid.to_modal
    tendency = make_state(
        vorticity=vort_dot,
        divergence=div_dot + ke + orog,
        temperature_variation=(to_modal(dT_h_nodal + dT_vertical + dT_adiabatic)
                               + dT_h_modal),
        log_surface_pressure=to_modal(lsp),
        tracers={k: to_modal(vert(aux.tracers[k]) + nm[0]) + nm[1]
                 for k, nm in tracer_terms.items()})
    return tree_map(self.grid.clip_wavenumbers, tendency)

  def implicit_terms(self, state):
    """:1196-1249 (dense vertical matmuls)."""
    ps = self.physics_specs
    g = get_geopotential_weights(self.vertical, ps.R)
    geopotential_diff = _vertical_matvec(g, state['temperature_variation'])
    rt_log_p = ps.ideal_gas_constant * self.T_ref * state['log_surface_pressure']
    h = get_temperature_implicit_weights(self.vertical,
                                         self.reference_temperature, ps.kappa)
    return make_state(
        vorticity=np.zeros_like(state['vorticity']),
        divergence=-self.grid.laplacian(geopotential_diff + rt_log_p),
        temperature_variation=_vertical_matvec(-h, state['divergence']),
        log_surface_pressure=-_vertical_matvec(
            self.vertical.layer_thickness[None], state['divergence']),
        tracers={k: np.zeros_like(v) for k, v in state['tracers'].items()})

  @functools.lru_cache(maxsize=16)
  def implicit_inverse_matrix(self, step_size: float):
    """FP64 inverse of the per-l implicit matrix (:1273-1296, 'split')."""
    mat = implicit_term_matrix(step_size, self.grid, self.vertical,
                               self.reference_temperature,
                               self.physics_specs.kappa, self.physics_specs.R)
    inverse = np.linalg.inv(mat)
    assert not np.isnan(inverse).any()
    return inverse

  def implicit_inverse(self, state, step_size: float):
    """(1 - step_size * implicit_terms)^-1, 'split' method (:1251-1330)."""
    inverse = self.implicit_inverse_matrix(float(step_size))
    k = self.vertical.layers
    div, temp, logp = slice(0, k), slice(k, 2 * k), slice(2 * k, 2 * k + 1)
    mv = _vertical_matvec_per_wavenumber
    d, t, p = (state['divergence'], state['temperature_variation'],
               state['log_surface_pressure'])
    out_d = mv(inverse[:, div, div], d) + mv(inverse[:, div, temp], t) + mv(
        inverse[:, div, logp], p)
    out_t = mv(inverse[:, temp, div], d) + mv(inverse[:, temp, temp], t) + mv(
        inverse[:, temp, logp], p)
    out_p = mv(inverse[:, logp, div], d) + mv(inverse[:, logp, temp], t) + mv(
        inverse[:, logp, logp], p)
    return make_state(state['vorticity'], out_d, out_t, out_p,
                      state['tracers'])

  def __hash__(self):
    return id(self)


# ---------------------------------------------------------------------------
# Held-Suarez forcing (held_suarez.py:47-167)
# ---------------------------------------------------------------------------

DAY_SI = 86400.0


@dataclasses.dataclass
class HeldSuarezForcingSigma:
  grid: sht.Grid
  vertical: SigmaCoordinates
  physics_specs: SimUnits
  reference_temperature: np.ndarray
  p0: float = nondim_pressure(1e5)
  sigma_b: float = 0.7
  kf: float = 1 / nondim_time(1 * DAY_SI)
  ka: float = 1 / nondim_time(40 * DAY_SI)
  ks: float = 1 / nondim_time(4 * DAY_SI)
  minT: float = 200.0
  maxT: float = 315.0
  dTy: float = 60.0
  dThz: float = 10.0

  @property
  def sigma(self):
    return self.vertical.centers

  @property
  def lat(self):
    _, sin_lat = self.grid.nodal_mesh
    return np.arcsin(sin_lat)

  def kv(self):
    """:99-103."""
    coeff = self.kf * np.maximum(0, (self.sigma - self.sigma_b)
                                 / (1 - self.sigma_b))
    return coeff[:, None, None]

  def kt(self):
    """:105-109."""
    cutoff = np.maximum(0, (self.sigma - self.sigma_b) / (1 - self.sigma_b))
    return self.ka + (self.ks - self.ka) * (
        cutoff[:, None, None] * np.cos(self.lat) ** 4)

  def equilibrium_temperature(self, nodal_surface_pressure):
    """:111-120."""
    p_over_p0 = self.sigma[:, None, None] * nodal_surface_pressure / self.p0
    temperature = p_over_p0 ** self.physics_specs.kappa * (
        self.maxT - self.dTy * np.sin(self.lat) ** 2
        - self.dThz * np.log(p_over_p0) * np.cos(self.lat) ** 2)
    return np.maximum(self.minT, temperature)

  def explicit_terms(self, state):
    """:122-167."""
    aux = compute_diagnostic_state(state, self.grid, self.vertical)
    cos2 = self.grid.cos_lat ** 2
    vel = tuple(-self.kv() * x / cos2 for x in aux.cos_lat_u)
    temperature = (np.asarray(self.reference_temperature)[:, None, None]
                   + aux.temperature_variation)
    ps = np.exp(self.grid.to_nodal(state['log_surface_pressure']))
    teq = self.equilibrium_temperature(ps)
    t_tend = -self.kt() * (temperature - teq)
    vel_m = tuple(self.grid.to_modal(v) for v in vel)
    return make_state(
        vorticity=self.grid.curl_cos_lat(vel_m),
        divergence=self.grid.div_cos_lat(vel_m),
        temperature_variation=self.grid.to_modal(t_tend),
        log_surface_pressure=np.zeros_like(state['log_surface_pressure']),
        tracers={k: np.zeros_like(v) for k, v in state['tracers'].items()})


@dataclasses.dataclass
class ComposedEquation:
  """compose_equations for one implicit-explicit equation (time_integration.py:141-161)."""

  equations: list

  def explicit_terms(self, state):
    tendencies = [eq.explicit_terms(state) for eq in self.equations]
    return tree_map(lambda *xs: sum(xs), *tendencies)

  def implicit_terms(self, state):
    return self.equations[0].implicit_terms(state)

  def implicit_inverse(self, state, step_size):
    return self.equations[0].implicit_inverse(state, step_size)


# ---------------------------------------------------------------------------
# Time integration (time_integration.py:313-455, :494-520)
# ---------------------------------------------------------------------------

SIL3 = dict(
    a_ex=[[1 / 3], [1 / 6, 1 / 2], [1 / 2, -1 / 2, 1]],
    a_im=[[1 / 6, 1 / 6], [1 / 3, 0, 1 / 3], [3 / 8, 0, 3 / 8, 1 / 4]],
    b_ex=[1 / 2, -1 / 2, 1, 0],
    b_im=[3 / 8, 0, 3 / 8, 1 / 4],
)


def imex_runge_kutta(tableau, equation, dt):
  """Generic IMEX-RK step (time_integration.py:329-372)."""
  a_ex, a_im, b_ex, b_im = (tableau['a_ex'], tableau['a_im'], tableau['b_ex'],
                            tableau['b_im'])
  n = len(b_ex)

  def step_fn(y0):
    f = [None] * n
    g = [None] * n
    f[0] = equation.explicit_terms(y0)
    g[0] = equation.implicit_terms(y0)
    for i in range(1, n):
      terms = [(1.0, y0)]
      terms += [(dt * a_ex[i - 1][j], f[j]) for j in range(i) if a_ex[i - 1][j]]
      terms += [(dt * a_im[i - 1][j], g[j]) for j in range(i) if a_im[i - 1][j]]
      y_star = tree_axpy(*terms)
      y = equation.implicit_inverse(y_star, dt * a_im[i - 1][i])
      if any(a_ex[j][i] for j in range(i, n - 1)) or b_ex[i]:
        f[i] = equation.explicit_terms(y)
      if any(a_im[j][i] for j in range(i, n - 1)) or b_im[i]:
        g[i] = equation.implicit_terms(y)
    terms = [(1.0, y0)]
    terms += [(dt * b_ex[j], f[j]) for j in range(n) if b_ex[j]]
    terms += [(dt * b_im[j], g[j]) for j in range(n) if b_im[j]]
    return tree_axpy(*terms)

  return step_fn


def imex_rk_sil3(equation, dt):
  """time_integration.py:375-405."""
  return imex_runge_kutta(SIL3, equation, dt)


def exponential_step_filter(grid: sht.Grid, dt, tau=0.010938, order=18,
                            cutoff=0.0):
  """time_integration.py:427-455 with filtering.py:38-89."""
  scaling = sht.exponential_filter_scaling(grid, dt / tau, order, cutoff)
  return lambda u, u_next: tree_map(lambda x: scaling * x, u_next)


def step_with_filters(step_fn, filters):
  """time_integration.py:494-505."""
  def _step(u):
    u_next = step_fn(u)
    for flt in filters:
      u_next = flt(u, u_next)
    return u_next
  return _step


class TimeReversedImExODE:
  """dx/dt = -explicit(x) - implicit(x) (time_integration.py:117-138)."""

  def __init__(self, forward_eq):
    self.forward_eq = forward_eq

  def explicit_terms(self, state):
    return tree_map(np.negative, self.forward_eq.explicit_terms(state))

  def implicit_terms(self, state):
    return tree_map(np.negative, self.forward_eq.implicit_terms(state))

  def implicit_inverse(self, state, step_size):
    return self.forward_eq.implicit_inverse(state, -step_size)


def accumulate_repeated(step_fn, weights, state):
  """time_integration.py:645-660: sum_n w_n x_n along x_{n+1} = step(x_n)."""
  averaged = tree_map(np.zeros_like, state)
  for w in weights:
    state = step_fn(state)
    averaged = tree_map(lambda s, a, w=w: a + w * s, state, averaged)
  return averaged


def dfi_lanczos_weights(time_span, cutoff_period, dt):
  """time_integration.py:663-670."""
  n_steps = round(time_span / (2 * dt))
  n = np.arange(1, n_steps + 1)
  return (np.sinc(n / (n_steps + 1)) *
          np.sinc(n * time_span / (cutoff_period * n_steps)))


def digital_filter_initialization(equation, ode_solver, filters, time_span,
                                  cutoff_period, dt):
  """time_integration.py:673-716 (Lynch & Huang 1992)."""
  def f(state):
    forward = step_with_filters(ode_solver(equation, dt), filters)
    backward = step_with_filters(
        ode_solver(TimeReversedImExODE(equation), dt), filters)
    weights = dfi_lanczos_weights(time_span, cutoff_period, dt)
    total = 1.0 + 2 * weights.sum()
    weights = weights / total
    init = tree_map(lambda x: x / total, state)
    fwd = accumulate_repeated(forward, weights, state)
    bwd = accumulate_repeated(backward, weights, state)
    return tree_map(lambda *xs: sum(xs), init, fwd, bwd)
  return f


def repeated(fn, steps):
  """time_integration.py:508-520 (a Python loop instead of lax.scan)."""
  def f(x):
    for _ in range(steps):
      x = fn(x)
    return x
  return f
