"""FP64 restatement of dinosaur's hybrid-coordinate primitive equations.

Test infrastructure (see ``oracle/__init__.py``).  Follows reference v1.3.6:
``dinosaur/hybrid_coordinates.py`` (``HybridCoordinates``, :239-471) and
``dinosaur/primitive_equations.py`` (``compute_diagnostic_state_hybrid``,
the Simmons & Burridge helpers and ``PrimitiveEquationsHybrid``,
:1467-2533).  The terms shared with the sigma equations (kinetic energy,
orography, horizontal advection, virtual temperature) come from
``oracle.dycore.PrimitiveEquationsSigma``, which follows the same base class
(:670-833).

Parity pins: ``tests/golden/pe_hybrid_T21_L6.npz`` holds the reference's own
PrimitiveEquationsHybrid outputs (explicit, implicit, implicit inverse, one
filtered SIL3 step on 6 analytic levels; the same on 6 ECMWF-like levels
whose top two layers are pure pressure in
``pe_hybrid_ecmwf_like_T21_L6.npz``; moist explicit terms with a tracer in
``pe_hybrid_moist_T21_L6.npz``), written by
``tests/golden/make_golden.py`` and checked in ``tests/test_oracle_golden.py``;
the reference test suite's sigma-like equivalence and implicit-inverse
identity are checked in ``tests/test_hybrid_oracle.py``.
"""

from __future__ import annotations

import dataclasses
import functools

import numpy as np

from oracle import dycore
from oracle import sht


@dataclasses.dataclass(frozen=True)
class HybridCoordinates:
  """a_boundaries (pressure units) and b_boundaries, top down (:239-266)."""

  a_boundaries: np.ndarray
  b_boundaries: np.ndarray

  @property
  def layers(self):
    return len(self.a_boundaries) - 1

  @property
  def pressure_thickness(self):
    return np.diff(self.a_boundaries)

  @property
  def sigma_thickness(self):
    return np.diff(self.b_boundaries)

  def layer_thickness(self, ps):
    """:456-462; ps scalar or nodal [lon, lat]."""
    ps = np.asarray(ps, np.float64)
    ex = (slice(None),) + (None,) * ps.ndim
    return self.pressure_thickness[ex] + self.sigma_thickness[ex] * ps

  @classmethod
  def from_sigma_levels(cls, sigma: dycore.SigmaCoordinates):
    """:464-471."""
    b = np.asarray(sigma.boundaries, np.float64)
    return cls(np.zeros_like(b), b)

  @classmethod
  def analytic_levels(cls, n_levels, p_top=0.0, p0=1000.0, sigma_exponent=3.0,
                      stretch_exponent=2.0):
    """:290-346 (coefficients times p0, :268-288)."""
    eta = np.linspace(0, 1, n_levels + 1) ** stretch_exponent
    p_profile = p_top + eta * (p0 - p_top)
    b = eta ** sigma_exponent
    a = p_profile / p0 - b
    a[0], b[0], a[-1], b[-1] = p_top / p0, 0.0, 0.0, 1.0
    return cls(a * p0, b)


def vertical_coeffs(levels: HybridCoordinates, ps):
  """(alpha_k, log(p_{k+1/2} / p_{k-1/2})) for scalar or nodal ps (:1483-1533)."""
  ps = np.asarray(ps, np.float64)
  ex = (slice(None),) + (None,) * ps.ndim
  p_half = levels.a_boundaries[ex] + levels.b_boundaries[ex] * ps
  dp = np.diff(p_half, axis=0)
  if ps.ndim == 0 and np.any(dp <= 0):
    raise ValueError('Pressure must decrease monotonically with height.')
  upper, lower = p_half[:-1], p_half[1:]
  log_ratio = np.log(np.maximum(lower, 1e-6 * ps) / np.maximum(upper, 1e-6 * ps))
  return 1 - (upper / dp) * log_ratio, log_ratio


def geopotential_weights(levels, R, ps_ref):
  """:1605-1625."""
  alpha, log_ratio = vertical_coeffs(levels, ps_ref)
  k = levels.layers
  w = np.zeros([k, k])
  for i in range(k):
    w[i, i] = alpha[i]
    for j in range(i + 1, k):
      w[i, j] = log_ratio[j]
  return R * w


def geopotential_diff_sparse(temperature, levels, R, ps):
  """'sparse' method with a per-column surface pressure (:1628-1675)."""
  alpha, log_ratio = vertical_coeffs(levels, ps)
  weighted = temperature * log_ratio
  full = np.cumsum(weighted[::-1], axis=0)[::-1]
  return R * ((full - weighted) + alpha * temperature)


def temperature_implicit_weights(levels, tref, kappa, ps_ref):
  """:1736-1783."""
  tref = np.asarray(tref, np.float64)
  k = levels.layers
  p = np.tril(np.ones([k, k]))
  alpha, _ = vertical_coeffs(levels, ps_ref)
  p_alpha = p * alpha[:, None]
  p_alpha_shifted = np.roll(p_alpha, 1, axis=0)
  p_alpha_shifted[0] = 0
  dp_ref = levels.pressure_thickness + levels.sigma_thickness * ps_ref
  h0 = kappa * tref[:, None] * (p_alpha + p_alpha_shifted) / dp_ref[:, None]
  k0 = np.concatenate((np.diff(tref) / (dp_ref[:-1] + dp_ref[1:]), [0]))[:, None]
  k1 = p - np.cumsum(levels.sigma_thickness)[:, None]
  kk = k0 * k1
  kk_shifted = np.roll(kk, 1, axis=0)
  kk_shifted[0] = 0
  return (h0 - kk - kk_shifted) * dp_ref


def pgf_coefficient(temperature, ps, levels, R):
  """C_k = (R T / dp_k) (log-ratio_k b_{k-1/2} + alpha_k db_k) p_s
  (:1826-1887; scalar or nodal ps)."""
  ps = np.asarray(ps, np.float64)
  ex = (slice(None),) + (None,) * ps.ndim
  alpha, log_ratio = vertical_coeffs(levels, ps)
  b_minus = levels.b_boundaries[:-1][ex]
  db = np.diff(levels.b_boundaries)[ex]
  dp = np.maximum(levels.layer_thickness(ps), 1e-6 * ps)
  weight = log_ratio * b_minus + alpha * db
  return (R * temperature / dp) * weight * ps


def implicit_term_matrix(eta, grid: sht.Grid, levels, tref, kappa, R, ps_ref):
  """:1890-1938."""
  k = levels.layers
  eye = np.eye(k)[None]
  lam = grid.laplacian_eigenvalues
  g = geopotential_weights(levels, R, ps_ref)
  h = temperature_implicit_weights(levels, tref, kappa, ps_ref)
  pgf = pgf_coefficient(np.asarray(tref, np.float64), ps_ref, levels, R)
  thick = levels.pressure_thickness / ps_ref + levels.sigma_thickness
  nl = grid.modal_shape[1]
  row0 = np.concatenate([np.broadcast_to(eye, [nl, k, k]),
                         eta * np.einsum('l,jk->ljk', lam, g),
                         eta * np.einsum('l,j->lj', lam, pgf)[..., None]], axis=2)
  row1 = np.concatenate([eta * np.broadcast_to(h[None], [nl, k, k]),
                         np.broadcast_to(eye, [nl, k, k]),
                         np.zeros([nl, k, 1])], axis=2)
  row2 = np.concatenate([np.broadcast_to(eta * thick[None, :], [nl, 1, k]),
                         np.zeros([nl, 1, k]), np.ones([nl, 1, 1])], axis=2)
  return np.concatenate((row0, row1, row2), axis=1)


def hybrid_vertical_advection(mass_flux, x, dp):
  """:1941-1958."""
  flux = mass_flux[1:-1] * np.diff(x, axis=0)
  pad = np.concatenate([np.zeros_like(flux[:1]), flux, np.zeros_like(flux[:1])])
  return -0.5 * (pad[1:] + pad[:-1]) / dp


@dataclasses.dataclass
class DiagnosticStateHybrid:
  vorticity: np.ndarray
  divergence: np.ndarray
  temperature_variation: np.ndarray
  cos_lat_u: tuple
  mass_flux_explicit: np.ndarray
  mass_flux_full: np.ndarray
  cos_lat_grad_log_sp: tuple
  u_dot_grad_log_sp: np.ndarray
  tracers: dict
  layer_pressure_thickness: np.ndarray


def compute_diagnostic_state(state, grid: sht.Grid, levels: HybridCoordinates):
  """:1536-1602 (levels nondimensional)."""
  to_nodal = grid.to_nodal
  vort = to_nodal(state['vorticity'])
  div = to_nodal(state['divergence'])
  temp = to_nodal(state['temperature_variation'])
  tracers = {k: to_nodal(v) for k, v in state['tracers'].items()}
  cos_lat_u = tuple(to_nodal(c) for c in sht.get_cos_lat_vector(
      state['vorticity'], state['divergence'], grid, clip=False))
  grad = tuple(to_nodal(g) for g in grid.cos_lat_grad(
      state['log_surface_pressure'], clip=False))
  udg = sum(x * y * grid.sec2_lat for x, y in zip(cos_lat_u, grad))
  ps = np.exp(to_nodal(state['log_surface_pressure']))[0]
  dp = levels.layer_thickness(ps)
  db = levels.sigma_thickness[:, None, None]
  d_full = dp * div + db * ps * udg
  d_explicit = db * ps * udg

  def mass_flux(d):
    cum = np.concatenate([np.zeros_like(d[:1]), np.cumsum(d, axis=0)], axis=0)
    return -cum + levels.b_boundaries[:, None, None] * d.sum(0, keepdims=True)

  return DiagnosticStateHybrid(vort, div, temp, cos_lat_u, mass_flux(d_explicit),
                               mass_flux(d_full), grad, udg, tracers, dp)


@dataclasses.dataclass
class PrimitiveEquationsHybrid(dycore.PrimitiveEquationsSigma):
  """FP64 oracle of PrimitiveEquationsHybrid (:1961-2533).

  ``vertical`` holds a_boundaries in hPa (``hpa`` pascals each) and the
  reference surface pressure is in pascals, both nondimensionalised here.
  """

  reference_surface_pressure: float = 101325.0
  hpa: float = 100.0

  def __post_init__(self):
    self.p_s_ref = dycore.nondim_pressure(self.reference_surface_pressure)
    self.levels = HybridCoordinates(
        dycore.nondim_pressure(np.asarray(self.vertical.a_boundaries) * self.hpa),
        np.asarray(self.vertical.b_boundaries, np.float64))

  def _vtend(self, w, x, dp):
    return hybrid_vertical_advection(w, x, dp)

  def _t_omega_over_p(self, temperature_field, g_term, v_dot_grad_ln_p, ps):
    """:2032-2056 (alpha at p_s_ref)."""
    dp = self.levels.layer_thickness(ps)
    f = np.cumsum(g_term * dp, axis=0)
    alpha, _ = vertical_coeffs(self.levels, self.p_s_ref)
    af = alpha[:, None, None] * f
    af_shift = np.concatenate([np.zeros_like(af[:1]), af[:-1]], axis=0)
    return temperature_field * (v_dot_grad_ln_p - (af + af_shift) / dp)

  def curl_and_div_tendencies(self, aux, ps):
    """:2058-2122."""
    sec2 = self.grid.sec2_lat
    u, v = aux.cos_lat_u
    total_vorticity = aux.vorticity + self.coriolis_parameter
    dp = aux.layer_pressure_thickness
    if self.include_vertical_advection:
      sdu = -self._vtend(aux.mass_flux_full, u, dp)
      sdv = -self._vtend(aux.mass_flux_full, v, dp)
    else:
      sdu = sdv = 0
    pgf = pgf_coefficient(aux.temperature_variation + self.T_ref, ps,
                          self.levels, self.physics_specs.R)
    pgf = pgf * self._virtual_temperature_adjustment(aux)
    pgf = pgf - pgf_coefficient(np.asarray(self.reference_temperature, np.float64),
                                self.p_s_ref, self.levels,
                                self.physics_specs.R)[:, None, None]
    gx, gy = aux.cos_lat_grad_log_sp
    cu = self.grid.to_modal(-v * total_vorticity * sec2 + (sdu + pgf * gx) * sec2)
    cv = self.grid.to_modal(u * total_vorticity * sec2 + (sdv + pgf * gy) * sec2)
    return (-self.grid.curl_cos_lat((cu, cv), clip=False),
            -self.grid.div_cos_lat((cu, cv), clip=False))

  def nodal_temperature_vertical_tendency(self, aux):
    """:2124-2144."""
    dp = aux.layer_pressure_thickness
    tendency = (self._vtend(aux.mass_flux_full, aux.temperature_variation, dp)
                if self.include_vertical_advection else 0)
    if np.unique(self.T_ref.ravel()).size > 1:
      tendency = tendency + self._vtend(aux.mass_flux_explicit, self.T_ref, dp)
    return tendency

  def nodal_temperature_adiabatic_tendency(self, aux, ps):
    """:2146-2224."""
    levels = self.levels
    alpha, log_ratio = vertical_coeffs(levels, ps)
    b_minus = levels.b_boundaries[:-1, None, None]
    db = np.diff(levels.b_boundaries)[:, None, None]
    weight = log_ratio * b_minus + alpha * db
    dp = np.maximum(levels.layer_thickness(ps), 1e-6 * ps)
    scaled = aux.u_dot_grad_log_sp * ps * weight / dp
    dp_k = levels.layer_thickness(ps)
    g = aux.divergence + (aux.u_dot_grad_log_sp * ps
                          * levels.sigma_thickness[:, None, None] / dp_k)
    g_explicit = g - aux.divergence
    mean_part = self._t_omega_over_p(self.T_ref, g_explicit, scaled, ps)
    p = self.physics_specs
    if self.humidity_key is None:
      var_part = self._t_omega_over_p(aux.temperature_variation, g, scaled, ps)
      return p.kappa * (mean_part + var_part)
    ratio, hc = p.R_vapor / p.R, p.Cp_vapor / p.Cp
    q = aux.tracers[self.humidity_key]
    var = aux.temperature_variation * ((1 + (ratio - 1) * q) / (1 + (hc - 1) * q))
    ref = self.T_ref * (((ratio - hc) * q) / (1 + (hc - 1) * q))
    return p.kappa * (mean_part + self._t_omega_over_p(var + ref, g, scaled, ps))

  def nodal_log_pressure_tendency(self, aux, ps):
    """:2226-2247."""
    da = self.levels.pressure_thickness[:, None, None]
    db = self.levels.sigma_thickness[:, None, None]
    div_a = np.sum(aux.divergence * da * (1 / ps - 1 / self.p_s_ref), axis=0)
    udg_b = np.sum(aux.u_dot_grad_log_sp * db, axis=0)
    return -(div_a + udg_b)

  def explicit_terms(self, state):
    """:2249-2360 (the humidity corrections are zero on hybrid levels,
    :2488-2531)."""
    aux = compute_diagnostic_state(state, self.grid, self.levels)
    ps = np.exp(self.grid.to_nodal(state['log_surface_pressure']))[0]
    vort_dot, div_dot = self.curl_and_div_tendencies(aux, ps)
    ke = self.kinetic_energy_tendency(aux)
    orog = self.orography_tendency()
    R = self.physics_specs.R
    temperature = self.T_ref + aux.temperature_variation
    phi_full = geopotential_diff_sparse(
        temperature * self._virtual_temperature_adjustment(aux), self.levels, R, ps)
    phi_lin = dycore._vertical_matvec(
        geopotential_weights(self.levels, R, self.p_s_ref), aux.temperature_variation)
    residual = -self.grid.laplacian(self.grid.to_modal(phi_full - phi_lin))
    dT_h_nodal, dT_h_modal = self.horizontal_scalar_advection(
        aux.temperature_variation, aux)
    tracer_terms = {k: self.horizontal_scalar_advection(v, aux)
                    for k, v in aux.tracers.items()}
    dT_v = self.nodal_temperature_vertical_tendency(aux)
    dT_a = self.nodal_temperature_adiabatic_tendency(aux, ps)
    lsp = self.nodal_log_pressure_tendency(aux, ps)
    dp = aux.layer_pressure_thickness
    if self.include_vertical_advection:
      vert = lambda x: self._vtend(aux.mass_flux_full, x, dp)
    else:
      vert = lambda x: 0
    to_modal = self.grid.to_modal
    tendency = dycore.make_state(
        vorticity=vort_dot,
        divergence=div_dot + ke + orog + residual,
        temperature_variation=to_modal(dT_h_nodal + dT_v + dT_a) + dT_h_modal,
        log_surface_pressure=to_modal(lsp)[None],
        tracers={k: to_modal(vert(aux.tracers[k]) + nm[0]) + nm[1]
                 for k, nm in tracer_terms.items()})
    return dycore.tree_map(self.grid.clip_wavenumbers, tendency)

  def implicit_terms(self, state):
    """:2362-2416 (dense vertical matmuls)."""
    p = self.physics_specs
    g = geopotential_weights(self.levels, p.R, self.p_s_ref)
    pgf = pgf_coefficient(np.asarray(self.reference_temperature, np.float64),
                          self.p_s_ref, self.levels, p.R)
    h = temperature_implicit_weights(self.levels, self.reference_temperature,
                                     p.kappa, self.p_s_ref)
    thick = self.levels.pressure_thickness / self.p_s_ref + self.levels.sigma_thickness
    return dycore.make_state(
        vorticity=np.zeros_like(state['vorticity']),
        divergence=-self.grid.laplacian(
            dycore._vertical_matvec(g, state['temperature_variation'])
            + pgf[:, None, None] * state['log_surface_pressure']),
        temperature_variation=dycore._vertical_matvec(-h, state['divergence']),
        log_surface_pressure=-dycore._vertical_matvec(thick[None],
                                                      state['divergence']),
        tracers={k: np.zeros_like(v) for k, v in state['tracers'].items()})

  @functools.lru_cache(maxsize=16)
  def implicit_inverse_matrix(self, step_size: float):
    """:2418-2438."""
    p = self.physics_specs
    mat = implicit_term_matrix(step_size, self.grid, self.levels,
                               self.reference_temperature, p.kappa, p.R,
                               self.p_s_ref)
    inverse = np.linalg.inv(mat)
    assert not np.isnan(inverse).any()
    return inverse

  def __hash__(self):
    return id(self)
