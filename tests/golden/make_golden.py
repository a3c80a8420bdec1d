"""Generates the golden fixtures in this directory from the reference itself.

Run where neuralgcm/dinosaur 1.3.6 is checked out, naming its root as the
argument or in the ``DINOSAUR_REFERENCE_ROOT`` environment variable::

    python tests/golden/make_golden.py REFERENCE_ROOT

``jax``, ``tree_math`` and ``pint`` are not installed there, so
``_standins.py`` provides NumPy stand-ins; the reference modules then run
eagerly in float64.  Every array written here is an output of the
reference's own functions on seeded inputs; the inputs are stored beside them.
The fixtures pin the FP64 oracle (``oracle/``) in ``tests/test_oracle_golden.py``.
"""

from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import _standins  # noqa: E402


def _save(name, **arrays):
  path = os.path.join(HERE, name)
  np.savez_compressed(path, **{k: np.asarray(v) for k, v in arrays.items()})
  size = os.path.getsize(path)
  print(f'wrote {name} ({size / 1024:.1f} KiB)')


def main(reference_root=None):
  reference_root = reference_root or os.environ.get('DINOSAUR_REFERENCE_ROOT')
  if not reference_root:
    raise SystemExit('usage: make_golden.py REFERENCE_ROOT '
                     '(or set DINOSAUR_REFERENCE_ROOT)')
  _standins.install(reference_root)
  from dinosaur import associated_legendre
  from dinosaur import coordinate_systems
  from dinosaur import filtering
  from dinosaur import fourier
  from dinosaur import held_suarez
  from dinosaur import hybrid_coordinates
  from dinosaur import primitive_equations
  from dinosaur import primitive_equations_states
  from dinosaur import sigma_coordinates
  from dinosaur import spherical_harmonic
  from dinosaur import time_integration
  from dinosaur import units

  rng = np.random.default_rng(1234)

  # -- basis ------------------------------------------------------------
  x, w = associated_legendre.gauss_legendre_nodes(32)
  p = associated_legendre.evaluate(n_m=22, n_l=23, x=x)
  xe, we = associated_legendre.equiangular_nodes(13)
  f = fourier.real_basis(22, 64)
  u = rng.standard_normal((3, 43))
  du = fourier.real_basis_derivative(u, axis=-1)
  _save('basis.npz', gauss_x=x, gauss_w=w, legendre_T21=p, equi_x=xe,
        equi_w=we, fourier_T21=f, deriv_in=u, deriv_out=du)

  # -- SHT and spectral operators --------------------------------------
  for name, grid in [('T21', spherical_harmonic.Grid.T21()),
                     ('TL31', spherical_harmonic.Grid.TL31()),
                     ('W16', spherical_harmonic.Grid.with_wavenumbers(16))]:
    _, l = grid.modal_mesh
    modal = rng.standard_normal((2,) + grid.modal_shape) * grid.mask / (
        l + 1.0) ** 2
    nodal = rng.standard_normal((2,) + grid.nodal_shape)
    vort = rng.standard_normal(grid.modal_shape) * grid.mask / (l + 1.0) ** 2
    div = rng.standard_normal(grid.modal_shape) * grid.mask / (l + 1.0) ** 2
    uc, vc = spherical_harmonic.get_cos_lat_vector(vort, div, grid, clip=False)
    uc2, vc2 = spherical_harmonic.get_cos_lat_vector(vort, div, grid)
    un, vn = spherical_harmonic.vor_div_to_uv_nodal(grid, vort, div)
    _save(f'sht_{name}.npz',
          modal_in=modal, nodal_out=grid.to_nodal(modal),
          nodal_in=nodal, modal_out=grid.to_modal(nodal),
          d_dlon=grid.d_dlon(modal),
          cos_lat_d_dlat=grid.cos_lat_d_dlat(modal),
          sec_lat_d_dlat_cos2=grid.sec_lat_d_dlat_cos2(modal),
          laplacian=grid.laplacian(modal),
          inverse_laplacian=grid.inverse_laplacian(modal),
          clip=grid.clip_wavenumbers(modal),
          div_cos_lat=grid.div_cos_lat((modal[0], modal[1])),
          curl_cos_lat=grid.curl_cos_lat((modal[0], modal[1]), clip=False),
          vort=vort, div=div, u_cos=uc, v_cos=vc, u_cos_clip=uc2,
          v_cos_clip=vc2, u_nodal=un, v_nodal=vn,
          integrate=grid.integrate(nodal),
          filter_default=filtering.exponential_filter(grid)(np.ones(
              grid.modal_shape)),
          filter_hs=filtering.exponential_filter(
              grid, attenuation=0.131256 / 0.0087504, order=1.5,
              cutoff=0.8)(np.ones(grid.modal_shape)))

  # -- sigma coordinates -------------------------------------------------
  sig = sigma_coordinates.SigmaCoordinates.equidistant(6)
  xs = rng.standard_normal((6, 5, 4))
  ws = rng.standard_normal((5, 5, 4))
  _save('sigma.npz', x=xs, w=ws,
        cumulative=sigma_coordinates.cumulative_sigma_integral(xs, sig),
        cumulative_up=sigma_coordinates.cumulative_sigma_integral(
            xs, sig, downward=False),
        integral=sigma_coordinates.sigma_integral(xs, sig),
        advection=sigma_coordinates.centered_vertical_advection(ws, xs, sig),
        centers=sig.centers, thickness=sig.layer_thickness)

  # -- primitive equations ----------------------------------------------
  physics_specs = units.SimUnits.from_si()
  layers = 6
  coords = coordinate_systems.CoordinateSystem(
      horizontal=spherical_harmonic.Grid.T21(),
      vertical=sigma_coordinates.SigmaCoordinates.equidistant(layers))
  grid = coords.horizontal
  init_fn, aux = primitive_equations_states.steady_state_jw(
      coords, physics_specs)
  state = init_fn()
  ref_temps = aux['ref_temperatures']
  orography = primitive_equations.truncated_modal_orography(
      aux['orography'], coords)
  bump = primitive_equations_states.gaussian_scalar(
      coords, physics_specs, lon_location=1.0, lat_location=0.3,
      perturbation_radius=0.1, amplitude=1.0)
  _, l = grid.modal_mesh
  noise = rng.standard_normal((layers,) + grid.modal_shape) * grid.mask / (
      l + 1.0) ** 2
  state = primitive_equations.State(
      vorticity=np.asarray(state.vorticity) + 1e-3 * noise,
      divergence=np.asarray(state.divergence) + 1e-3 * noise[::-1],
      temperature_variation=np.asarray(state.temperature_variation) + bump,
      log_surface_pressure=np.asarray(state.log_surface_pressure)
      + 1e-3 * noise[:1])
  eq = primitive_equations.PrimitiveEquationsSigma(
      ref_temps, orography, coords, physics_specs)
  expl = eq.explicit_terms(state)
  impl = eq.implicit_terms(state)
  inv = eq.implicit_inverse(state, 0.05)
  dt = 0.175008
  step = time_integration.step_with_filters(
      time_integration.imex_rk_sil3(eq, dt),
      [time_integration.exponential_step_filter(grid, dt)])
  s1 = step(state)
  s2 = step(s1)

  def pack(prefix, s):
    return {f'{prefix}_{k}': np.asarray(getattr(s, k)) for k in
            ('vorticity', 'divergence', 'temperature_variation',
             'log_surface_pressure')}

  jw_state, _ = primitive_equations_states.steady_state_jw(
      coords, physics_specs)
  jw = jw_state()
  _save('pe_T21_L6.npz', ref_temps=ref_temps, orography=orography,
        orography_nodal=aux['orography'], bump=bump,
        jw_vorticity=jw.vorticity, jw_temperature=jw.temperature_variation,
        jw_log_ps=jw.log_surface_pressure,
        **pack('in', state), **pack('explicit', expl),
        **pack('implicit', impl), **pack('inverse', inv),
        **pack('step1', s1), **pack('step2', s2))

  # -- hybrid level constructors (hybrid_coordinates.py:268-471) ----------
  lv_a = hybrid_coordinates.HybridCoordinates.analytic_levels(17)
  lv_e = hybrid_coordinates.HybridCoordinates.analytic_ecmwf_like(20)
  lv_s = hybrid_coordinates.HybridCoordinates.from_sigma_levels(
      sigma_coordinates.SigmaCoordinates.equidistant(8))
  lv_c = hybrid_coordinates.HybridCoordinates.from_coefficients(
      [0.0, 0.1, 0.05, 0.0], [0.0, 0.2, 0.6, 1.0], p0=1013.25)
  _save('hybrid_levels.npz',
        analytic_a=lv_a.a_boundaries, analytic_b=lv_a.b_boundaries,
        ecmwf_like_a=lv_e.a_boundaries, ecmwf_like_b=lv_e.b_boundaries,
        sigma_a=lv_s.a_boundaries, sigma_b=lv_s.b_boundaries,
        coeffs_a=lv_c.a_boundaries, coeffs_b=lv_c.b_boundaries,
        analytic_thickness_at_900=np.asarray(lv_a.layer_thickness(900.0)),
        analytic_centers_at_900=np.asarray(lv_a.pressure_centers(900.0)))

  # -- hybrid sigma-pressure levels (primitive_equations.py:1961-2533) -----
  # The same input state on 6 analytic hybrid levels (a in hPa).
  hyb_levels = hybrid_coordinates.HybridCoordinates.analytic_levels(layers)
  hyb_coords = coordinate_systems.CoordinateSystem(horizontal=grid,
                                                   vertical=hyb_levels)
  hyb_eq = primitive_equations.PrimitiveEquationsHybrid(
      ref_temps, orography, hyb_coords, physics_specs)
  hyb_step = time_integration.step_with_filters(
      time_integration.imex_rk_sil3(hyb_eq, dt),
      [time_integration.exponential_step_filter(grid, dt)])
  _save('pe_hybrid_T21_L6.npz',
        a_boundaries=hyb_levels.a_boundaries, b_boundaries=hyb_levels.b_boundaries,
        **pack('explicit', hyb_eq.explicit_terms(state)),
        **pack('implicit', hyb_eq.implicit_terms(state)),
        **pack('inverse', hyb_eq.implicit_inverse(state, 0.05)),
        **pack('step1', hyb_step(state)))
  # The same state on 6 ECMWF-like levels: the top two layers are pure
  # pressure (b = 0 at both of their boundaries).
  ecm_levels = hybrid_coordinates.HybridCoordinates.analytic_ecmwf_like(layers)
  ecm_eq = primitive_equations.PrimitiveEquationsHybrid(
      ref_temps, orography,
      coordinate_systems.CoordinateSystem(horizontal=grid, vertical=ecm_levels),
      physics_specs)
  ecm_step = time_integration.step_with_filters(
      time_integration.imex_rk_sil3(ecm_eq, dt),
      [time_integration.exponential_step_filter(grid, dt)])
  _save('pe_hybrid_ecmwf_like_T21_L6.npz',
        a_boundaries=ecm_levels.a_boundaries, b_boundaries=ecm_levels.b_boundaries,
        **pack('explicit', ecm_eq.explicit_terms(state)),
        **pack('implicit', ecm_eq.implicit_terms(state)),
        **pack('inverse', ecm_eq.implicit_inverse(state, 0.05)),
        **pack('step1', ecm_step(state)))

  # -- digital filter initialisation (time_integration.py:645-712) ---------
  dfi_dt = dt
  dfi = time_integration.digital_filter_initialization(
      eq, time_integration.imex_rk_sil3,
      [time_integration.exponential_step_filter(grid, dfi_dt)],
      time_span=8 * dfi_dt, cutoff_period=8 * dfi_dt, dt=dfi_dt)
  dfi_out = dfi(state)
  reversed_eq = time_integration.TimeReversedImExODE(eq)
  rev_step = time_integration.imex_rk_sil3(reversed_eq, dfi_dt)
  _save('dfi_T21_L6.npz', dt=dfi_dt,
        weights=time_integration._dfi_lanczos_weights(8 * dfi_dt, 8 * dfi_dt, dfi_dt),
        **pack('dfi', dfi_out), **pack('reversed_step', rev_step(state)))

  # -- moist primitive equations with a passive tracer -------------------
  q = 5e-3 * (1 + 0.2 * bump / np.abs(bump).max())
  q_modal = np.asarray(q)
  tracer = np.asarray(primitive_equations_states.gaussian_scalar(
      coords, physics_specs, amplitude=2.0))
  moist_state = primitive_equations.State(
      vorticity=state.vorticity, divergence=state.divergence,
      temperature_variation=state.temperature_variation,
      log_surface_pressure=state.log_surface_pressure,
      tracers={'specific_humidity': q_modal, 'tracer': tracer})
  eq_moist = primitive_equations.PrimitiveEquationsSigma(
      ref_temps, orography, coords, physics_specs,
      humidity_key='specific_humidity')
  expl_m = eq_moist.explicit_terms(moist_state)
  _save('pe_moist_T21_L6.npz', humidity=q_modal, tracer=tracer,
        **pack('explicit', expl_m),
        explicit_humidity=expl_m.tracers['specific_humidity'],
        explicit_tracer=expl_m.tracers['tracer'])
  # the same moist state on the 6 analytic hybrid levels
  hyb_eq_moist = primitive_equations.PrimitiveEquationsHybrid(
      ref_temps, orography, hyb_coords, physics_specs,
      humidity_key='specific_humidity')
  expl_hm = hyb_eq_moist.explicit_terms(moist_state)
  _save('pe_hybrid_moist_T21_L6.npz', **pack('explicit', expl_hm),
        explicit_humidity=expl_hm.tracers['specific_humidity'],
        explicit_tracer=expl_hm.tracers['tracer'])

  # -- Held-Suarez forcing composed with the primitive equations ---------
  hs_coords = coordinate_systems.CoordinateSystem(
      horizontal=spherical_harmonic.Grid.T21(),
      vertical=sigma_coordinates.SigmaCoordinates.equidistant(layers))
  hs_ref = np.full((layers,), 285.0)
  nodal_noise = 0.1 * rng.standard_normal((layers,) + grid.nodal_shape)
  log_ps = grid.to_modal(np.log(
      physics_specs.nondimensionalize(1e5 * _standins.pint.UnitRegistry().Pa)
      * np.ones((1,) + grid.nodal_shape)))
  hs_state = primitive_equations.State(
      vorticity=np.zeros((layers,) + grid.modal_shape),
      divergence=np.zeros((layers,) + grid.modal_shape),
      temperature_variation=grid.to_modal(nodal_noise),
      log_surface_pressure=log_ps)
  hs_state = primitive_equations.State(
      vorticity=hs_state.vorticity + 1e-4 * noise,
      divergence=hs_state.divergence + 1e-4 * noise[::-1],
      temperature_variation=hs_state.temperature_variation,
      log_surface_pressure=hs_state.log_surface_pressure)
  hs = held_suarez.HeldSuarezForcingSigma(hs_coords, physics_specs, hs_ref)
  hs_expl = hs.explicit_terms(hs_state)
  pe_hs = primitive_equations.PrimitiveEquationsSigma(
      hs_ref, np.zeros(grid.modal_shape), hs_coords, physics_specs)
  composed = time_integration.compose_equations([pe_hs, hs])
  hs_dt = 0.131256
  hs_step = time_integration.step_with_filters(
      time_integration.imex_rk_sil3(composed, hs_dt),
      [time_integration.exponential_step_filter(
          grid, hs_dt, tau=0.0087504, order=1.5, cutoff=0.8)])
  hs1 = hs_step(hs_state)
  _save('hs_T21_L6.npz', **pack('in', hs_state), **pack('forcing', hs_expl),
        **pack('step1', hs1))

  # -- shallow water (two layers) --------------------------------------
  from dinosaur import layer_coordinates
  from dinosaur import shallow_water
  from dinosaur import shallow_water_states
  swe_coords = coordinate_systems.CoordinateSystem(
      spherical_harmonic.Grid.T21(), layer_coordinates.LayerCoordinates(2))
  swe_grid = swe_coords.horizontal
  _, l = swe_grid.modal_mesh
  smooth = lambda n, a: a * rng.standard_normal((n,) + swe_grid.modal_shape) * (
      swe_grid.mask / (l + 1.0) ** 2)
  densities = np.array([0.9, 1.0])
  ref_potential = np.array([0.1, 0.12])
  swe_orog = smooth(1, 1e-3)[0]
  lat = np.arccos(swe_grid.cos_lat)
  u_layers = np.stack([np.cos(lat) / 5, np.cos(lat) ** 2 / 6])
  steady = shallow_water_states.multi_layer(u_layers, densities, swe_coords)
  swe_state = shallow_water.State(
      vorticity=np.asarray(steady.vorticity) + smooth(2, 1e-2),
      divergence=np.asarray(steady.divergence) + smooth(2, 1e-2),
      potential=np.asarray(steady.potential) + smooth(2, 1e-2))
  swe_eq = shallow_water.ShallowWaterEquations(
      swe_coords, physics_specs, swe_orog, ref_potential, densities=densities)
  swe_dt = 1e-3 * 20
  swe_step = time_integration.step_with_filters(
      time_integration.imex_rk_sil3(swe_eq, swe_dt),
      [time_integration.exponential_step_filter(swe_grid, swe_dt)])
  w1 = swe_step(swe_state)
  w2 = swe_step(w1)

  def swe_pack(prefix, st):
    return {f'{prefix}_{k}': np.asarray(getattr(st, k)) for k in
            ('vorticity', 'divergence', 'potential')}

  _save('swe_T21_L2.npz', densities=densities, ref_potential=ref_potential,
        orography=swe_orog, u_layers=u_layers, dt=swe_dt,
        **swe_pack('steady', steady), **swe_pack('in', swe_state),
        **swe_pack('explicit', swe_eq.explicit_terms(swe_state)),
        **swe_pack('implicit', swe_eq.implicit_terms(swe_state)),
        **swe_pack('inverse', swe_eq.implicit_inverse(swe_state, 0.03)),
        **swe_pack('step1', w1), **swe_pack('step2', w2))

  # -- Fast (m-stacked, zero imaginary m = 0 row) layout ----------------
  fast = spherical_harmonic.Grid.T21(
      spherical_harmonics_impl=spherical_harmonic.FastSphericalHarmonics)
  fx = rng.standard_normal((3,) + fast.modal_shape) * fast.mask
  fz = rng.standard_normal((3,) + fast.nodal_shape)
  _save('fast_T21.npz', modal_axes_m=fast.modal_axes[0],
        modal_axes_l=fast.modal_axes[1], mask=fast.mask, modal_in=fx,
        nodal_out=fast.to_nodal(fx), nodal_in=fz, modal_out=fast.to_modal(fz),
        d_dlon=fast.d_dlon(fx), laplacian=fast.laplacian(fx),
        cos_lat_d_dlat=fast.cos_lat_d_dlat(fx),
        sec_lat_d_dlat_cos2=fast.sec_lat_d_dlat_cos2(fx),
        clip=fast.clip_wavenumbers(fx))

  # -- nondimensional constants ----------------------------------------
  _save('units.npz', radius=physics_specs.radius,
        angular_velocity=physics_specs.angular_velocity,
        g=physics_specs.g, R=physics_specs.R, R_vapor=physics_specs.R_vapor,
        Cp_vapor=physics_specs.Cp_vapor, kappa=physics_specs.kappa,
        kf=hs.kf, ka=hs.ka, ks=hs.ks, p0=hs.p0)


if __name__ == '__main__':
  main(*sys.argv[1:])
