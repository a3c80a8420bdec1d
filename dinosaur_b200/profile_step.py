"""Runs a few filtered SIL3 steps of the primitive equations for profiling.

    python -m dinosaur_b200.profile_step --grid T42 --layers 24 --members 16 \
        --held-suarez --steps 3

Seeded small random states; eager launches (no CUDA graph) so that a kernel
profiler sees every launch.  Prints the mean step time.
"""

from __future__ import annotations

import argparse

import numpy as np
import torch

from dinosaur_b200 import coordinate_systems, held_suarez, hybrid_coordinates
from dinosaur_b200 import primitive_equations as pe
from dinosaur_b200 import sigma_coordinates, spherical_harmonic as sh
from dinosaur_b200 import time_integration as ti, units


def main():
  ap = argparse.ArgumentParser()
  ap.add_argument('--grid', default='T42')
  ap.add_argument('--layers', type=int, default=24)
  ap.add_argument('--members', type=int, default=1)
  ap.add_argument('--held-suarez', action='store_true')
  ap.add_argument('--moist', action='store_true',
                  help='specific humidity and two passive tracers')
  ap.add_argument('--precision', default='fp32', choices=['fp32', 'bf16x3', 'tf32x3'])
  ap.add_argument('--hybrid', action='store_true',
                  help='analytic hybrid sigma-pressure levels (PrimitiveEquationsHybrid)')
  ap.add_argument('--steps', type=int, default=3)
  ap.add_argument('--dt-minutes', type=float, default=15.0)
  args = ap.parse_args()
  impl = lambda **kw: sh.CudaSphericalHarmonics(precision=args.precision, **kw)
  g = getattr(sh.Grid, args.grid)(spherical_harmonics_impl=impl)
  vert = (hybrid_coordinates.HybridCoordinates.analytic_levels(args.layers) if args.hybrid
          else sigma_coordinates.SigmaCoordinates.equidistant(args.layers))
  coords = coordinate_systems.CoordinateSystem(g, vert)
  ps = units.SimUnits()
  tref = np.full(args.layers, 285.0) if args.held_suarez else np.linspace(
      220.0, 288.0, args.layers)
  eq_cls = pe.PrimitiveEquationsHybrid if args.hybrid else pe.PrimitiveEquationsSigma
  eq = eq_cls(
      tref, np.zeros(g.modal_shape, np.float32), coords, ps,
      humidity_key='specific_humidity' if args.moist else None)
  if args.held_suarez:
    eq = ti.compose_equations(
        [eq, held_suarez.HeldSuarezForcingSigma(coords, ps, tref)])
  dt = units.nondim_time(args.dt_minutes * 60.0)
  step = ti.step_with_filters(ti.imex_rk_sil3(eq, dt),
                              [ti.exponential_step_filter(g, dt)])
  rng = np.random.default_rng(0)
  lead = (args.members,) if args.members > 1 else ()
  _, l = g.modal_mesh
  scale = g.mask / (l + 1.0) ** 2
  t = lambda shp: torch.as_tensor(
      (1e-4 * rng.standard_normal(shp) * scale).astype(np.float32), device='cuda')
  shape = lead + (args.layers,) + g.modal_shape
  tracers = {}
  if args.moist:
    const = np.zeros(shape, np.float32)
    const[..., 0, 0] = 2.0 * np.sqrt(np.pi)  # the constant field 1
    dev = lambda a: torch.as_tensor(a, device='cuda')
    tracers = {'specific_humidity': dev(5e-3 * const) + 1e-2 * t(shape),
               'tracer_a': dev(const) + t(shape), 'tracer_b': dev(const) + t(shape)}
  lnps = t(lead + (1,) + g.modal_shape)
  if args.hybrid:
    # A physical surface pressure (1e5 Pa) as the l = 0 term.
    lnps[..., 0, 0] += float(np.log(units.nondim_pressure(1e5)) * 2.0 * np.sqrt(np.pi))
  state = pe.State(t(shape), t(shape), t(shape), lnps, tracers=tracers)
  eng = eq.engine(state)
  buf = eng.pack(state)
  eng.step_(buf, dt, step.filter_scaling, 1, graph=False)
  torch.cuda.synchronize()
  e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
  e0.record()
  eng.step_(buf, dt, step.filter_scaling, args.steps, graph=False)
  e1.record()
  torch.cuda.synchronize()
  print(f'{args.grid} K={args.layers} members={args.members} '
        f'hs={args.held_suarez} moist={args.moist} hybrid={args.hybrid} '
        f'{args.precision}: '
        f'{e0.elapsed_time(e1) / args.steps * 1e3:.1f} us/step, '
        f'finite={bool(torch.isfinite(buf).all())}')


if __name__ == '__main__':
  main()
