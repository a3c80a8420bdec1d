"""Shared cases for the GPU parity tests: matched oracle / CUDA set-ups.

Every case feeds both sides the same FP32-rounded FP64 state.
"""

import numpy as np
import torch

from oracle import dycore as od
from oracle import sht as osht
from oracle import states as ost

from dinosaur_b200 import coordinate_systems
from dinosaur_b200 import primitive_equations as pe
from dinosaur_b200 import sigma_coordinates
from dinosaur_b200 import spherical_harmonic as sh
from dinosaur_b200 import units

KEYS = ('vorticity', 'divergence', 'temperature_variation',
        'log_surface_pressure')


def to_state(d, members_axis=False):
  t = lambda x: torch.as_tensor(np.asarray(x), device='cuda',
                                dtype=torch.float32)
  return pe.State(*[t(d[k]) for k in KEYS],
                  tracers={k: t(v) for k, v in d['tracers'].items()})


def rel(a, b):
  a = a.detach().double().cpu().numpy() if torch.is_tensor(a) else np.asarray(a)
  b = np.asarray(b, np.float64)
  return np.abs(a - b).max() / max(np.abs(b).max(), 1e-30)


def assert_state(got, ref, tol, keys=KEYS):
  for k in keys:
    e = rel(getattr(got, k), ref[k])
    assert e < tol, (k, e)
  for name in ref['tracers']:
    e = rel(got.tracers[name], ref['tracers'][name])
    assert e < tol, (name, e)


def make(grid_name='T21', layers=6, amplitude=1.0, tracers=None,
         humidity=None, perturb=True):
  og = getattr(osht.Grid, grid_name)()
  st, tref, orog, vert = ost.baroclinic_config(og, layers, seed=0,
                                               amplitude=amplitude)
  if tracers:
    st['tracers'] = dict(tracers(og, layers))
  if perturb:
    # Smooth seeded perturbations so that no tendency is identically zero
    # (the balanced JW state has a vanishing vorticity tendency).
    rng = np.random.default_rng(7)
    _, l = og.modal_mesh
    noise = lambda n: rng.standard_normal((n,) + og.modal_shape) * og.mask / (
        l + 1.0) ** 2
    st['vorticity'] = st['vorticity'] + 1e-3 * noise(layers)
    st['divergence'] = st['divergence'] + 1e-3 * noise(layers)
    st['log_surface_pressure'] = st['log_surface_pressure'] + 1e-3 * noise(1)
  oeq = od.PrimitiveEquationsSigma(tref, orog, og, vert, od.SimUnits(),
                                   humidity_key=humidity)
  g = getattr(sh.Grid, grid_name)()
  coords = coordinate_systems.CoordinateSystem(
      g, sigma_coordinates.SigmaCoordinates.equidistant(layers))
  eq = pe.PrimitiveEquationsSigma(tref, orog.astype(np.float32), coords,
                                  units.SimUnits(), humidity_key=humidity)
  # Feed both sides the same FP32-rounded state.
  st = od.tree_map(lambda x: np.asarray(x, np.float32).astype(np.float64), st)
  return og, oeq, st, g, eq


def tracers(og, layers):
  q = ost.gaussian_scalar(og, layers, amplitude=5e-3, perturbation_radius=0.3)
  q = q + og.to_modal(np.full((layers,) + og.nodal_shape, 5e-3))
  a = ost.gaussian_scalar(og, layers, amplitude=2.0, lon_location=2.0)
  return [('specific_humidity', q), ('tracer_a', a)]


