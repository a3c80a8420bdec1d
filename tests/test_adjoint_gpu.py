"""Reverse mode on the GPU against central differences of the FP64 oracle.

Every GPU gradient goes through the hand-written VJP entry points of the C ABI
(dino_pe_explicit_vjp, dino_pe_step_vjp, dino_pe_implicit_vjp,
dino_pe_implicit_inverse_vjp) via the torch.autograd wrappers.  Tolerances:

* dot tests <J^T w, v> against <w, J v>, with J v from central differences
  of the FP64 oracle (eps = 1e-6): relative error <= 1e-4;
* implicit_terms / implicit_inverse VJPs against the GPU forward maps
  (exact transposes): <= 1e-5;
* the gradient of a 24-step T42 / 20-level rollout's tracking loss along 8
  unit-norm masked random directions (seed 2): against the FP64 oracle's
  central differences (eps = 1e-3) of the final state contracted with the
  FP32 residual, <= 1e-4; against the FP64 loss's own central differences,
  <= 5e-3 (the FP32 forward's rounding, amplified by the loss residual; see
  the test).
"""

import numpy as np
import pytest
import torch

from oracle import dycore as od
from oracle import sht as osht
from oracle import states as ost

import config_cases
import oracle_fd

pytestmark = pytest.mark.gpu

from dinosaur_b200 import coordinate_systems  # noqa: E402
from dinosaur_b200 import held_suarez  # noqa: E402
from dinosaur_b200 import primitive_equations as pe  # noqa: E402
from dinosaur_b200 import sigma_coordinates  # noqa: E402
from dinosaur_b200 import spherical_harmonic as sh  # noqa: E402
from dinosaur_b200 import time_integration as ti  # noqa: E402
from dinosaur_b200 import units  # noqa: E402

from pe_cases import KEYS, make, to_state, tracers  # noqa: E402


def random_tree(og, like, rng):
  """Masked random modal coefficients with the structure of `like`."""
  _, l = og.modal_mesh
  noise = lambda a: (rng.standard_normal(a.shape) * og.mask / (l + 1.0))
  out = {k: noise(like[k]) for k in KEYS}
  out['tracers'] = {n: noise(a) for n, a in like['tracers'].items()}
  return out


def tree_dot(a, b):
  total = sum(float(np.sum(a[k] * b[k])) for k in KEYS)
  return total + sum(float(np.sum(a['tracers'][n] * b['tracers'][n]))
                     for n in a['tracers'])


def state_leaves(s):
  return [getattr(s, k) for k in KEYS] + [s.tracers[n] for n in s.tracers]


def gpu_vjp(fn, st, w):
  """Gradient of <w, fn(x)> at x = st through the CUDA VJPs."""
  x = to_state(st)
  leaves = state_leaves(x)
  for t in leaves:
    t.requires_grad_(True)
  y = fn(x)
  wt = to_state(w)
  loss = sum((a * b).sum() for a, b in zip(state_leaves(y), state_leaves(wt)))
  grads = torch.autograd.grad(loss, leaves)
  out = {k: g.double().cpu().numpy() for k, g in zip(KEYS, grads)}
  out['tracers'] = {n: g.double().cpu().numpy()
                    for n, g in zip(st['tracers'], grads[len(KEYS):])}
  return out


def central_dot(ofn, st, w, v, eps=1e-6):
  plus = ofn(od.tree_axpy((1.0, st), (eps, v)))
  minus = ofn(od.tree_axpy((1.0, st), (-eps, v)))
  return (tree_dot(w, plus) - tree_dot(w, minus)) / (2 * eps)


def hs_case():
  og = osht.Grid.T21()
  layers = 6
  st, tref, orog, vert = ost.held_suarez_config(og, layers, member=3)
  ops = od.SimUnits()
  ocomp = od.ComposedEquation([
      od.PrimitiveEquationsSigma(tref, orog, og, vert, ops),
      od.HeldSuarezForcingSigma(og, vert, ops, tref)])
  g = sh.Grid.T21()
  coords = coordinate_systems.CoordinateSystem(
      g, sigma_coordinates.SigmaCoordinates.equidistant(layers))
  comp = ti.compose_equations([
      pe.PrimitiveEquationsSigma(tref, orog, coords, units.SimUnits()),
      held_suarez.HeldSuarezForcingSigma(coords, units.SimUnits(), tref)])
  rng = np.random.default_rng(5)
  noise = rng.standard_normal((layers,) + og.modal_shape) * og.mask / 1e3
  st['vorticity'] = st['vorticity'] + noise
  st['divergence'] = st['divergence'] + noise[::-1]
  st = od.tree_map(lambda x: np.asarray(x, np.float32).astype(np.float64), st)
  return og, ocomp, st, g, comp


def explicit_case(kind):
  if kind == 'held_suarez':
    return hs_case()
  if kind == 'moist':
    return make(tracers=tracers, humidity='specific_humidity')
  if kind == 'dry_tracers':
    return make(tracers=tracers)
  return make()


@pytest.mark.parametrize('kind', ['dry', 'dry_tracers', 'moist', 'held_suarez'])
def test_explicit_terms_vjp_dot(kind):
  og, oeq, st, g, eq = explicit_case(kind)
  rng = np.random.default_rng(11)
  w = random_tree(og, st, rng)
  v = random_tree(og, st, rng)
  lhs = tree_dot(gpu_vjp(eq.explicit_terms, st, w), v)
  rhs = central_dot(oeq.explicit_terms, st, w, v)
  assert abs(lhs - rhs) <= 1e-4 * abs(rhs), (lhs, rhs)


def test_implicit_vjps_are_transposes():
  og, oeq, st, g, eq = make()
  rng = np.random.default_rng(12)
  w = random_tree(og, st, rng)
  v = random_tree(og, st, rng)
  vs = to_state(v)
  ws = to_state(w)
  dot = lambda a, b: sum(float((x.double() * y.double()).sum())
                         for x, y in zip(state_leaves(a), state_leaves(b)))
  lhs = tree_dot(gpu_vjp(eq.implicit_terms, st, w), v)
  rhs = dot(ws, eq.implicit_terms(vs))
  assert abs(lhs - rhs) <= 1e-5 * abs(rhs), (lhs, rhs)
  for eta in (0.05, 0.175008 / 3):
    lhs = tree_dot(gpu_vjp(lambda s: eq.implicit_inverse(s, eta), st, w), v)
    rhs = dot(ws, eq.implicit_inverse(vs, eta))
    assert abs(lhs - rhs) <= 1e-5 * abs(rhs), (eta, lhs, rhs)


@pytest.mark.parametrize('kind', ['dry', 'moist', 'held_suarez'])
def test_filtered_step_vjp_dot(kind):
  og, oeq, st, g, eq = explicit_case(kind)
  if kind == 'held_suarez':
    dt = 0.131256
    oflt = od.exponential_step_filter(og, dt, tau=0.0087504, order=1.5,
                                      cutoff=0.8)
    flt = ti.exponential_step_filter(g, dt, tau=0.0087504, order=1.5,
                                     cutoff=0.8)
  else:
    dt = 0.175008
    oflt = od.exponential_step_filter(og, dt)
    flt = ti.exponential_step_filter(g, dt)
  ostep = od.step_with_filters(od.imex_rk_sil3(oeq, dt), [oflt])
  step = ti.step_with_filters(ti.imex_rk_sil3(eq, dt), [flt])
  assert isinstance(step, ti.FusedSIL3Step)
  rng = np.random.default_rng(13)
  w = random_tree(og, st, rng)
  v = random_tree(og, st, rng)
  lhs = tree_dot(gpu_vjp(step, st, w), v)
  rhs = central_dot(ostep, st, w, v)
  assert abs(lhs - rhs) <= 1e-4 * abs(rhs), (lhs, rhs)


def test_rollout_gradient_t42_l20_24_steps():
  """Tracking-loss gradient through 24 filtered SIL3 steps (T42, 20 levels),
  per-step checkpointed, along 8 unit-norm masked random directions.

  The loss mean((T' - T'_t)^2) + mean((zeta - zeta_t)^2) differences two
  states that share the JW background, so its residual is ~1e-3 of the
  fields and the FP32 forward rounding (~1e-6 relative after 24 steps) moves
  the loss gradient by ~1e-3 relative: the gradient of any FP32 evaluation
  of this loss differs from the FP64 loss's by that much.  The adjoint is
  therefore checked against g.v = 2/N sum r . (J v) with the FP32 residual r
  of the GPU forward and J v from FP64 central differences of the final
  state (the gradient an exact adjoint of the FP32 evaluation gives):
  <= 1e-4 max |g.v|.  The gap to the FP64 loss's central difference is
  bounded by the forward's precision: <= 5e-3.
  """
  grid_name, layers, dt, n_steps, eps = 'T42', 20, 0.175008, 24, 1e-3
  og = getattr(osht.Grid, grid_name)()
  rnd32 = lambda t: od.tree_map(
      lambda x: np.asarray(x, np.float32).astype(np.float64), t)
  st0 = rnd32(ost.baroclinic_config(og, layers, seed=0)[0])
  og_, oeq = oracle_fd.dry_setup(grid_name, layers)
  start_t = ost.baroclinic_config(og, layers, seed=1)[0]
  target = rnd32(oracle_fd.rollout(og_, oeq, dt, n_steps, start_t))
  rng = np.random.default_rng(2)
  dirs = []
  for _ in range(8):
    v = random_tree(og, st0, rng)
    norm = np.sqrt(tree_dot(v, v))
    dirs.append(od.tree_map(lambda x, n=norm: x / n, v))
  with config_cases.oracle_pool(8) as pool:
    futs = [pool.submit(oracle_fd.rollout_jvp_fd, grid_name, layers, dt,
                        n_steps, st0, target, v, eps) for v in dirs]
    # GPU gradient while the oracle runs.
    g = sh.Grid.T42()
    coords = coordinate_systems.CoordinateSystem(
        g, sigma_coordinates.SigmaCoordinates.equidistant(layers))
    _, tref, orog, _ = ost.baroclinic_config(og, layers, seed=0)
    eq = pe.PrimitiveEquationsSigma(tref, orog.astype(np.float32), coords,
                                    units.SimUnits())
    step = ti.repeated(ti.step_with_filters(
        ti.imex_rk_sil3(eq, dt), [ti.exponential_step_filter(g, dt)]), n_steps)
    x = to_state(st0)
    leaves = state_leaves(x)
    for t in leaves:
      t.requires_grad_(True)
    final = step(x)
    tgt = to_state(target)
    loss = (((final.temperature_variation.double() -
              tgt.temperature_variation.double()) ** 2).mean() +
            ((final.vorticity.double() - tgt.vorticity.double()) ** 2).mean())
    grads = torch.autograd.grad(loss, leaves)
    gd = {k: t.double().cpu().numpy() for k, t in zip(KEYS, grads)}
    gd['tracers'] = {}
    res = {k: (getattr(final, k).detach().double().cpu().numpy() - target[k])
           for k in ('temperature_variation', 'vorticity')}
    results = [f.result() for f in futs]
  gv = np.array([tree_dot(gd, v) for v in dirs])
  lin = np.array([sum(2.0 * np.sum(res[k] * jv[k]) / res[k].size for k in res)
                  for jv, _ in results])
  loss_fd = np.array([fd for _, fd in results])
  err = np.abs(gv - lin).max() / np.abs(lin).max()
  assert err <= 1e-4, (err, gv, lin)
  err_fd = np.abs(gv - loss_fd).max() / np.abs(loss_fd).max()
  assert err_fd <= 5e-3, (err_fd, gv, loss_fd)
