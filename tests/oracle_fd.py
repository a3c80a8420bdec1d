"""Central finite differences of the FP64 oracle for the reverse-mode tests.

The functions run in spawned worker processes, so they import only NumPy and
the oracle and rebuild their equations from plain arguments.
"""

import numpy as np

from oracle import dycore as od
from oracle import sht as osht
from oracle import states as ost


def dry_setup(grid_name, layers):
  og = getattr(osht.Grid, grid_name)()
  _, tref, orog, vert = ost.baroclinic_config(og, layers, seed=0)
  oeq = od.PrimitiveEquationsSigma(tref, orog, og, vert, od.SimUnits())
  return og, oeq


def rollout(og, oeq, dt, n_steps, state):
  step = od.step_with_filters(od.imex_rk_sil3(oeq, dt),
                              [od.exponential_step_filter(og, dt)])
  return od.repeated(step, n_steps)(state)


def tracking_loss(final, target):
  """mean((T' - T'_target)^2) + mean((zeta - zeta_target)^2)."""
  return (np.mean((final['temperature_variation'] -
                   target['temperature_variation']) ** 2) +
          np.mean((final['vorticity'] - target['vorticity']) ** 2))




def rollout_jvp_fd(grid_name, layers, dt, n_steps, state, target, direction,
                   eps):
  """Central differences through n filtered steps along `direction`.

  Returns (J v of the final state as a dict, the tracking loss's central
  difference against `target`)."""
  og, oeq = dry_setup(grid_name, layers)
  plus = rollout(og, oeq, dt, n_steps, od.tree_axpy((1.0, state), (eps, direction)))
  minus = rollout(og, oeq, dt, n_steps, od.tree_axpy((1.0, state), (-eps, direction)))
  jv = od.tree_axpy((0.5 / eps, plus), (-0.5 / eps, minus))
  loss_fd = (tracking_loss(plus, target) - tracking_loss(minus, target)) / (2 * eps)
  return jv, loss_fd
