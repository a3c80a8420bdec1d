"""Inputs of the benchmark configurations at their stated sizes, and FP64
oracle runs on them, for the GPU parity tests.

The oracle functions run in spawned worker processes (one member each), so
they import only NumPy and the oracle and rebuild their equations from plain
arguments.

* Held-Suarez ensemble: T42, 24 sigma levels, dt = 15 min (0.131256), rest
  atmosphere at 285 K plus white noise (0.1 K per nodal point, seed = member
  id), compose_equations([PrimitiveEquationsSigma, HeldSuarezForcingSigma]),
  exponential filter tau = 0.0087504, order 1.5, cutoff 0.8.
* Large moist: TL255, 32 sigma levels, dt = 6 min (0.0525024), the JW
  steady state plus a 1 K Gaussian bump (radius 500 km, centre drawn from
  seed = member id), specific humidity exp(N(ln 5e-3, 0.5^2)) clipped to
  <= 0.03 (seed 10) and two passive tracers exp(N(0, 0.5^2)) (seeds 11, 12),
  seeded per nodal point and transformed to modal coefficients; default
  exponential filter.
"""

import numpy as np

from oracle import dycore as od
from oracle import sht as osht
from oracle import states as ost

HS_DT = 0.131256
HS_FILTER = dict(tau=0.0087504, order=1.5, cutoff=0.8)
LARGE_DT = 0.0525024


def rnd32(tree):
  """The FP32-rounded state both sides start from."""
  return od.tree_map(lambda x: np.asarray(x, np.float32).astype(np.float64), tree)


# -- Held-Suarez ensemble -----------------------------------------------------

def hs_member(member, grid_name='T42', layers=24):
  og = getattr(osht.Grid, grid_name)()
  st, tref, orog, vert = ost.held_suarez_config(og, layers, member=member)
  return og, rnd32(st), tref, orog, vert


def hs_oracle_rollout(member, n_steps, grid_name='T42', layers=24):
  """Final FP64 state after n filtered SIL3 steps of one ensemble member."""
  og, st, tref, orog, vert = hs_member(member, grid_name, layers)
  ops = od.SimUnits()
  eq = od.ComposedEquation([od.PrimitiveEquationsSigma(tref, orog, og, vert, ops),
                            od.HeldSuarezForcingSigma(og, vert, ops, tref)])
  step = od.step_with_filters(od.imex_rk_sil3(eq, HS_DT),
                              [od.exponential_step_filter(og, HS_DT, **HS_FILTER)])
  return od.repeated(step, n_steps)(st)


# -- Large moist configuration ----------------------------------------------

LARGE_TRACERS = ('specific_humidity', 'tracer_a', 'tracer_b')


def large_tracers(og, layers):
  """Seeded log-normal nodal fields, transformed to modal coefficients."""
  shape = (layers,) + og.nodal_shape
  q = np.minimum(np.exp(np.random.default_rng(10).normal(np.log(5e-3), 0.5, shape)),
                 0.03)
  a = np.exp(np.random.default_rng(11).normal(0.0, 0.5, shape))
  b = np.exp(np.random.default_rng(12).normal(0.0, 0.5, shape))
  return {name: og.to_modal(f) for name, f in zip(LARGE_TRACERS, (q, a, b))}


def large_member(member, grid_name='TL255', layers=32):
  og = getattr(osht.Grid, grid_name)()
  st, tref, orog, vert = ost.baroclinic_config(og, layers, seed=member)
  st['tracers'] = large_tracers(og, layers)
  return og, rnd32(st), tref, orog, vert


def large_equation(og, tref, orog, vert):
  return od.PrimitiveEquationsSigma(tref, orog, og, vert, od.SimUnits(),
                                    humidity_key='specific_humidity')


def large_step(og, eq):
  return od.step_with_filters(od.imex_rk_sil3(eq, LARGE_DT),
                              [od.exponential_step_filter(og, LARGE_DT)])


def large_oracle_rollout(member, n_steps, grid_name='TL255', layers=32):
  og, st, tref, orog, vert = large_member(member, grid_name, layers)
  step = large_step(og, large_equation(og, tref, orog, vert))
  return od.repeated(step, n_steps)(st)


def large_oracle_step_jvp(member, direction, eps, grid_name='TL255', layers=32):
  """Central difference of one filtered step along `direction` (FP64)."""
  og, st, tref, orog, vert = large_member(member, grid_name, layers)
  step = large_step(og, large_equation(og, tref, orog, vert))
  plus = step(od.tree_axpy((1.0, st), (eps, direction)))
  minus = step(od.tree_axpy((1.0, st), (-eps, direction)))
  return od.tree_axpy((0.5 / eps, plus), (-0.5 / eps, minus))


_THREAD_LIMIT = None


def limit_blas_threads(n):
  """Pool initializer: n BLAS threads per worker, so that workers share the
  host's cores instead of each claiming all of them."""
  global _THREAD_LIMIT
  from threadpoolctl import threadpool_limits
  _THREAD_LIMIT = threadpool_limits(n)


def oracle_pool(workers):
  """A spawn-started process pool for the oracle (never forked after the
  first GPU call), each worker with its share of the host threads."""
  import concurrent.futures
  import multiprocessing
  import os
  cpus = os.cpu_count() or 1
  workers = max(1, min(workers, cpus))
  return concurrent.futures.ProcessPoolExecutor(
      workers, mp_context=multiprocessing.get_context('spawn'),
      initializer=limit_blas_threads, initargs=(max(1, cpus // workers),))
