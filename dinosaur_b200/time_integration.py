"""Time integration: IMEX Runge-Kutta (SIL3), step filters, rollouts.

Mirrors ``dinosaur/time_integration.py`` (reference v1.3.6): the ODE
protocols (:56-114), ``compose_equations`` (:141-161), ``imex_runge_kutta`` /
``imex_rk_sil3`` (:313-405), the step filters (:414-486), ``step_with_filters``,
``repeated`` and ``trajectory_from_step`` (:494-564).

For ``PrimitiveEquationsSigma`` the SIL3 step is fused: ``imex_rk_sil3``
returns a ``FusedSIL3Step`` that runs the whole step (three explicit
evaluations, three per-wavenumber solves, the final combination and the
per-l step filters) inside ``libdino_b200`` on a packed state, optionally as a
replayed CUDA graph.  Any other equation uses the generic tableau loop below,
which follows the reference step for step.
"""

from __future__ import annotations

import dataclasses
from typing import Any, Callable, Sequence

import numpy as np
import torch

from dinosaur_b200 import pytree


class ExplicitODE:
  """ODE with explicit terms only (time_integration.py:56-71)."""

  def explicit_terms(self, state):
    raise NotImplementedError

  @classmethod
  def from_functions(cls, explicit_terms):
    ode = cls()
    ode.explicit_terms = explicit_terms
    return ode


class ImplicitExplicitODE:
  """dx/dt = explicit_terms(x) + implicit_terms(x) (time_integration.py:74-114)."""

  def explicit_terms(self, state):
    raise NotImplementedError

  def implicit_terms(self, state):
    raise NotImplementedError

  def implicit_inverse(self, state, step_size: float):
    raise NotImplementedError

  @classmethod
  def from_functions(cls, explicit_terms, implicit_terms, implicit_inverse):
    ode = cls()
    ode.explicit_terms = explicit_terms
    ode.implicit_terms = implicit_terms
    ode.implicit_inverse = implicit_inverse
    return ode


def _tree_add(*trees):
  return pytree.tree_map(
      lambda *xs: sum(x for x in xs if x is not None), *trees)


def compose_equations(equations: Sequence[Any]) -> ImplicitExplicitODE:
  """time_integration.py:141-161.

  The primitive equations composed with Held-Suarez forcing become one fused
  equation that shares the diagnostic state between the two tendencies.
  """
  from dinosaur_b200 import held_suarez  # pylint: disable=g-import-not-at-top
  from dinosaur_b200 import primitive_equations as pe  # pylint: disable=g-import-not-at-top
  imex = [e for e in equations if isinstance(e, ImplicitExplicitODE)]
  if len(imex) != 1:
    raise ValueError('compose_equations supports at most 1 ImplicitExplicitODE '
                     f'got {len(imex)}')
  (primary,) = imex
  others = [e for e in equations if e is not primary]
  if (isinstance(primary, pe.PrimitiveEquationsSigma) and len(others) == 1
      and isinstance(others[0], held_suarez.HeldSuarezForcingSigma)
      and primary.held_suarez is None):
    return dataclasses.replace(primary, held_suarez=others[0])

  def explicit_fn(x):
    return _tree_add(*[fn.explicit_terms(x) for fn in equations])

  return ImplicitExplicitODE.from_functions(
      explicit_fn, primary.implicit_terms, primary.implicit_inverse)


@dataclasses.dataclass
class ImExButcherTableau:
  a_ex: Sequence[Sequence[float]]
  a_im: Sequence[Sequence[float]]
  b_ex: Sequence[float]
  b_im: Sequence[float]

  def __post_init__(self):
    if len({len(self.a_ex) + 1, len(self.a_im) + 1, len(self.b_ex),
            len(self.b_im)}) > 1:
      raise ValueError('inconsistent Butcher tableau')


SIL3_TABLEAU = ImExButcherTableau(
    a_ex=[[1 / 3], [1 / 6, 1 / 2], [1 / 2, -1 / 2, 1]],
    a_im=[[1 / 6, 1 / 6], [1 / 3, 0, 1 / 3], [3 / 8, 0, 3 / 8, 1 / 4]],
    b_ex=[1 / 2, -1 / 2, 1, 0],
    b_im=[3 / 8, 0, 3 / 8, 1 / 4],
)


def _axpy(terms):
  """sum_i c_i * tree_i over (c_i, tree_i)."""
  coeffs = [c for c, _ in terms]
  trees = [t for _, t in terms]
  return pytree.tree_map(
      lambda *xs: sum(c * x for c, x in zip(coeffs, xs)), *trees)


def imex_runge_kutta(tableau: ImExButcherTableau, equation, time_step: float):
  """Generic IMEX-RK step (time_integration.py:329-372)."""
  dt = time_step
  F, G, G_inv = (equation.explicit_terms, equation.implicit_terms,
                 equation.implicit_inverse)
  a_ex, a_im, b_ex, b_im = tableau.a_ex, tableau.a_im, tableau.b_ex, tableau.b_im
  n = len(b_ex)

  def step_fn(y0):
    f = [None] * n
    g = [None] * n
    f[0] = F(y0)
    g[0] = G(y0)
    for i in range(1, n):
      terms = [(1.0, y0)]
      terms += [(dt * a_ex[i - 1][j], f[j]) for j in range(i) if a_ex[i - 1][j]]
      terms += [(dt * a_im[i - 1][j], g[j]) for j in range(i) if a_im[i - 1][j]]
      y = G_inv(_axpy(terms), dt * a_im[i - 1][i])
      if any(a_ex[j][i] for j in range(i, n - 1)) or b_ex[i]:
        f[i] = F(y)
      if any(a_im[j][i] for j in range(i, n - 1)) or b_im[i]:
        g[i] = G(y)
    terms = [(1.0, y0)]
    terms += [(dt * b_ex[j], f[j]) for j in range(n) if b_ex[j]]
    terms += [(dt * b_im[j], g[j]) for j in range(n) if b_im[j]]
    return _axpy(terms)

  return step_fn


@dataclasses.dataclass
class FusedSIL3Step:
  """One or more filtered SIL3 steps of the primitive equations on the GPU.

  Calling it is ``repeated(step_with_filters(imex_rk_sil3(eq, dt), filters),
  n_steps)`` of the reference; ``use_graph`` replays a captured CUDA graph of
  one step.
  """

  equation: Any
  dt: float
  filter_scaling: np.ndarray | None = None
  n_steps: int = 1
  use_graph: bool = True

  def __call__(self, state):
    from dinosaur_b200 import primitive_equations as pe  # pylint: disable=g-import-not-at-top
    eng = self.equation.engine(state)
    buf = eng.pack(state)  # a fresh buffer: the input state is not modified
    if torch.is_grad_enabled() and buf.requires_grad:
      # Differentiable rollout with hand-written step VJPs.
      buf = pe._RolloutFn.apply(buf, eng, self.dt, self.filter_scaling,  # pylint: disable=protected-access
                                self.n_steps)
    else:
      eng.step_(buf, self.dt, self.filter_scaling, self.n_steps,
                graph=self.use_graph)
    sim_time = state.sim_time
    if sim_time is not None:
      sim_time = sim_time + self.dt * self.n_steps
    return eng.unpack(buf, state, sim_time)

  def step_packed_(self, eng, buf):
    """Advances a packed state buffer in place (no copies)."""
    eng.step_(buf, self.dt, self.filter_scaling, self.n_steps,
              graph=self.use_graph)
    return buf


@dataclasses.dataclass
class TimeReversedImExODE(ImplicitExplicitODE):
  """An ImplicitExplicitODE reversed in time (time_integration.py:117-138):
  dx/dt = -explicit_terms(x) - implicit_terms(x)."""

  forward_eq: Any

  def explicit_terms(self, state):
    return pytree.tree_map(lambda x: -x if _is_tensor_like(x) else x,
                           self.forward_eq.explicit_terms(state))

  def implicit_terms(self, state):
    return pytree.tree_map(lambda x: -x if _is_tensor_like(x) else x,
                           self.forward_eq.implicit_terms(state))

  def implicit_inverse(self, state, step_size: float):
    return self.forward_eq.implicit_inverse(state, -step_size)


def _is_tensor_like(x):
  return isinstance(x, (torch.Tensor, np.ndarray, float, int)) and x is not None


def imex_rk_sil3(equation, time_step: float):
  """SIL3 IMEX-RK step (time_integration.py:375-405).

  The primitive equations take the fused CUDA step; their time-reversed ODE
  is the same step with -dt (negated explicit and implicit terms, implicit
  inverse at -eta)."""
  from dinosaur_b200 import primitive_equations as pe  # pylint: disable=g-import-not-at-top
  if isinstance(equation, pe.PrimitiveEquationsSigma):
    return FusedSIL3Step(equation, float(time_step))
  if (isinstance(equation, TimeReversedImExODE) and
      isinstance(equation.forward_eq, pe.PrimitiveEquationsSigma)):
    return FusedSIL3Step(equation.forward_eq, -float(time_step))
  return imex_runge_kutta(SIL3_TABLEAU, equation, time_step)


# ---------------------------------------------------------------------------
# Filters
# ---------------------------------------------------------------------------


@dataclasses.dataclass
class SpectralStepFilter:
  """A step filter that scales every modal leaf by a per-l factor."""

  scaling: np.ndarray

  def __call__(self, u, u_next):
    del u
    from dinosaur_b200 import filtering  # pylint: disable=g-import-not-at-top
    return filtering.apply_scaling(self.scaling, u_next)


def runge_kutta_step_filter(state_filter):
  """time_integration.py:414-424."""
  def _filter(u, u_next):
    del u
    return state_filter(u_next)
  return _filter


def exponential_step_filter(grid, dt: float, tau: float = 0.010938,
                            order: int = 18, cutoff: float = 0.0):
  """time_integration.py:427-455 with filtering.exponential_filter."""
  from dinosaur_b200 import filtering  # pylint: disable=g-import-not-at-top
  return SpectralStepFilter(filtering.exponential_scaling(
      grid, dt / tau, order, cutoff))


def horizontal_diffusion_step_filter(grid, dt: float, tau: float,
                                     order: int = 1):
  """time_integration.py:458-486."""
  from dinosaur_b200 import filtering  # pylint: disable=g-import-not-at-top
  eigenvalues = grid.laplacian_eigenvalues
  scale = dt / (tau * abs(eigenvalues[-1]) ** order)
  return SpectralStepFilter(filtering.diffusion_scaling(grid, scale, order))


# ---------------------------------------------------------------------------
# Rollouts
# ---------------------------------------------------------------------------


def step_with_filters(step_fn, filters: Sequence[Callable]):
  """time_integration.py:494-505 (fused when every filter is spectral)."""
  if isinstance(step_fn, FusedSIL3Step) and step_fn.n_steps == 1 and all(
      isinstance(f, SpectralStepFilter) for f in filters):
    scaling = step_fn.filter_scaling
    for f in filters:
      s = np.asarray(f.scaling, np.float64)
      scaling = s if scaling is None else scaling * s
    return dataclasses.replace(step_fn, filter_scaling=scaling)

  def _step_fn(u):
    u_next = step_fn(u)
    for filter_fn in filters:
      u_next = filter_fn(u, u_next)
    return u_next

  return _step_fn


def repeated(fn, steps: int, scan_fn=None):
  """time_integration.py:508-520."""
  del scan_fn
  if steps == 1:
    return fn
  if isinstance(fn, FusedSIL3Step):
    return dataclasses.replace(fn, n_steps=fn.n_steps * steps)

  def f_repeated(x):
    for _ in range(steps):
      x = fn(x)
    return x

  return f_repeated


def _stack(frames):
  return pytree.tree_map(
      lambda *xs: torch.stack([torch.as_tensor(x) for x in xs])
      if isinstance(xs[0], torch.Tensor) else (
          np.stack(xs) if isinstance(xs[0], np.ndarray) else xs[-1]), *frames)


def _identity(x):
  return x


def trajectory_from_step(step_fn, outer_steps: int, inner_steps: int, *,
                         start_with_input: bool = False,
                         post_process_fn=_identity, outer_scan_fn=None,
                         inner_scan_fn=None):
  """time_integration.py:523-564: returns x -> (final, stacked frames).

  For the fused primitive-equation step the whole rollout runs natively
  (dino_pe_trajectory): the step graph is replayed and each frame is copied
  on the device into one frame buffer, with no host round trip per frame;
  post_process_fn then maps each frame.  A differentiable rollout, or any
  other step function, runs frame by frame.
  """
  del outer_scan_fn, inner_scan_fn
  if inner_steps != 1:
    step_fn = repeated(step_fn, inner_steps)

  if isinstance(step_fn, FusedSIL3Step):
    fused = step_fn

    def native(x):
      eng = fused.equation.engine(x)
      buf = eng.pack(x)
      if torch.is_grad_enabled() and buf.requires_grad:
        return None
      frames = eng.trajectory_(buf, fused.dt, fused.filter_scaling, outer_steps,
                               fused.n_steps, start_with_input)
      t0 = x.sim_time
      final_time = None if t0 is None else t0 + fused.dt * fused.n_steps * outer_steps
      times = None
      if t0 is not None:
        first = 0 if start_with_input else 1
        times = torch.as_tensor([t0 + fused.dt * fused.n_steps * (i + first)
                                 for i in range(outer_steps)])
      final = eng.unpack(buf, x, final_time)
      if post_process_fn is _identity:
        return final, eng.unpack_frames(frames, x, times)
      per = [post_process_fn(eng.unpack(frames[i], x,
                                        None if times is None else times[i]))
             for i in range(outer_steps)]
      return final, _stack(per)
  else:
    native = None

  def multistep(x):
    if native is not None:
      out = native(x)
      if out is not None:
        return out
    frames = []
    for _ in range(outer_steps):
      x_next = step_fn(x)
      frames.append(post_process_fn(x if start_with_input else x_next))
      x = x_next
    return x, _stack(frames)

  return multistep


# ---------------------------------------------------------------------------
# Digital filter initialisation (time_integration.py:640-716)
# ---------------------------------------------------------------------------


def accumulate_repeated(step_fn, weights, state, scan_fn=None):
  """Weighted sum of the states along repeated steps (time_integration.py:645-660)."""
  del scan_fn

  def zeros(x):
    return torch.zeros_like(x) if isinstance(x, torch.Tensor) else (
        np.zeros_like(x) if isinstance(x, np.ndarray) else x)

  averaged = pytree.tree_map(zeros, state)
  for w in np.asarray(weights):
    state = step_fn(state)
    averaged = pytree.tree_map(
        lambda s, a, w=float(w): a + w * s if _is_array_leaf(s) else a,
        state, averaged)
  return averaged


def _is_array_leaf(x):
  return isinstance(x, (torch.Tensor, np.ndarray)) and x.ndim > 0


def _dfi_lanczos_weights(time_span: float, cutoff_period: float,
                         dt: float) -> np.ndarray:
  """Lanczos weights of the filter window (time_integration.py:663-670)."""
  n_steps = round(time_span / (2 * dt))
  n = np.arange(1, n_steps + 1)
  return (np.sinc(n / (n_steps + 1)) *
          np.sinc(n * time_span / (cutoff_period * n_steps)))


def digital_filter_initialization(equation, ode_solver, filters,
                                  time_span: float, cutoff_period: float,
                                  dt: float):
  """Digital filter initialisation (time_integration.py:673-716; Lynch &
  Huang 1992): the Lanczos-weighted mean of forward and time-reversed
  rollouts over [-time_span / 2, time_span / 2]."""

  def f(state):
    forward_step = step_with_filters(ode_solver(equation, dt), filters)
    backward_step = step_with_filters(
        ode_solver(TimeReversedImExODE(equation), dt), filters)
    weights = _dfi_lanczos_weights(time_span, cutoff_period, dt)
    init_weight = 1.0
    total_weight = init_weight + 2 * weights.sum()
    init_weight /= total_weight
    weights = weights / total_weight
    init_term = pytree.tree_map(
        lambda x: x * init_weight if _is_array_leaf(x) else x, state)
    forward_term = accumulate_repeated(forward_step, weights, state)
    backward_term = accumulate_repeated(backward_step, weights, state)
    return pytree.tree_map(
        lambda a, b, c: a + b + c if _is_array_leaf(a) else a,
        init_term, forward_term, backward_term)

  return f


def maybe_fix_sim_time_roundoff(state, dt: float):
  """Rounds sim_time to a multiple of dt (time_integration.py:719-726)."""
  if getattr(state, 'sim_time', None) is not None:
    state.sim_time = dt * round(state.sim_time / dt)
  return state
