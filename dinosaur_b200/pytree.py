"""Minimal pytree mapping (dicts, lists, tuples, dataclasses, tensors).

Follows the semantics of ``pytree_utils.tree_map_over_nonscalars``
(dinosaur/pytree_utils.py:86-98): ``f`` is applied to every array leaf with at
least one dimension; scalars (``sim_time`` and the like) pass through.
"""

from __future__ import annotations

import dataclasses

import numpy as np
import torch


def _is_array(x):
  return isinstance(x, (torch.Tensor, np.ndarray))


def tree_map(f, x, *rest):
  """Maps f over matching leaves of x and rest (same structure)."""
  if isinstance(x, dict):
    return type(x)({k: tree_map(f, v, *[r[k] for r in rest])
                    for k, v in x.items()})
  if isinstance(x, (list, tuple)) and not hasattr(x, '_fields'):
    return type(x)(tree_map(f, v, *[r[i] for r in rest])
                   for i, v in enumerate(x))
  if dataclasses.is_dataclass(x) and not isinstance(x, type):
    kw = {fld.name: tree_map(f, getattr(x, fld.name),
                             *[getattr(r, fld.name) for r in rest])
          for fld in dataclasses.fields(x)}
    return dataclasses.replace(x, **kw)
  if x is None:
    return None
  return f(x, *rest)


def map_over_nonscalars(f, x):
  def g(leaf):
    if _is_array(leaf) and leaf.ndim > 0:
      return f(leaf)
    return leaf
  return tree_map(g, x)


def leaves(x):
  out = []
  tree_map(lambda v: out.append(v), x)
  return out
