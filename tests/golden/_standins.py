"""NumPy stand-ins for ``jax``, ``tree_math`` and ``pint``.

Used only by ``make_golden.py`` in a container where the reference
(neuralgcm/dinosaur) is present but its dependencies are not installed.  The
stand-ins give the reference's modules just enough of those APIs to execute
the hot-path functions eagerly in FP64 NumPy: ``jax.numpy`` maps to NumPy,
``jit``/``named_call``/``checkpoint`` are identities, ``lax.scan`` is a Python
loop, pytrees are tuples/lists/dicts/``tree_math.struct`` dataclasses, and
units are a four-dimension (length, time, mass, temperature) SI quantity.
None of this is product code.
"""

from __future__ import annotations

import dataclasses
import functools
import sys
import types

import numpy as np


# ---------------------------------------------------------------------------
# Pytrees
# ---------------------------------------------------------------------------

_STRUCTS = set()


def _is_node(x):
  return (x is None or isinstance(x, (tuple, list, dict))
          or type(x) in _STRUCTS)


def tree_flatten(tree, is_leaf=None):
  leaves = []

  def rec(x):
    if is_leaf is not None and is_leaf(x):
      leaves.append(x)
      return ('leaf',)
    if x is None:
      return ('none',)
    if type(x) in _STRUCTS:
      names = [f.name for f in dataclasses.fields(x)]
      return ('struct', type(x), names, [rec(getattr(x, n)) for n in names])
    if isinstance(x, dict):
      keys = sorted(x.keys())
      return ('dict', type(x), keys, [rec(x[k]) for k in keys])
    if isinstance(x, (tuple, list)):
      return ('seq', type(x), [rec(v) for v in x])
    leaves.append(x)
    return ('leaf',)

  return leaves, rec(tree)


def tree_unflatten(treedef, leaves):
  it = iter(leaves)

  def rec(d):
    kind = d[0]
    if kind == 'leaf':
      return next(it)
    if kind == 'none':
      return None
    if kind == 'struct':
      _, cls, names, subs = d
      return cls(**{n: rec(s) for n, s in zip(names, subs)})
    if kind == 'dict':
      _, cls, keys, subs = d
      return cls({k: rec(s) for k, s in zip(keys, subs)})
    _, cls, subs = d
    vals = [rec(s) for s in subs]
    return cls(vals) if cls in (list, tuple) else cls(*vals)

  return rec(treedef)


def _flatten_up_to(treedef, tree):
  """Subtrees of ``tree`` at the leaf positions of ``treedef`` (jax semantics)."""
  out = []

  def rec(d, x):
    kind = d[0]
    if kind == 'leaf':
      out.append(x)
    elif kind == 'none':
      pass
    elif kind == 'struct':
      for n, s in zip(d[2], d[3]):
        rec(s, getattr(x, n))
    elif kind == 'dict':
      for k, s in zip(d[2], d[3]):
        rec(s, x[k])
    else:
      for s, v in zip(d[2], x):
        rec(s, v)

  rec(treedef, tree)
  return out


def tree_map(f, tree, *rest, is_leaf=None):
  leaves, treedef = tree_flatten(tree, is_leaf)
  others = [_flatten_up_to(treedef, r) for r in rest]
  return tree_unflatten(treedef, [f(*xs) for xs in zip(leaves, *others)])


# ---------------------------------------------------------------------------
# jax.numpy
# ---------------------------------------------------------------------------

class AtArray(np.ndarray):
  """ndarray with a functional ``.at[idx].set/add`` like jax arrays."""

  @property
  def at(self):
    arr = self

    class _Idx:
      def __getitem__(self, idx):
        class _Op:
          def set(self, v):
            out = np.array(arr).view(AtArray)
            out[idx] = v
            return out

          def add(self, v):
            out = np.array(arr).view(AtArray)
            out[idx] += v
            return out
        return _Op()
    return _Idx()


def _at(x):
  return np.asarray(x).view(AtArray)


def _strip(kw):
  kw.pop('precision', None)
  kw.pop('preferred_element_type', None)
  return kw


def _einsum(*args, **kw):
  args = [list(a) if isinstance(a, range) else a for a in args]
  return _at(np.einsum(*args, **_strip(kw)))


class _JnpModule(types.ModuleType):
  def __getattr__(self, name):
    return getattr(np, name)


jnp = _JnpModule('jax.numpy')
jnp.einsum = _einsum
jnp.dot = lambda a, b, **kw: np.dot(a, b)
jnp.matmul = lambda a, b, **kw: np.matmul(a, b)
jnp.ones = lambda *a, **k: _at(np.ones(*a, **k))
jnp.zeros = lambda *a, **k: _at(np.zeros(*a, **k))
jnp.full = lambda *a, **k: _at(np.full(*a, **k))
jnp.zeros_like = lambda *a, **k: _at(np.zeros_like(*a, **k))
jnp.ones_like = lambda *a, **k: _at(np.ones_like(*a, **k))
jnp.asarray = lambda x, dtype=None: _at(np.asarray(x, dtype=dtype))
jnp.array = lambda x, dtype=None: _at(np.array(x, dtype=dtype))
jnp.searchsorted = lambda a, v, side='left', method=None: np.searchsorted(
    a, v, side=side)
jnp.ndarray = np.ndarray


# ---------------------------------------------------------------------------
# jax.lax
# ---------------------------------------------------------------------------

class _Precision:
  DEFAULT = 'default'
  HIGH = 'high'
  HIGHEST = 'highest'


def _slice_in_dim(x, start, limit, stride=1, axis=0):
  idx = [slice(None)] * np.ndim(x)
  idx[axis] = slice(start, limit, stride)
  return np.asarray(x)[tuple(idx)]


def _lax_pad(x, padding_value, padding_config):
  pads = []
  for lo, hi, interior in padding_config:
    assert interior == 0 and lo >= 0 and hi >= 0
    pads.append((lo, hi))
  return np.pad(x, pads, constant_values=padding_value)


def _scan(f, init, xs=None, length=None):
  carry = init
  ys = []
  n = length if length is not None else len(tree_flatten(xs)[0][0])
  for i in range(n):
    x = None if xs is None else tree_map(lambda a: a[i], xs)
    carry, y = f(carry, x)
    ys.append(y)
  if ys and ys[0] is not None:
    stacked = tree_map(lambda *a: np.stack(a), ys[0], *ys[1:])
  else:
    stacked = None
  return carry, stacked


lax = types.ModuleType('jax.lax')
lax.Precision = _Precision
lax.slice_in_dim = _slice_in_dim
lax.pad = _lax_pad
lax.scan = _scan
lax.with_sharding_constraint = lambda x, s: x


# ---------------------------------------------------------------------------
# jax
# ---------------------------------------------------------------------------

def _decorator_or_identity(fn=None, *a, **k):
  if fn is None or not callable(fn):
    return lambda g: g
  return fn


def _vmap(fn, in_axes=0, out_axes=0, *a, **k):
  """jax.vmap over axis 0 of every positional argument (the only form the
  reference's state constructors use): maps a Python loop and stacks each
  output leaf."""
  def mapped(*args):
    if in_axes != 0 or out_axes != 0:
      raise NotImplementedError('the stand-in vmap maps axis 0 only')
    n = len(np.asarray(tree_flatten(args[0])[0][0]))
    outs = [fn(*[tree_map(lambda x, i=i: np.asarray(x)[i], arg) for arg in args])
            for i in range(n)]
    return tree_map(lambda *xs: np.stack([np.asarray(x) for x in xs]), *outs)
  return mapped


class _Dummy:
  def __init__(self, *a, **k):
    pass

  def __call__(self, *a, **k):
    return _Dummy()


jax = types.ModuleType('jax')
jax.numpy = jnp
jax.lax = lax
jax.Array = np.ndarray
jax.named_call = lambda fn=None, name=None: (
    (lambda g: g) if fn is None else fn)
jax.jit = _decorator_or_identity
jax.checkpoint = _decorator_or_identity
jax.vmap = _vmap
jax.device_get = lambda x: x
jax.tree_util = types.ModuleType('jax.tree_util')
jax.tree_util.tree_map = tree_map
jax.tree_util.tree_flatten = tree_flatten
jax.tree_util.tree_unflatten = tree_unflatten
jax.tree_util.register_pytree_node = lambda *a, **k: None
jax.tree_util.register_dataclass = lambda *a, **k: None
jax.tree = types.SimpleNamespace(map=tree_map, flatten=tree_flatten,
                                 unflatten=tree_unflatten)
jax.core = types.SimpleNamespace(Tracer=type('Tracer', (), {}))
jax.dtypes = types.SimpleNamespace(canonicalize_dtype=np.dtype)
jax.config = types.SimpleNamespace(update=lambda *a, **k: None,
                                   parse_flags_with_absl=lambda: None)
jax.sharding = types.SimpleNamespace(PartitionSpec=_Dummy, Mesh=_Dummy,
                                     NamedSharding=_Dummy)
jax.shard_map = _Dummy()
jax.experimental = types.ModuleType('jax.experimental')
jax.experimental.shard_map = types.SimpleNamespace(shard_map=_Dummy())
jax.ShapeDtypeStruct = _Dummy
jax.random = types.SimpleNamespace()


# ---------------------------------------------------------------------------
# tree_math
# ---------------------------------------------------------------------------

class Vector:
  """Vector-space view of a pytree (tree_math.Vector)."""

  def __init__(self, tree):
    self.tree = tree

  def _binary(self, other, op):
    if isinstance(other, Vector):
      return Vector(tree_map(op, self.tree, other.tree))
    return Vector(tree_map(lambda x: op(x, other), self.tree))

  def __add__(self, o): return self._binary(o, lambda a, b: a + b)
  def __radd__(self, o):
    if isinstance(o, (int, float)) and o == 0:
      return self
    return self._binary(o, lambda a, b: b + a)
  def __sub__(self, o): return self._binary(o, lambda a, b: a - b)
  def __mul__(self, o): return self._binary(o, lambda a, b: a * b)
  def __rmul__(self, o): return self._binary(o, lambda a, b: b * a)
  def __truediv__(self, o): return self._binary(o, lambda a, b: a / b)
  def __neg__(self): return Vector(tree_map(lambda a: -a, self.tree))


def _struct(cls):
  cls = dataclasses.dataclass(cls)
  _STRUCTS.add(cls)

  def _bin(op):
    def f(self, other):
      if type(other) in _STRUCTS:
        return tree_map(op, self, other)
      return tree_map(lambda a: op(a, other), self)
    return f

  cls.__add__ = _bin(lambda a, b: a + b)
  cls.__sub__ = _bin(lambda a, b: a - b)
  cls.__mul__ = _bin(lambda a, b: a * b)
  cls.__rmul__ = _bin(lambda a, b: b * a)
  cls.__truediv__ = _bin(lambda a, b: a / b)
  cls.__neg__ = lambda self: tree_map(lambda a: -a, self)
  cls.fields = property(lambda self: dataclasses.fields(self))
  return cls


def _wrap(fn):
  @functools.wraps(fn)
  def wrapped(*args):
    out = fn(*[Vector(a) for a in args])
    return out.tree if isinstance(out, Vector) else out
  return wrapped


def _unwrap(fn, vector_argnums=None):
  @functools.wraps(fn)
  def unwrapped(*args):
    new = []
    for i, a in enumerate(args):
      is_vec = vector_argnums is None or i == vector_argnums or (
          isinstance(vector_argnums, (tuple, list)) and i in vector_argnums)
      new.append(a.tree if (is_vec and isinstance(a, Vector)) else a)
    return Vector(fn(*new))
  return unwrapped


tree_math = types.ModuleType('tree_math')
tree_math.struct = _struct
tree_math.wrap = _wrap
tree_math.unwrap = _unwrap
tree_math.Vector = Vector


# ---------------------------------------------------------------------------
# pint (SI, four base dimensions)
# ---------------------------------------------------------------------------

class _Dims(dict):
  def __str__(self):
    if len(self) == 1:
      (k, v), = self.items()
      if v == 1:
        return k
    return ' * '.join(f'{k} ** {v}' for k, v in sorted(self.items()))

  def __hash__(self):
    return hash(tuple(sorted(self.items())))


def _dims_mul(a, b, sign=1):
  out = dict(a)
  for k, v in b.items():
    out[k] = out.get(k, 0) + sign * v
    if out[k] == 0:
      del out[k]
  return _Dims(out)


class Quantity:
  # NumPy defers ndarray * Quantity to __rmul__ (as with pint's quantities).
  __array_ufunc__ = None

  def __init__(self, magnitude, dims=None):
    self.magnitude = magnitude
    self.dimensionality = _Dims(dims or {})

  @property
  def m(self):
    return self.magnitude

  def _coerce(self, o):
    return o if isinstance(o, Quantity) else Quantity(o)

  def __mul__(self, o):
    o = self._coerce(o)
    return Quantity(self.magnitude * o.magnitude,
                    _dims_mul(self.dimensionality, o.dimensionality))

  __rmul__ = __mul__

  def __truediv__(self, o):
    o = self._coerce(o)
    return Quantity(self.magnitude / o.magnitude,
                    _dims_mul(self.dimensionality, o.dimensionality, -1))

  def __rtruediv__(self, o):
    return self._coerce(o) / self

  def __pow__(self, p):
    return Quantity(self.magnitude ** p,
                    {k: v * p for k, v in self.dimensionality.items()})

  def __neg__(self):
    return Quantity(-self.magnitude, self.dimensionality)

  def to_base_units(self):
    return self

  def check(self, dims):
    return dict(self.dimensionality) == dict(dims)

  def to(self, unit):
    unit = self._coerce(unit)
    if dict(self.dimensionality) != dict(unit.dimensionality):
      raise ValueError(f'incompatible units {self.dimensionality} -> '
                       f'{unit.dimensionality}')
    return Quantity(self.magnitude / unit.magnitude, unit.dimensionality)


_L, _T, _M, _K = '[length]', '[time]', '[mass]', '[temperature]'


class UnitRegistry:
  Quantity = Quantity
  Unit = Quantity

  def __init__(self, *a, **k):
    kg = Quantity(1.0, {_M: 1})
    m = Quantity(1.0, {_L: 1})
    s = Quantity(1.0, {_T: 1})
    k_ = Quantity(1.0, {_K: 1})
    joule = kg * m ** 2 / s ** 2
    pascal = kg / m / s ** 2
    self._units = dict(
        m=m, meter=m, km=m * 1000.0, s=s, sec=s, second=s,
        minute=s * 60.0, hour=s * 3600.0, day=s * 86400.0,
        kg=kg, kilogram=kg, gram=kg * 1e-3, degK=k_, kelvin=k_, K=k_,
        J=joule, joule=joule, Pa=pascal, pascal=pascal,
        hPa=pascal * 100.0, dimensionless=Quantity(1.0),
        radian=Quantity(1.0), W=joule / s)

  def __getattr__(self, name):
    try:
      return self.__dict__['_units'][name]
    except KeyError:
      raise AttributeError(name) from None

  def parse_expression(self, s):
    return getattr(self, s.strip())


pint = types.ModuleType('pint')
pint.UnitRegistry = UnitRegistry
pint.Quantity = Quantity
pint.util = types.SimpleNamespace(UnitsContainer=_Dims)


# ---------------------------------------------------------------------------
# Installation
# ---------------------------------------------------------------------------

def install(reference_root: str):
  """Registers the stand-ins and a bare ``dinosaur`` package.

  The package object is created directly (its ``__init__`` would import
  xarray-based I/O modules that the hot path does not use); submodules load
  from ``<reference_root>/dinosaur``.  ``dinosaur.xarray_utils`` is replaced
  by the three key names that the state constructors use.
  """
  sys.modules['jax'] = jax
  sys.modules['jax.numpy'] = jnp
  sys.modules['jax.lax'] = lax
  sys.modules['jax.tree_util'] = jax.tree_util
  sys.modules['jax.experimental'] = jax.experimental
  sys.modules['jax.experimental.shard_map'] = jax.experimental.shard_map
  sys.modules['tree_math'] = tree_math
  sys.modules['pint'] = pint
  pkg = types.ModuleType('dinosaur')
  pkg.__path__ = [f'{reference_root}/dinosaur']
  sys.modules['dinosaur'] = pkg
  xu = types.ModuleType('dinosaur.xarray_utils')
  xu.OROGRAPHY = 'orography'
  xu.GEOPOTENTIAL_KEY = 'geopotential'
  xu.REF_TEMP_KEY = 'ref_temperatures'
  sys.modules['dinosaur.xarray_utils'] = xu
  pkg.xarray_utils = xu
