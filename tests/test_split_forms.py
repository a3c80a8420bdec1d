"""Error floor of the split-operand Legendre forms, emulated on the CPU.

The tensor-core forms split every FP32 operand and every FP64 table entry v
into hi = round(v) and lo = round(v - hi) in the operand format and form
hi*hi + hi*lo + lo*hi.  Here the same splits are applied to the oracle's
inverse transform with exact products and FP64 sums, which isolates the
error of the split from the rounding of the tensor cores' FP32 accumulation:

* tf32 (10 stored mantissa bits, round to nearest with ties away from zero,
  as cvt.rna.tf32.f32): relative L2 error ~7e-8 at TL255, so on the GPU the
  accumulator's per-instruction rounding is what remains;
* bf16 (7 stored bits, round to nearest even, as the bf16 conversions): ~4e-6,
  the dropped lo*lo term and lo's own rounding, i.e. most of what the GPU's
  split-BF16 form measures.
"""

import numpy as np
import pytest

from oracle import sht as osht
from oracle import states as ost


def round_tf32(a):
  u = np.asarray(a, np.float32).view(np.uint32).astype(np.uint64)
  return ((u + 0x1000) & 0xFFFFE000).astype(np.uint32).view(np.float32)


def round_bf16(a):
  u = np.asarray(a, np.float32).view(np.uint32).astype(np.uint64)
  u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
  return u.astype(np.uint32).view(np.float32)


def split(v, rnd):
  hi = rnd(np.asarray(v, np.float64).astype(np.float32)).astype(np.float64)
  lo = rnd((np.asarray(v, np.float64) - hi).astype(np.float32)).astype(np.float64)
  return hi, lo


def split_inverse(og, x, rnd):
  """The oracle's to_nodal with the Legendre products formed from splits."""
  f, p, _ = og.basis
  ph, pl = split(p, rnd)
  xh, xl = split(x, rnd)
  mv = lambda a, b: np.matmul(a, b[..., None])[..., 0]
  return np.matmul(f, mv(ph, xh) + mv(ph, xl) + mv(pl, xh))


def test_rounding_helpers():
  x = np.float32(1.0) + np.float32(2.0 ** -11)   # halfway between tf32 neighbours
  assert round_tf32(x) == np.float32(1.0 + 2.0 ** -10)  # ties away
  assert round_tf32(np.float32(1.0 + 2.0 ** -12)) == 1.0
  y = np.float32(1.0) + np.float32(2.0 ** -8)    # halfway between bf16 neighbours
  assert round_bf16(y) == 1.0                    # ties to even
  assert round_bf16(np.float32(1.0 + 3 * 2.0 ** -8)) == np.float32(1.0 + 2.0 ** -6)


@pytest.mark.parametrize('name', ['T85', 'TL255'])
def test_split_error_floor(name):
  og = getattr(osht.Grid, name)()
  x = ost.sht_modal_input(og, 4, seed=0)
  ref = og.to_nodal(x.astype(np.float64))
  rel = lambda y: np.linalg.norm(y - ref) / np.linalg.norm(ref)
  e_tf32 = rel(split_inverse(og, x, round_tf32))
  e_bf16 = rel(split_inverse(og, x, round_bf16))
  assert e_tf32 < 2e-7, e_tf32
  assert 1e-6 < e_bf16 < 1e-5, e_bf16
