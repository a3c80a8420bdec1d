"""Builds ``libdino_b200.so`` in-tree with nvcc for sm_100a.

Usage: ``python -m dinosaur_b200.build`` (or ``__graft_entry__.build()``).
Each ``csrc/*.cu`` compiles to an object under ``_build/`` in parallel, then
the objects link into ``dinosaur_b200/libdino_b200.so`` with a static CUDA
runtime.
"""

from __future__ import annotations

import concurrent.futures
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, 'csrc')
BUILD = os.path.join(ROOT, '_build')
LIB = os.path.join(PKG, 'libdino_b200.so')

ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
FLAGS = ['-O3', '-lineinfo', '-std=c++17', '--expt-relaxed-constexpr',
         '-Xcompiler', '-fPIC', '-Xcompiler', '-fvisibility=hidden',
         '-I', os.path.join(ROOT, 'include')]


def nvcc() -> str:
  path = shutil.which('nvcc') or '/usr/local/cuda/bin/nvcc'
  if not os.path.exists(path):
    raise RuntimeError('nvcc not found; the CUDA toolkit is required to build')
  return path


def _compile(src: str, extra: list[str]) -> str:
  obj = os.path.join(BUILD, os.path.basename(src) + '.o')
  if os.path.exists(obj) and os.path.getmtime(obj) >= max(
      os.path.getmtime(src), _newest_header()):
    return obj
  cmd = [nvcc(), *ARCH, *FLAGS, *extra, '-c', src, '-o', obj]
  proc = subprocess.run(cmd, capture_output=True, text=True)
  if proc.returncode != 0:
    raise RuntimeError(f'nvcc failed for {src}:\n{proc.stderr}')
  if proc.stderr.strip():
    sys.stderr.write(proc.stderr)
  return obj


def _newest_header() -> float:
  heads = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith('.cuh')]
  heads.append(os.path.join(ROOT, 'include', 'dino_b200.h'))
  return max(os.path.getmtime(h) for h in heads)


def build(verbose: bool = False, extra: list[str] | None = None) -> str:
  """Compiles and links the library; returns its path."""
  os.makedirs(BUILD, exist_ok=True)
  sources = sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC)
                   if f.endswith('.cu'))
  extra = list(extra or [])
  with concurrent.futures.ThreadPoolExecutor(max_workers=8) as ex:
    objs = list(ex.map(lambda s: _compile(s, extra), sources))
  newest_obj = max(os.path.getmtime(o) for o in objs)
  if not os.path.exists(LIB) or os.path.getmtime(LIB) < newest_obj:
    tmp = LIB + '.tmp'
    cmd = [nvcc(), *ARCH, '-shared', '-Xlinker', '--no-undefined', '-o', tmp, *objs]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
      raise RuntimeError(f'link failed:\n{proc.stderr}')
    os.replace(tmp, LIB)
  if verbose:
    print(f'built {LIB}')
  return LIB


if __name__ == '__main__':
  build(verbose=True, extra=sys.argv[1:])
