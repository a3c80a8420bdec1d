"""CPU-side checks of the C ABI: the library loads and exports every symbol
declared in include/dino_b200.h (no kernel is launched)."""

import ctypes
import os
import re

import pytest

from dinosaur_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
  text = open(os.path.join(ROOT, 'include', 'dino_b200.h')).read()
  return sorted(set(re.findall(r'DINO_API\s+[\w\s\*]+?\b(dino_\w+)\s*\(', text)))


def test_library_is_built():
  assert os.path.exists(_lib.LIB_PATH), 'run python -m dinosaur_b200.build'


def test_every_declared_symbol_is_exported():
  handle = ctypes.CDLL(_lib.LIB_PATH)
  names = declared_symbols()
  assert len(names) >= 15
  missing = [n for n in names if not hasattr(handle, n)]
  assert not missing, missing


def test_bindings_cover_header():
  assert set(declared_symbols()) <= set(_lib.SIGNATURES)


def test_version_and_error_string():
  lib = _lib.lib()
  assert b'sm_100a' in lib.dino_version()
  assert _lib.last_error() is not None


def test_null_arguments_are_rejected_without_gpu():
  lib = _lib.lib()
  rc = lib.dino_sht_inverse(None, None, None, 1, None)
  assert rc == _lib.DINO_ERR_ARG
  assert 'null' in _lib.last_error()
  with pytest.raises(ValueError):
    _lib.check(rc)


def test_plan_rejects_bad_shapes_without_gpu():
  lib = _lib.lib()
  desc = _lib.GridDesc(10, 5, 64, 32, 0, 0, 1.0, None, None)
  h = ctypes.c_void_p()
  rc = lib.dino_plan_create(ctypes.byref(desc), 8, 0, ctypes.byref(h))
  assert rc == _lib.DINO_ERR_SHAPE
  assert 'n_m <= n_l' in _lib.last_error()


@pytest.mark.parametrize('cname,pyname', [('dino_grid_desc', 'GridDesc'),
                                          ('dino_pe_desc', 'PEDesc'),
                                          ('dino_swe_desc', 'SWEDesc')])
def test_descriptor_layouts_match_the_header(cname, pyname, tmp_path):
  """The ctypes mirrors of the descriptor structs have the header's size and
  field offsets (a C program compiled against include/dino_b200.h prints
  them)."""
  import shutil
  import subprocess
  gcc = shutil.which('gcc') or shutil.which('cc')
  if gcc is None:
    pytest.skip('no C compiler')
  py = getattr(_lib, pyname)
  fields = [f[0] for f in py._fields_]
  src = tmp_path / 'layout.c'
  lines = ['#include <stdio.h>', '#include "dino_b200.h"', 'int main(void) {',
           f'  printf("%zu\\n", sizeof({cname}));']
  lines += [f'  printf("%zu\\n", offsetof({cname}, {f}));' for f in fields]
  lines += ['  return 0;', '}']
  src.write_text('\n'.join(lines) + '\n')
  exe = tmp_path / 'layout'
  subprocess.run([gcc, '-I', os.path.join(ROOT, 'include'), str(src), '-o', str(exe)],
                 check=True, capture_output=True)
  out = [int(x) for x in subprocess.run([str(exe)], check=True, capture_output=True,
                                        text=True).stdout.split()]
  assert out[0] == ctypes.sizeof(py), (out[0], ctypes.sizeof(py))
  assert out[1:] == [getattr(py, f).offset for f in fields]
