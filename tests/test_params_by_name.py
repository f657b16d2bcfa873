"""pg_params by field name, and the header next to the reference's macros.

The reference configures itself with macros that share names with pg_params
fields (global.h:16-26: EOS, plnt_flag, FrRot_flag, ... and `#define
flat_flag` with no value).  include/penguin_b200.h sets those macros aside
around its struct, so it compiles after the reference's headers, and
pg_params_set / pg_params_get reach every field by name from such a unit."""
import ctypes as C
import math
import os
import subprocess

import pytest

from penguin_2_0_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PG_OK, PG_ERR_ARG = 0, 9


def _fields():
    return [(n, t) for n, t in _lib.pg_params._fields_ if n != "reserved"]


def test_every_field_round_trips_by_name():
    L = _lib.lib()
    p = _lib.pg_params()
    assert L.pg_config_params(0, C.byref(p)) == PG_OK
    for k, (name, t) in enumerate(_fields()):
        v = float(k + 3) if t is not C.c_double else 0.125 * (k + 1)
        assert L.pg_params_set(C.byref(p), name.encode(), v) == PG_OK, name
        assert float(getattr(p, name)) == v, name                # the struct field itself
        out = C.c_double()
        assert L.pg_params_get(C.byref(p), name.encode(), C.byref(out)) == PG_OK, name
        assert out.value == v, name


def test_bad_names_and_values_are_refused_unchanged():
    L = _lib.lib()
    p = _lib.pg_params()
    assert L.pg_config_params(0, C.byref(p)) == PG_OK
    before = bytes(p)
    for name, v in ((b"no_such_field", 1.0), (b"imax", 2.5), (b"imax", math.nan), (b"EOS", 1e12),
                    (b"seed", -1.0), (b"reserved", 0.0)):
        assert L.pg_params_set(C.byref(p), name, v) == PG_ERR_ARG, (name, v)
    assert bytes(p) == before


UNIT = r"""
/* the reference's configuration style: flag macros named like the fields */
#define ndim 2
#define flat_flag
#define EOS 0
#define plnt_flag 1
#define FrRot_flag 1
#define kill_flag 0
#define visc_flag 1
#define FARGO_flag 1
#define dump_flag 1
#include "penguin_b200.h"

int fill(pg_params *p) {
  int st = pg_default_params(p);
  st |= pg_params_set(p, "ndim", ndim);
  st |= pg_params_set(p, "EOS", EOS);
  st |= pg_params_set(p, "plnt_flag", plnt_flag);
#ifdef flat_flag
  st |= pg_params_set(p, "flat_flag", 1);
#endif
  return st + EOS + ndim;   /* the macros are still in force after the header */
}
"""


@pytest.mark.parametrize("compiler,std", [("gcc", "-std=c11"), ("g++", "-std=c++17")])
def test_header_compiles_after_the_reference_macros(tmp_path, compiler, std):
    src = tmp_path / ("unit.c" if compiler == "gcc" else "unit.cpp")
    src.write_text(UNIT)
    r = subprocess.run([compiler, std, "-Wall", "-Werror", "-fsyntax-only", "-I", os.path.join(ROOT, "include"),
                        str(src)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
