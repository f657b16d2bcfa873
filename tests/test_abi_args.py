"""Argument checks of the C ABI, on the CPU.

The reference exits the process on any error (cuSafe.cu:8-47); this library
returns a status instead, and that holds for bad arguments too: every entry
point given NULL handles or NULL output pointers returns PG_ERR_ARG (the
destroy calls accept NULL and return PG_OK; the three planet functions that
return a double give NaN), and an undersized buffer is refused before
anything is written.  None of these calls reach the GPU.  They run in a child
process so that a crash shows up as a failure of this test."""
import ctypes as C
import json
import subprocess
import sys

from penguin_2_0_b200 import _lib

PG_OK, PG_ERR_ARG = 0, 9

# entry point -> (call with NULL arguments; p is a valid pg_params), expected
NULL_CALLS = {
    "pg_default_params": ("L.pg_default_params(None)", PG_ERR_ARG),
    "pg_config_params": ("L.pg_config_params(0, None)", PG_ERR_ARG),
    "pg_check_params": ("L.pg_check_params(None)", PG_ERR_ARG),
    "pg_params_set": ("L.pg_params_set(C.byref(p), None, 1.0)", PG_ERR_ARG),
    "pg_params_get": ("L.pg_params_get(C.byref(p), b'EOS', None)", PG_ERR_ARG),
    "pg_write_ic": ("L.pg_write_ic(C.byref(p), None)", PG_ERR_ARG),
    "pg_build_ic": ("L.pg_build_ic(C.byref(p), None, 0)", PG_ERR_ARG),
    "pg_boundary_rings": ("L.pg_boundary_rings(C.byref(p), None, 0, None)", PG_ERR_ARG),
    "pg_label": ("L.pg_label(C.byref(p), None, 0)", PG_ERR_ARG),
    "pg_dump_name": ("L.pg_dump_name(C.byref(p), None, 0, None, 0)", PG_ERR_ARG),
    "pg_write_time_rows": ("L.pg_write_time_rows(C.byref(p), None, None, 1, 0)", PG_ERR_ARG),
    "pg_write_para_file": ("L.pg_write_para_file(None, None, None)", PG_ERR_ARG),
    "pg_create": ("L.pg_create(C.byref(p), 0, None)", PG_ERR_ARG),
    "pg_destroy": ("L.pg_destroy(None)", PG_OK),
    "pg_sync": ("L.pg_sync(None)", PG_ERR_ARG),
    "pg_load_rings": ("L.pg_load_rings(None, None, 0)", PG_ERR_ARG),
    "pg_load_dump": ("L.pg_load_dump(None, None)", PG_ERR_ARG),
    "pg_save_rings": ("L.pg_save_rings(None, None, 0)", PG_ERR_ARG),
    "pg_save_dump": ("L.pg_save_dump(None, None)", PG_ERR_ARG),
    "pg_get_dt": ("L.pg_get_dt(None, 0.1, 0.0, None)", PG_ERR_ARG),
    "pg_index_shift": ("L.pg_index_shift(None, 0.1, 0.0)", PG_ERR_ARG),
    "pg_sweep2d": ("L.pg_sweep2d(None, 0.1, None, 0.0)", PG_ERR_ARG),
    "pg_sweep3d": ("L.pg_sweep3d(None, 0.1, None, 0.0)", PG_ERR_ARG),
    "pg_sweep_axis": ("L.pg_sweep_axis(None, 0, 0.1, None, 0.0)", PG_ERR_ARG),
    "pg_rotate": ("L.pg_rotate(None)", PG_ERR_ARG),
    "pg_damp": ("L.pg_damp(None, 0.1)", PG_ERR_ARG),
    "pg_reduce": ("L.pg_reduce(None, None, 0.0, 0, None)", PG_ERR_ARG),
    "pg_init_planet": ("L.pg_init_planet(C.byref(p), None, None)", PG_ERR_ARG),
    "pg_planet_forces": ("L.pg_planet_forces(None, None, 0.0, 0.0)", PG_ERR_ARG),
    "pg_kick_drift_kick": ("L.pg_kick_drift_kick(None, None, None, 0.1, 0)", PG_ERR_ARG),
    "pg_clock_reset": ("L.pg_clock_reset(None, 0)", PG_ERR_ARG),
    "pg_clock_get": ("L.pg_clock_get(None, None, None)", PG_ERR_ARG),
    "pg_advance": ("L.pg_advance(None, 1, None)", PG_ERR_ARG),
    "pg_history": ("L.pg_history(None, None, 0, None)", PG_ERR_ARG),
    "pg_advance_graph": ("L.pg_advance_graph(None, 1, 1, None)", PG_ERR_ARG),
    "pg_device_view_get": ("L.pg_device_view_get(None, None)", PG_ERR_ARG),
    "pg_timing": ("L.pg_timing(None, 1)", PG_ERR_ARG),
    "pg_timing_read": ("L.pg_timing_read(None, None, None, 0)", PG_ERR_ARG),
    "pg_reduce_noalloc": ("L.pg_reduce_noalloc(None, 0, None, None, None, None, None, 0, 0, None, "
                          "0.0, 0, 0.0, 0.0, None, None)", PG_ERR_ARG),
    "pg_post_harmonic": ("L.pg_post_harmonic(None, 1.0, None, None)", PG_ERR_ARG),
    "pg_post_torque": ("L.pg_post_torque(None, 1.0, None)", PG_ERR_ARG),
    "pg_batch_create": ("L.pg_batch_create(0, None)", PG_ERR_ARG),
    "pg_batch_destroy": ("L.pg_batch_destroy(None)", PG_OK),
    "pg_batch_add": ("L.pg_batch_add(None, None)", PG_ERR_ARG),
    "pg_batch_remove": ("L.pg_batch_remove(None, None)", PG_ERR_ARG),
    "pg_batch_advance": ("L.pg_batch_advance(None, 1, 1)", PG_ERR_ARG),
    "pg_batch_sync": ("L.pg_batch_sync(None)", PG_ERR_ARG),
    "pg_batch_status": ("L.pg_batch_status(None, None, 0)", PG_ERR_ARG),
    "pg_batch_set_shape": ("L.pg_batch_set_shape(None, 0, None)", PG_ERR_ARG),
    "pg_batch_get_shape": ("L.pg_batch_get_shape(None, 0, None)", PG_ERR_ARG),
    "pg_batch_tune": ("L.pg_batch_tune(None, 1)", PG_ERR_ARG),
    "pg_server_create": ("L.pg_server_create(0, 0, 0, 0, 0, None)", PG_ERR_ARG),
    "pg_server_destroy": ("L.pg_server_destroy(None)", PG_OK),
    "pg_server_run_trace": ("L.pg_server_run_trace(None, None, None, None, 0, None)", PG_ERR_ARG),
    "pg_server_result": ("L.pg_server_result(None, 0, None, 0)", PG_ERR_ARG),
    "pg_server_batch": ("L.pg_server_batch(None, None)", PG_ERR_ARG),
    # no status to return: NaN, a count or size of 0, no stream, a message
    "pg_set_M_p": ("L.pg_set_M_p(None, 0.0)", "nan"),
    "pg_get_ecc": ("L.pg_get_ecc(None, 0.0)", "nan"),
    "pg_get_E": ("L.pg_get_E(None, 0.0)", "nan"),
    "pg_batch_size": ("L.pg_batch_size(None)", 0),
    "pg_launch_count": ("L.pg_launch_count(None)", 0),
    "pg_batch_launch_count": ("L.pg_batch_launch_count(None)", 0),
    "pg_server_rounds": ("L.pg_server_rounds(None)", 0),
    "pg_run_device_bytes": ("L.pg_run_device_bytes(None)", 0),
    "pg_ring_bytes": ("L.pg_ring_bytes(-1)", 0),
    "pg_batch_stream": ("L.pg_batch_stream(None)", None),
    "pg_last_error": ("L.pg_last_error(None)", "str"),
    "pg_batch_last_error": ("L.pg_batch_last_error(None)", "str"),
    "pg_server_last_error": ("L.pg_server_last_error(None)", "str"),
}

CHILD = """
import ctypes as C, json, math, sys
from penguin_2_0_b200 import _lib
L = _lib.lib()
p = _lib.pg_params()
assert L.pg_config_params(0, C.byref(p)) == 0
out = {}
for name, call in json.loads(sys.argv[1]).items():
    r = eval(call)
    if isinstance(r, float) and math.isnan(r):
        r = "nan"
    elif isinstance(r, bytes):
        r = "str" if r else ""
    out[name] = r
    print(json.dumps({name: r}), flush=True)
"""


def test_every_entry_point_refuses_null_arguments():
    calls = {k: v[0] for k, v in NULL_CALLS.items()}
    r = subprocess.run([sys.executable, "-c", CHILD, json.dumps(calls)], capture_output=True, text=True,
                       timeout=600)
    got = {}
    for line in r.stdout.splitlines():
        if line.startswith("{"):
            got.update(json.loads(line))
    assert r.returncode == 0, f"child died after {list(got)[-1:]}: {r.stderr[-2000:]}"
    want = {k: v[1] for k, v in NULL_CALLS.items()}
    assert got == want


def test_every_declared_entry_point_is_covered():
    exported = set(_lib.exported_symbols())
    assert exported - set(NULL_CALLS) == set()


def _p(**over):
    L = _lib.lib()
    p = _lib.pg_params()
    assert L.pg_config_params(0, C.byref(p)) == 0
    p.update(**over)
    return L, p


def test_undersized_buffers_are_refused():
    L, p = _p(imax=16, jmax=136)
    small = (C.c_char * 10)()
    assert L.pg_build_ic(C.byref(p), small, 10) == PG_ERR_ARG
    cnt = C.c_int(0)
    assert L.pg_boundary_rings(C.byref(p), None, 0, C.byref(cnt)) == PG_OK and cnt.value == 12
    few = (C.c_double * 5)(*([7.0] * 5))
    assert L.pg_boundary_rings(C.byref(p), few, 5, C.byref(cnt)) == PG_ERR_ARG
    assert list(few) == [7.0] * 5
    name = (C.c_char * 4)()
    assert L.pg_dump_name(C.byref(p), b"/tmp", 0, name, 4) == PG_ERR_ARG
    assert L.pg_label(C.byref(p), name, 2) == PG_ERR_ARG
    assert L.pg_write_time_rows(C.byref(p), b"/nonexistent-dir/t.dat", None, -1, 0) == PG_ERR_ARG
