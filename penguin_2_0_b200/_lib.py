"""ctypes binding of libpenguin_b200.so (the C ABI in include/penguin_b200.h).

The shared library is built in-tree by ``penguin_2_0_b200/build.py``; loading
fails loudly when it is missing -- there is no Python or CPU fallback for the
hydro step.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpenguin_b200.so")

PG_OK = 0
STATUS = {
    0: "PG_OK", 1: "PG_ERR_CUDA", 2: "PG_ERR_PARAMS", 3: "PG_ERR_NONFINITE",
    4: "PG_ERR_DT_COLLAPSE", 5: "PG_ERR_TIMEOUT", 6: "PG_ERR_IO", 7: "PG_ERR_STATE",
    8: "PG_ERR_NOMEM", 9: "PG_ERR_ARG",
}


class pg_params(C.Structure):
    """Runtime image of variable_types.h:11-20 + global.h:16-96."""
    _fields_ = [
        ("ndim", C.c_int), ("imax", C.c_int), ("jmax", C.c_int), ("kmax", C.c_int),
        ("flat_flag", C.c_int), ("bary_flag", C.c_int), ("EOS", C.c_int), ("plnt_flag", C.c_int),
        ("FrRot_flag", C.c_int), ("kill_flag", C.c_int),
        ("visc_flag", C.c_int), ("FARGO_flag", C.c_int), ("dump_flag", C.c_int),
        ("p_alpha", C.c_double), ("p_beta", C.c_double), ("ss_alpha", C.c_double),
        ("sc_h", C.c_double), ("Sigma_0", C.c_double),
        ("M_p", C.c_double), ("R_p", C.c_double), ("t_growth", C.c_double), ("rs_fac", C.c_double),
        ("gam", C.c_double), ("courant", C.c_double),
        ("nlft", C.c_int), ("nrgh", C.c_int), ("nudr", C.c_int), ("ntop", C.c_int),
        ("endtime", C.c_double), ("tmovie", C.c_double),
        ("ncycend", C.c_int), ("nprin", C.c_int),
        ("xmin", C.c_double), ("xmax", C.c_double), ("ymin", C.c_double), ("ymax", C.c_double),
        ("zmin", C.c_double), ("zmax", C.c_double),
        ("ngeomx", C.c_int), ("ngeomy", C.c_int), ("ngeomz", C.c_int),
        ("grspx", C.c_int), ("grspy", C.c_int), ("grspz", C.c_int),
        ("dx_min", C.c_double), ("dx_max", C.c_double), ("dy_min", C.c_double),
        ("dy_max", C.c_double), ("dz_min", C.c_double), ("dz_max", C.c_double),
        ("seed", C.c_uint64), ("noise_amp", C.c_double),
        ("kill_rin", C.c_double), ("kill_rout", C.c_double),
        ("precision", C.c_int), ("reserved", C.c_int * 7),
    ]

    def as_dict(self) -> dict:
        out = {}
        for name, _ in self._fields_:
            if name == "reserved":
                continue
            out[name] = getattr(self, name)
        return out

    def update(self, **kw) -> "pg_params":
        for k, v in kw.items():
            if not hasattr(self, k):
                raise KeyError(k)
            setattr(self, k, v)
        return self


class pg_body(C.Structure):
    """struct body (variable_types.h:26-37)."""
    _fields_ = [(n, C.c_double) for n in ("m", "x", "y", "vx", "vy", "fx", "fy", "rs")]


class pg_clock(C.Structure):
    _fields_ = [
        ("simtime", C.c_double), ("timem", C.c_double), ("dt", C.c_double),
        ("dt_used", C.c_double), ("frrot", C.c_double), ("ncycle", C.c_int64),
        ("make_pict", C.c_int), ("done", C.c_int), ("status", C.c_int), ("pad", C.c_int),
    ]


class pg_device_view(C.Structure):
    _fields_ = [
        ("sigma", C.c_void_p), ("vr", C.c_void_p), ("vphi", C.c_void_p),
        ("row_stride", C.c_int64), ("slab_stride", C.c_int64), ("imax", C.c_int), ("jmax", C.c_int), ("kmax", C.c_int),
        ("elem_bytes", C.c_int), ("stream", C.c_void_p),
    ]


class pg_batch_member(C.Structure):
    _fields_ = [("halted", C.c_int), ("status", C.c_int), ("ncycle", C.c_int64), ("simtime", C.c_double)]


class pg_batch_shape(C.Structure):
    _fields_ = [("grid_x", C.c_int), ("grid_y", C.c_int), ("minb", C.c_int), ("pad", C.c_int)]


class pg_completion(C.Structure):
    _fields_ = [("id", C.c_int64), ("arrival_s", C.c_double), ("admit_s", C.c_double), ("finish_s", C.c_double),
                ("steps", C.c_int64), ("cells", C.c_int64), ("simtime", C.c_double), ("status", C.c_int),
                ("pad", C.c_int)]


_lib = None


def lib() -> C.CDLL:
    """Load libpenguin_b200.so once; raise if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is missing: run `python -c 'import __graft_entry__ as g; g.build()'` "
            "(there is no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    P, B = C.POINTER(pg_params), C.POINTER(pg_body)
    vp, dp, ip = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int)
    sigs = {
        "pg_default_params": (C.c_int, [P]),
        "pg_config_params": (C.c_int, [C.c_int, P]),
        "pg_check_params": (C.c_int, [P]),
        "pg_ring_bytes": (C.c_size_t, [C.c_int]),
        "pg_write_ic": (C.c_int, [P, C.c_char_p]),
        "pg_build_ic": (C.c_int, [P, vp, C.c_size_t]),
        "pg_boundary_rings": (C.c_int, [P, C.POINTER(C.c_double), C.c_size_t, C.POINTER(C.c_int)]),
        "pg_label": (C.c_int, [P, C.c_char_p, C.c_size_t]),
        "pg_dump_name": (C.c_int, [P, C.c_char_p, C.c_int, C.c_char_p, C.c_size_t]),
        "pg_write_time_rows": (C.c_int, [P, C.c_char_p, dp, C.c_int, C.c_int]),
        "pg_params_set": (C.c_int, [P, C.c_char_p, C.c_double]),
        "pg_params_get": (C.c_int, [P, C.c_char_p, dp]),
        "pg_write_para_file": (C.c_int, [P, C.c_char_p, C.c_char_p]),
        "pg_create": (C.c_int, [P, C.c_int, C.POINTER(vp)]),
        "pg_destroy": (C.c_int, [vp]),
        "pg_last_error": (C.c_char_p, [vp]),
        "pg_sync": (C.c_int, [vp]),
        "pg_load_rings": (C.c_int, [vp, vp, C.c_size_t]),
        "pg_load_dump": (C.c_int, [vp, C.c_char_p]),
        "pg_save_rings": (C.c_int, [vp, vp, C.c_size_t]),
        "pg_save_dump": (C.c_int, [vp, C.c_char_p]),
        "pg_get_dt": (C.c_int, [vp, C.c_double, C.c_double, dp]),
        "pg_index_shift": (C.c_int, [vp, C.c_double, C.c_double]),
        "pg_sweep2d": (C.c_int, [vp, C.c_double, B, C.c_double]),
        "pg_sweep3d": (C.c_int, [vp, C.c_double, B, C.c_double]),
        "pg_damp": (C.c_int, [vp, C.c_double]),
        "pg_sweep_axis": (C.c_int, [vp, C.c_int, C.c_double, B, C.c_double]),
        "pg_rotate": (C.c_int, [vp]),
        "pg_reduce": (C.c_int, [vp, B, C.c_double, C.c_int, dp]),
        "pg_init_planet": (C.c_int, [P, B, dp]),
        "pg_set_M_p": (C.c_double, [P, C.c_double]),
        "pg_planet_forces": (C.c_int, [vp, B, C.c_double, C.c_double]),
        "pg_kick_drift_kick": (C.c_int, [P, B, dp, C.c_double, C.c_int]),
        "pg_get_ecc": (C.c_double, [B, C.c_double]),
        "pg_get_E": (C.c_double, [B, C.c_double]),
        "pg_clock_reset": (C.c_int, [vp, C.c_int]),
        "pg_clock_get": (C.c_int, [vp, C.POINTER(pg_clock), B]),
        "pg_advance": (C.c_int, [vp, C.c_int, ip]),
        "pg_advance_graph": (C.c_int, [vp, C.c_int, C.c_int, ip]),
        "pg_history": (C.c_int, [vp, dp, C.c_int, ip]),
        "pg_device_view_get": (C.c_int, [vp, C.POINTER(pg_device_view)]),
        "pg_launch_count": (C.c_int64, [vp]),
        "pg_timing": (C.c_int, [vp, C.c_int]),
        "pg_timing_read": (C.c_int, [vp, dp, C.POINTER(C.c_int64), C.c_int]),
        "pg_reduce_noalloc": (C.c_int, [vp, C.c_int64, vp, vp, vp, vp, vp, C.c_int, C.c_int, B,
                                        C.c_double, C.c_int, C.c_double, C.c_double, vp, vp]),
        "pg_batch_create": (C.c_int, [C.c_int, C.POINTER(vp)]),
        "pg_batch_destroy": (C.c_int, [vp]),
        "pg_batch_last_error": (C.c_char_p, [vp]),
        "pg_batch_add": (C.c_int, [vp, vp]),
        "pg_batch_remove": (C.c_int, [vp, vp]),
        "pg_batch_size": (C.c_int, [vp]),
        "pg_batch_advance": (C.c_int, [vp, C.c_int, C.c_int]),
        "pg_batch_sync": (C.c_int, [vp]),
        "pg_batch_status": (C.c_int, [vp, C.POINTER(pg_batch_member), C.c_int]),
        "pg_batch_set_shape": (C.c_int, [vp, C.c_int, C.POINTER(pg_batch_shape)]),
        "pg_batch_get_shape": (C.c_int, [vp, C.c_int, C.POINTER(pg_batch_shape)]),
        "pg_batch_tune": (C.c_int, [vp, C.c_int]),
        "pg_batch_launch_count": (C.c_int64, [vp]),
        "pg_batch_stream": (vp, [vp]),
        "pg_run_device_bytes": (C.c_size_t, [P]),
        "pg_post_harmonic": (C.c_int, [vp, C.c_double, dp, dp]),
        "pg_post_torque": (C.c_int, [vp, C.c_double, dp]),
        "pg_server_create": (C.c_int, [C.c_int, C.c_size_t, C.c_int, C.c_int, C.c_int, C.POINTER(vp)]),
        "pg_server_destroy": (C.c_int, [vp]),
        "pg_server_last_error": (C.c_char_p, [vp]),
        "pg_server_run_trace": (C.c_int, [vp, P, dp, C.POINTER(C.c_int64), C.c_int, C.POINTER(pg_completion)]),
        "pg_server_result": (C.c_int, [vp, C.c_int64, vp, C.c_size_t]),
        "pg_server_rounds": (C.c_int64, [vp]),
        "pg_server_batch": (C.c_int, [vp, C.POINTER(vp)]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(L, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def exported_symbols() -> list[str]:
    """Names declared in include/*.h (parsed from the header text)."""
    import re
    inc = os.path.join(os.path.dirname(_HERE), "include")
    names = []
    for fn in sorted(os.listdir(inc)):
        if not fn.endswith(".h"):
            continue
        txt = open(os.path.join(inc, fn)).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        for m in re.finditer(r"\b(pg_[a-z0-9_]+)\s*\(", txt):
            names.append(m.group(1))
    return sorted(set(names))
