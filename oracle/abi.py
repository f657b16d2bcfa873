"""ctypes images of the two C-ABI structs the oracle takes (TEST
INFRASTRUCTURE ONLY): pg_params and pg_body of include/penguin_b200.h.

The oracle keeps its own copy so that a process can drive it (the timed CPU
baseline of bench.py, for one) without importing or loading the product
library; tests/test_oracle_cpu.py checks that the layout equals the
product's binding field for field.
"""
import ctypes as C


class pg_params(C.Structure):
    """include/penguin_b200.h pg_params (variable_types.h:11-20 + global.h:16-96)."""
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

    @classmethod
    def from_dict(cls, d: dict) -> "pg_params":
        """From {field: value}; floats may be hex strings (float.hex())."""
        p = cls()
        for k, v in d.items():
            if isinstance(v, str) and v.lstrip("-").startswith("0x"):
                v = float.fromhex(v)
            setattr(p, k, v)
        return p


class pg_body(C.Structure):
    """include/penguin_b200.h pg_body (struct body, variable_types.h:26-37)."""
    _fields_ = [(n, C.c_double) for n in ("m", "x", "y", "vx", "vy", "fx", "fy", "rs")]
