"""Host-side checks that need no GPU: the C ABI library loads and exports
every symbol include/penguin_b200.h declares, parameter validation, the
seeded initial condition and the dump layout."""
import ctypes as C
import subprocess

import numpy as np
import pytest

import penguin_2_0_b200 as pg
from penguin_2_0_b200 import _lib


def test_library_exports_every_header_symbol():
    names = _lib.exported_symbols()
    assert len(names) >= 30
    L = _lib.lib()
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    for n in names:
        assert f" T {n}" in out, n


def test_ring_bytes_matches_reference_layout():
    # sizeof(hydr_ring) = 72*jmax + 96 (144,096 at jmax = 2000)
    assert pg.host.ring_bytes(2000) == 144096
    assert pg.host.ring_bytes(768) == 72 * 768 + 96


def test_default_params_are_global_h():
    p = pg.params(None)
    assert (p.imax, p.jmax, p.kmax, p.ndim) == (850, 2000, 1, 2)
    assert p.p_alpha == 1.5 and p.p_beta == 0.5 and p.ss_alpha == 1e-4 and p.sc_h == 0.05
    assert p.plnt_flag == 2 and p.FARGO_flag == 1 and p.flat_flag == 1 and p.courant == 0.5


@pytest.mark.parametrize("over,ok", [
    (dict(), True),
    (dict(EOS=1), False),
    (dict(bary_flag=1), False),
    (dict(jmax=116 * 3 + 3), False),     # azimuthal wrap would read updated cells
    (dict(jmax=116 * 3), True),          # last chunk idle, reproduced
    (dict(jmax=120), False),             # single chunk: r_rg read before written
    (dict(imax=116 * 2 + 2), True),      # radial remainder 1..5 is fine
    (dict(kmax=4), False),               # 2D with kmax > 1
    (dict(nlft=0), False),
])
def test_check_params(over, ok):
    p = pg.params(0, **over)
    st = pg.host.check_params(p)
    assert (st == 0) == ok, (over, st)


def test_ic_is_seeded_and_consistent():
    p = pg.params(0, imax=130, jmax=240)
    a, b = pg.build_ic(p), pg.build_ic(p)
    assert bytes(a) == bytes(b)
    p2 = pg.params(0, imax=130, jmax=240, seed=7)
    c = pg.build_ic(p2)
    assert bytes(a) != bytes(c)
    f = pg.dump_fields(a, p)
    # Sigma = r^-1 (1 +- 1e-4), v_r = 0, w = 0, rot_j = 0, ring-major indices
    sig0 = f["xc"][:, None] ** -1.0
    dev = f["r"] / sig0 - 1.0
    assert np.all(np.abs(dev) <= 1e-4 * (1 + 1e-12))
    assert np.std(dev) > 3e-5
    assert np.all(f["u"] == 0.0) and np.all(f["w"] == 0.0)
    assert np.all(f["rot_j"] == 0) and np.all(f["i"] == np.arange(130))
    # EOS-0 invariant p = Sigma * h^2 r^-p_beta
    np.testing.assert_allclose(f["p"], f["r"] * (0.05 ** 2) / f["xc"][:, None], rtol=2e-16 * 8)
    # log grid in r (grid.cu lg=1), uniform phi
    assert f["x"][0] == 0.4
    np.testing.assert_allclose(f["x"][1:] / f["x"][:-1], (2.5 / 0.4) ** (1 / 130), rtol=1e-12)


def test_label_matches_create_label():
    p = pg.params(0)
    assert pg.label(p) == "256x768x1_c50_p333_s60_i40_o250_a10_b10_rot_fargo"


def test_dump_name_and_time_file(tmp_path):
    import ctypes as C
    p = pg.params(0)
    L = _lib.lib()
    b = C.create_string_buffer(512)
    assert L.pg_dump_name(C.byref(p), b"binary", 7, b, 512) == 0
    assert b.value.decode() == "binary/binary_256x768x1_c50_p333_s60_i40_o250_a10_b10_rot_fargo_00007"
    rows = np.arange(22, dtype=np.float64).reshape(2, 11) + 0.5
    path = str(tmp_path / "time.dat")
    assert L.pg_write_time_rows(path.encode(), rows.ctypes.data_as(C.POINTER(C.c_double)), 2, 0) == 0
    back = np.loadtxt(path)
    np.testing.assert_array_equal(back, rows)
    assert open(path).readline().startswith("0.5 1.5 2.5")
