"""Host-side checks that need no GPU: the C ABI library loads and exports
every symbol include/penguin_b200.h declares, parameter validation, the
seeded initial condition and the dump layout."""
import ctypes as C
import os
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


def test_ctypes_signatures_match_header_parameter_counts():
    """Every declaration in include/penguin_b200.h has ctypes argtypes with
    as many parameters (a mismatch would pass arguments in the wrong slots)."""
    import re
    txt = open(os.path.join(os.path.dirname(_lib.LIB_PATH), "..", "include", "penguin_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    decls = re.findall(r"\b(pg_[a-z0-9_]+)\s*\(([^;{]*?)\)\s*;", txt, flags=re.S)
    assert len(decls) == len(_lib.exported_symbols())
    L = _lib.lib()
    for name, args in decls:
        a = args.strip()
        n = 0 if a in ("", "void") else len(a.split(","))
        at = getattr(L, name).argtypes
        assert at is not None and len(at) == n, (name, n, at)


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
    (dict(EOS=1, gam=1.4), True),        # isentropic (riemann.cu:75-111)
    (dict(EOS=1, gam=1.0), True),        # 2D isentropic at gam 1
    (dict(EOS=2, gam=1.4), False),       # energy equation: marked buggy by the reference
    (dict(EOS=1, gam=1.4, precision=1), False),  # FP32 planes: EOS 0 only
    (dict(EOS=0, gam=0.9), False),
    (dict(bary_flag=1), False),
    (dict(jmax=116 * 3 + 3), False),     # azimuthal wrap would read updated cells
    (dict(jmax=116 * 3), True),          # last chunk idle, reproduced
    (dict(jmax=120), False),             # single chunk: r_rg read before written
    (dict(imax=116 * 2 + 2), True),      # radial remainder 1..5 is fine
    (dict(kmax=4), False),               # 2D with kmax > 1
    (dict(nlft=0), False),
    (dict(imax=65535), True),            # rings on CUDA grid y: at most 65535
    (dict(imax=65536), False),
    (dict(jmax=116 * 600), True),        # 2D: jmax is not on a grid y
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
    # EOS 1 names gamma instead of the temperature slope (output.cu:72-79)
    assert pg.label(pg.params(0, EOS=1, gam=1.4)) == "256x768x1_c50_p333_s60_i40_o250_a10_g14_rot_fargo"


def test_3d_isentropic_needs_gam_above_one():
    assert pg.host.check_params(pg.params(1, EOS=1, gam=1.0)) != 0
    assert pg.host.check_params(pg.params(1, EOS=1, gam=5.0 / 3.0)) == 0


def test_3d_polar_columns_fit_cuda_grid_y():
    assert pg.host.check_params(pg.params(1, jmax=116 * 564)) == 0      # 65424
    assert pg.host.check_params(pg.params(1, jmax=116 * 565)) != 0      # 65540


def test_isentropic_ic_pressure_and_profile():
    # p = cs2 Sigma^gam / gam (the EOS-1 store, ppm.cu:140-141); the 2D
    # surface density keeps its r^-p_alpha slope (disk_profile.cu:9-28) and
    # v_phi^2 = 1/r + r dP/dr / Sigma with the isentropic P(r)
    gam = 1.4
    p = pg.params(0, imax=130, jmax=240, EOS=1, gam=gam)
    f = pg.dump_fields(pg.build_ic(p), p)
    cs2 = 0.05 ** 2 / f["xc"][:, None]
    np.testing.assert_allclose(f["p"], cs2 * f["r"] ** gam / gam, rtol=1e-15)
    dev = f["r"] / f["xc"][:, None] ** -1.0 - 1.0
    assert np.all(np.abs(dev) <= 1e-4 * (1 + 1e-12))
    r = f["xc"]
    P = lambda x: 0.05 ** 2 / x * (x ** -1.0) ** gam / gam
    dP = (P(r + 1.27245e-8) - P(r - 1.27245e-8)) / 2.5449e-8
    vk = np.sqrt(1.0 / r + r * dP / r ** -1.0)
    # the centred difference over 2.5e-8 turns last-ulp pow differences
    # (numpy vs libm) into ~1e-11 of v_phi
    np.testing.assert_allclose(f["v"][:, 0], vk, rtol=1e-10)
    # differs from the isothermal disk's rotation
    f0 = pg.dump_fields(pg.build_ic(pg.params(0, imax=130, jmax=240)), p)
    assert np.max(np.abs(f0["v"][:, 0] / f["v"][:, 0] - 1.0)) > 1e-5


def test_isentropic_3d_ic_is_the_polytrope():
    # rho(r, z)^(gam-1) = rho_mid^(gam-1) - (gam-1)/(r cs2) (1 - r/sqrt(r^2+z^2))
    # below z_0, continued above z_0 by a decade per h/6 (disk_profile.cu:86-103),
    # with rho_mid ~ r^(-p_alpha 2/(gam+1))
    gam = 5.0 / 3.0
    p = pg.params(1, imax=64, jmax=132, kmax=16, EOS=1, gam=gam)
    f = pg.dump_fields(pg.build_ic(p), p)
    nr, nk = p.imax, p.kmax
    sig = f["r"].reshape(nk, nr, -1)
    xc = f["xc"].reshape(nk, nr)[0]
    zc = f["zc"].reshape(nk, nr)[:, 0]
    gm = gam - 1.0
    below = above = 0
    for k in range(nk):
        R = xc * np.sin(zc[k])
        Z = xc * np.cos(zc[k])
        c2 = 0.05 ** 2 * R ** -1.0
        h = np.sqrt(c2 * R ** 3)
        z0 = np.sqrt(2 * h * h * R ** (-1.5 * (2 / (gam + 1)) * gm) / gm)
        mid = R ** (-1.5 * 2 / (gam + 1))
        poly = lambda zz: (mid ** gm - gm / (R * c2) * (1 - R / np.sqrt(R * R + zz * zz))) ** (1 / gm)
        want = np.where(Z < z0, poly(np.minimum(Z, z0)), 10.0 ** (np.log10(poly(z0)) - 6.0 * (Z - z0) / h))
        below += int(np.sum(Z < z0))
        above += int(np.sum(Z >= z0))
        np.testing.assert_allclose(sig[k, :, 0], want, rtol=1.1e-4)   # the seeded noise is 1e-4
    assert below > 0 and above > 0


def test_write_ic_file_equals_build_ic_bytes(tmp_path):
    """pg_write_ic writes the restart file binary_<label>_00000 that the
    reference's restart path reads (main.cu:246-262): the same bytes as
    pg_build_ic, ring after ring in the dump layout."""
    for which, over in ((0, dict(imax=64, jmax=132)), (1, dict(imax=32, jmax=132, kmax=8))):
        p = pg.params(which, **over)
        path = str(tmp_path / f"ic_{which}.bin")
        assert _lib.lib().pg_write_ic(C.byref(p), path.encode()) == 0
        assert open(path, "rb").read() == bytes(pg.build_ic(p))
