"""Short chunks packed several per CTA give the same bits as one per CTA.

A radial pencil's last chunk of at most 64 cells runs 4 adjacent columns per
CTA, and a polar pencil that is a single chunk (nk + 12 <= 56 cells) runs 8
per CTA (nk + 12 <= 44: whole warps) or 4, by default; PG_POLAR_PACK=0 runs
one per 32/64-thread CTA.  A CTA past the last column computes its padding
pencils without storing them.  The cell arithmetic
is the same device body either way, so the results must be bitwise equal."""
import numpy as np
import pytest

import penguin_2_0_b200 as pg

CASES = [
    dict(which=0, imax=256, jmax=384),                        # radial last chunk: 24 + 12 cells
    dict(which=0, imax=136, jmax=408, precision=1),          # 20 + 12, FP32
    dict(which=1, imax=128, jmax=132, kmax=16),               # radial 12 + 12, polar 16 + 12
    dict(which=1, imax=64, jmax=132, kmax=24),                # single radial chunk, polar 24 + 12
    dict(which=1, imax=63, jmax=132, kmax=32),                # polar 32 + 12, 8316 pencils: 4 padding
    dict(which=1, imax=64, jmax=132, kmax=40),                # polar 40 + 12: 4 pencils per CTA
    dict(which=1, imax=64, jmax=132, kmax=16, precision=1),   # FP32 3D
]


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
def test_packed_short_chunks_are_bitwise(gpu, monkeypatch, case):
    c = dict(case)
    p = pg.params(c.pop("which"), nprin=1, **c)
    ic = pg.build_ic(p)
    out = {}
    for pack in ("0", "4"):
        monkeypatch.setenv("PG_POLAR_PACK", pack)
        with pg.Run(p, 0) as r:
            r.load(ic)
            r.clock_reset(0)
            r.advance(4)
            out[pack] = pg.dump_fields(r.save(), p)
    for k in ("r", "u", "v", "w", "rot_j"):
        np.testing.assert_array_equal(out["4"][k], out["0"][k], err_msg=k)


RADIAL_CASES = [
    dict(which=0, imax=256, jmax=384),                        # 2 full radial chunks per column + packed last chunk
    dict(which=0, imax=252, jmax=390),                        # jmax not a multiple of 4: padding columns
    dict(which=1, imax=128, jmax=132, kmax=16),               # 3D
    dict(which=0, imax=232, jmax=200),                        # imax % 116 == 0: stuck last chunk
    dict(which=0, imax=200, jmax=300),                        # last chunk 84 + 12 cells in the full chunks' launch
    dict(which=0, imax=256, jmax=391, precision=1),           # FP32 (1 or 2 columns), an odd column count
    dict(which=0, imax=200, jmax=300, precision=1),           # FP32, last chunk in the full chunks' launch
    dict(which=1, imax=128, jmax=132, kmax=16, precision=1),  # FP32 3D
]


@pytest.mark.gpu
@pytest.mark.parametrize("case", RADIAL_CASES)
def test_radial_column_packing_is_bitwise(gpu, monkeypatch, case):
    """Full radial chunks run one column per CTA, or 2 or 4 adjacent columns
    per CTA (PG_RADIAL_PACK; FP32 runs take 1 or 2 and one column for 4):
    the same device body per cell, so the results must be bitwise equal."""
    c = dict(case)
    p = pg.params(c.pop("which"), nprin=1, **c)
    ic = pg.build_ic(p)
    out = {}
    for pack in ("1", "2", "4"):
        monkeypatch.setenv("PG_RADIAL_PACK", pack)
        with pg.Run(p, 0) as r:
            r.load(ic)
            r.clock_reset(0)
            r.advance(4)
            out[pack] = pg.dump_fields(r.save(), p)
    for pack in ("2", "4"):
        for k in ("r", "u", "v", "w", "rot_j"):
            np.testing.assert_array_equal(out[pack][k], out["1"][k], err_msg=f"{k} pack {pack}")
