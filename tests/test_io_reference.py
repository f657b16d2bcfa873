"""Run label, dump names, para file and time-file rows against the reference's
own writers, byte for byte.

tests/golden/io_ref.json holds what the reference's create_label
(output.cu:57-88), dump naming with frame_num (main.cu:124, global.cu),
write_para_file (output.cu:90-109) and its time-file stream
(append_output_file, output.cu:25-34; the row of main.cu:417-427) produced on
the host for six flag sets (tests/golden/make_io_golden.py,
oracle/ref/io_harness.cu).  The library's pg_label, pg_dump_name,
pg_write_para_file and pg_write_time_rows must give the same text: a user's
post-processing (the reference's read/ tools, its scripts) finds the files
under the same names with the same contents."""
import json
import os

import pytest

import penguin_2_0_b200 as pg
from tests._golden import HERE  # puts tests/golden on sys.path
from make_io_golden import IO_CASES, io_params  # noqa: E402

G = json.load(open(os.path.join(HERE, "golden", "io_ref.json")))
MAINP = G["mainp"]
ROW = [float.fromhex(v) for v in G["row_values"]]
FRAMES = (0, 7, 42, 1234, 99999)


@pytest.mark.parametrize("case", list(IO_CASES))
def test_label_matches_reference(case):
    assert pg.label(io_params(case)) == G["cases"][case]["label.txt"]


@pytest.mark.parametrize("case", list(IO_CASES))
def test_dump_names_match_reference(case):
    p = io_params(case)
    want = G["cases"][case]["frames.txt"].splitlines()
    assert [pg.dump_name(p, MAINP + "/binary", n) for n in FRAMES] == want


@pytest.mark.parametrize("case", list(IO_CASES))
def test_para_file_matches_reference(case, tmp_path):
    path = str(tmp_path / "para.dat")
    pg.write_para_file(io_params(case), path, MAINP)
    assert open(path).read() == G["cases"][case]["para.dat"]


@pytest.mark.parametrize("case", list(IO_CASES))
def test_time_rows_match_reference(case, tmp_path):
    p = io_params(case)
    path = str(tmp_path / "time.dat")
    pg.write_time_rows(p, path, [ROW])
    want = G["cases"][case]["time.dat"]
    assert open(path).read() == want
    # appending adds rows after the existing ones, as the reference's
    # append_output_file does on a restart
    pg.write_time_rows(p, path, [ROW, ROW], append=True)
    assert open(path).read() == want * 3
