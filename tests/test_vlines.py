"""Veto lines of a band (tdfstat_b200/vlines.py, mirroring common.c:155-553,
main.c:84-94 and vlinegen.c) against the reference's own veto-line
generator: the fixtures <name>.vlines hold the file the reference's
vlinegen program wrote for each case of VLINE_CASES (make_golden.py), and
the text written here must be the same, character for character.  The
search case g5_vlines (test_oracle, test_gpu_parity) checks that the lines
extracted here veto the triggers the reference vetoes."""
import dataclasses
import math
import os
import shutil
import tempfile

import numpy as np
import pytest

import refkit
from golden.cases import CASES, GOLDEN_DIR, VLINE_CASES, input_checksum
from tdfstat_b200 import host, synth, vlines


def _fixture(name):
    with open(os.path.join(GOLDEN_DIR, name + ".vlines"), encoding="latin-1") as f:
        first = f.readline()
        return first.split()[-1], f.read()


@pytest.fixture
def tmp():
    d = tempfile.mkdtemp(prefix="tdf_vl_")
    yield d
    shutil.rmtree(d, ignore_errors=True)


@pytest.mark.parametrize("name", sorted(VLINE_CASES))
def test_vlinegen_matches_reference_fixture(tmp, name):
    cks, text = _fixture(name)
    ini = synth.write_case(tmp, VLINE_CASES[name])
    assert input_checksum(tmp) == cks, "case inputs changed since the fixture was made"
    path = host.vlinegen(ini)
    with open(path, encoding="latin-1") as f:
        assert f.read() == text


@pytest.mark.skipif(not os.path.exists(refkit.REF_BIN["vlinegen"]), reason="reference vlinegen not built")
@pytest.mark.parametrize("name", sorted(VLINE_CASES))
def test_vlinegen_matches_reference_program(tmp, name):
    a, b = os.path.join(tmp, "a"), os.path.join(tmp, "b")
    ref = refkit.run_vlinegen(synth.write_case(a, VLINE_CASES[name]))
    with open(host.vlinegen(synth.write_case(b, VLINE_CASES[name])), encoding="latin-1") as f:
        assert f.read() == ref


def test_search_extracts_then_reads(tmp):
    """A search without a veto file extracts the lines, applies them with
    veto_flag and writes the file (main.c:93); the next search reads it
    (main.c:89) and gets the same intervals to the 15 decimals written."""
    case = CASES["g5_vlines"]
    ini = synth.write_case(tmp, case)
    job = host.Job(ini)
    _, text = _fixture("v1_band100")
    with open(job.vlines_file, encoding="latin-1") as f:
        assert f.read() == text
    nd = case.narrowdown * math.pi
    assert job.lines[:2] == vlines.narrow_down_lines(nd)
    assert job.vlines.nvlines_all_inband == 6 == job.numlines         # veto_flag = 1
    veto = job.lines[2:]
    assert veto == sorted(veto)                                         # lines_veto_fraction sorts them
    assert job.vlines.veto_fraction == pytest.approx(0.4380, abs=5e-5)
    again = host.Job(ini)
    assert again.numlines == 6
    np.testing.assert_allclose(sorted(again.lines[2:]), veto, rtol=0, atol=1e-15)
    o = again.search_opts()
    assert o.numlines == 6


def test_veto_flag_off_keeps_lines_out_of_the_search(tmp):
    case = dataclasses.replace(CASES["g5_vlines"], veto_flag=0)
    job = host.Job(synth.write_case(tmp, case))
    assert job.vlines.nvlines_all_inband == 6
    assert job.numlines == 2                  # the narrow-down intervals only
    case = VLINE_CASES["v2_band250"]          # narrowdown = pi/2: none at all
    job = host.Job(synth.write_case(os.path.join(tmp, "b"), case))
    assert job.numlines == 0 and job.vlines.nvlines_all_inband == 4
    assert job.vlines.veto_fraction == 1.0


def test_veto_fraction_of_overlapping_intervals():
    pi = math.pi
    vf, srt = vlines.lines_veto_fraction([[2.0, 2.5], [0.5, 1.0], [0.75, 1.25], [0.8, 0.9]])
    assert srt == [[0.5, 1.0], [0.75, 1.25], [0.8, 0.9], [2.0, 2.5]]
    assert vf == float(np.float32(float(np.float32(pi - (0.5 + 0.75 + (pi - 2.5)))) / pi))
    assert vlines.lines_veto_fraction([])[0] == 0.0
    assert vlines.lines_veto_fraction([[0.0, pi]])[0] == 1.0


def test_line_in_band_clips():
    assert vlines.line_in_band(99.9, 100.01, 100.0, 0.0625) == (100.0, 100.01)
    assert vlines.line_in_band(100.06, 100.2, 100.0, 0.0625) == (100.06, 100.0625)
    assert vlines.line_in_band(99.0, 99.99, 100.0, 0.0625) is None
    assert vlines.line_in_band(100.0625, 100.07, 100.0, 0.0625) == (100.0625, 100.0625)


def test_c_field_parsing(tmp):
    assert vlines.c_atof(" 1.5e1xyz") == 15.0 and vlines.c_atof("abc") == 0.0
    assert vlines.c_atoi(" -12.7") == -12 and vlines.c_atoi("x") == 0
    d = os.path.join(tmp, "in", "lines")
    os.makedirs(d)
    with open(os.path.join(d, "H1lines.csv"), "w") as f:
        f.write("% comment\n 1.0, 1, 0.5, 99, 100, 0.0, 0.0, white space\n"
                "2.0,,0,0,0,0,0,0.1,an empty field vanishes, as strtok drops it\n")
    vl = vlines.read_veto_files("in", ["H1", "L1"], base=tmp)
    assert [(v.f, v.type, v.offset, v.iharm1, v.iharm2, v.nline) for v in vl] == \
        [(1.0, 1, 0.5, 99, 100, 2), (2.0, 0, 0.0, 0, 0, 3)]
    assert vl[1].rwidth == 0.1 and vl[0].vfile == "in/lines/H1lines.csv"
    with open(os.path.join(d, "H1lines.csv"), "w") as f:
        f.write("1.0,0,0\n")
    with pytest.raises(vlines.VlinesError):
        vlines.read_veto_files("in", ["H1"], base=tmp)


def test_read_band_vlines_errors(tmp):
    p = os.path.join(tmp, "v.dat")
    with open(p, "w") as f:
        f.write("# header\n   0.5  0.75  100.01  100.015  x\n")
    with pytest.raises(vlines.VlinesError, match="veto fraction missing"):
        vlines.read_band_vlines(p, [], 1)
    with open(p, "a") as f:
        f.write("#band_veto_fraction= 0.0796\n")
    bv = vlines.read_band_vlines(p, [[0.0, 0.1]], 1)
    assert bv.lines == [[0.0, 0.1], [0.5, 0.75]] and bv.numlines_band == 2
    assert bv.veto_fraction == float(np.float32(0.0796))
    assert vlines.read_band_vlines(p, [[0.0, 0.1]], 0).numlines_band == 1
    with open(p, "a") as f:
        f.write("not a number\n")
    with pytest.raises(vlines.VlinesError, match="Can't parse line 4"):
        vlines.read_band_vlines(p, [], 1)
