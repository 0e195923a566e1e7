"""Coincidences between segments (tdf_coincidences) against the reference's
own coincidence program (coincidences/coincidences.c, compiled unmodified by
oracle/Makefile with its HDF5 I/O replaced by oracle/coinc_io.c) on golden
case c1_4seg: four segments searched by the reference, its coincidences
stored per shift.  Here the segments' records come from the oracle (which
reproduces the reference's records bit for bit), so the comparison is exact:
every coincidence, its members and the per-shift segment counts.  Runs on
the host; tdf_coincidences needs no device."""
import os
import shutil
import tempfile

import numpy as np
import pytest

import refkit
from golden.cases import COINC_CASES, GOLDEN_DIR, input_checksum, write_coinc_case
from tdfstat_b200 import host
from tdfstat_b200.coinc import CoincOptions, Segment, coincidences


class CoincGolden:
    def __init__(self, name):
        self.cc = COINC_CASES[name]
        self.root = tempfile.mkdtemp(prefix="tdf_" + name + "_")
        self.segs = write_coinc_case(self.root, name)
        self.checksum = input_checksum(self.root)
        self.fix = np.load(os.path.join(GOLDEN_DIR, name + ".npz"))
        self.jobs = {seg: host.Job(ini, float_build=False) for seg, ini in self.segs}
        self.jobs32 = {seg: host.Job(ini, float_build=True) for seg, ini in self.segs}

    def points(self, job):
        pm, mm, nn = (np.asarray(v) for v in job.sky_points())
        keep = pm == self.cc["hemi"]
        return pm[keep], mm[keep], nn[keep]

    def segment(self, seg, job, hdr, pairs):
        return Segment(seg=seg, N=job.sett.N, nfftf=job.sett.nfftf, dt=job.sett.dt, narrowdown=job.narrowdown,
                       hdr=hdr, pairs=pairs, lines=np.zeros((len(job.lines), 2)))

    def expected(self, key, ish):
        p = "%s_%02d_" % (key, ish)
        f = self.fix
        return f[p + "seginfo"], f[p + "w"], f[p + "vals"], f[p + "cseg"], f[p + "trig"], f[p + "ntrig"]

    def close(self):
        shutil.rmtree(self.root, ignore_errors=True)


@pytest.fixture(scope="module")
def c1():
    g = CoincGolden("c1_4seg")
    yield g
    g.close()


def compare(g, key, got, seginfo, exact=True, rtol=0.0):
    """got: coincidences of all 16 shifts; returns the number compared."""
    n = 0
    for ish in range(16):
        si, w, vals, cseg, trig, ntrig = g.expected(key, ish)
        mine = [c for c in got if c.shift == ish]
        np.testing.assert_array_equal(seginfo[ish], si)
        assert len(mine) == len(w), (ish, len(mine), len(w))
        m = 0
        for k, c in enumerate(mine):
            assert c.w == w[k]
            got_v = np.array([c.avg_snr, c.avg_f, c.avg_fdot, c.avg_ra, c.avg_dec], dtype=np.float32)
            if exact:
                np.testing.assert_array_equal(got_v, vals[k])
            else:
                np.testing.assert_allclose(got_v, vals[k], rtol=rtol)
            np.testing.assert_array_equal(c.cseg, cseg[m:m + c.w])
            np.testing.assert_array_equal(c.trig, trig[m:m + c.w])
            np.testing.assert_array_equal(c.ntrig, ntrig[m:m + c.w])
            m += c.w
        n += len(mine)
    return n


def test_inputs_regenerate_identically(c1):
    assert c1.checksum == str(c1.fix["checksum"])


@pytest.mark.parametrize("threads", ["1", "3", None])
@pytest.mark.parametrize("key", ["a", "b"])
def test_coincidences_match_reference_bit_for_bit(c1, oracle, key, threads, monkeypatch):
    """The 16 shifts run on TDF_COINC_THREADS host threads (default: all);
    the result is the reference's for any thread count."""
    if threads is None:
        monkeypatch.delenv("TDF_COINC_THREADS", raising=False)
    else:
        monkeypatch.setenv("TDF_COINC_THREADS", threads)
    segs = []
    for seg, _ in c1.segs:
        job = c1.jobs[seg]
        pm, mm, nn = c1.points(job)
        st, rec, per = refkit.search_points(oracle.orc_search_points, job.segment(), job.search_opts(), pm, mm, nn)
        assert st == 0
        segs.append(c1.segment(seg, job, rec.hdr, rec.pairs))
    got, seginfo = coincidences(CoincOptions(**c1.cc["opts"][key]), segs)
    n = compare(c1, key, got, seginfo)
    assert n > 1000
    # the injected signal is the leading coincidence of shift 0: all four segments
    top = [c for c in got if c.shift == 0][0]
    assert top.w == 4
    st = c1.jobs[1].sett
    assert abs(st.fpo + top.avg_f / np.pi * st.B - c1.cc["base"].injections[0].f) < 1e-3


def test_single_shift_and_capacity(c1, oracle):
    import ctypes as C
    from tdfstat_b200 import _abi
    from tdfstat_b200.engine import load_library
    segs = []
    for seg, _ in c1.segs:
        job = c1.jobs[seg]
        pm, mm, nn = c1.points(job)
        st, rec, per = refkit.search_points(oracle.orc_search_points, job.segment(), job.search_opts(), pm, mm, nn)
        segs.append(c1.segment(seg, job, rec.hdr, rec.pairs))
    opts = dict(c1.cc["opts"]["a"])
    got, seginfo = coincidences(CoincOptions(shift=5, **opts), segs)
    si, w, vals, cseg, trig, ntrig = c1.expected("a", 5)
    assert all(c.shift == 5 for c in got) and len(got) == len(w)
    np.testing.assert_array_equal(seginfo[0], si)
    # invalid options are refused
    lib = load_library()
    o = _abi.TdfCoincOpts(1, 7.0, 0, 1, 1, 1, 2, -1)
    n1, n2 = C.c_int64(0), C.c_int64(0)
    assert lib.tdf_coincidences(C.byref(o), 0, None, None, 0, C.byref(n1), None, None, None, 0, C.byref(n2),
                                None) == _abi.TDF_ERR_INVALID
