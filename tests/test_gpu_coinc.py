"""Coincidences of GPU searches: the four segments of golden case c1_4seg
searched by libtdfcuda, then tdf_coincidences, against the reference's
coincidence program run on the reference's own searches (the fixture).

FP64 form: the records equal the reference's, so every coincidence and its
members must match (values to float rounding).  Split form: F differs from
the reference by ~1e-6, which can swap which of two nearly equal triggers is
the loudest of a cell; at least 99% of the coincidences must have the
reference's members, 98% also its values (1e-4), the leading three of every
shift in order, and the counts stay within 1%."""
import numpy as np
import pytest

from tdfstat_b200.coinc import CoincOptions, coincidences
from tdfstat_b200.engine import Engine
from test_coinc import CoincGolden, compare

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c1():
    g = CoincGolden("c1_4seg")
    yield g
    g.close()


def _gpu_segments(g, form):
    segs = []
    for seg, _ in g.segs:
        job = g.jobs[seg] if form == "fp64" else g.jobs32[seg]
        pm, mm, nn = g.points(job)
        eng = Engine.from_job(job, form=form)
        res = eng.search(pm, mm, nn)
        eng.close()
        segs.append(g.segment(seg, job, res.hdr, res.pairs))
    return segs


@pytest.mark.parametrize("key", ["a", "b"])
def test_fp64_gpu_coincidences_match_reference(c1, key):
    segs = _gpu_segments(c1, "fp64")
    got, seginfo = coincidences(CoincOptions(**c1.cc["opts"][key]), segs)
    assert compare(c1, key, got, seginfo, exact=False, rtol=1e-6) > 1000


def test_split_gpu_coincidences_close_to_reference(c1):
    """Every shift: the count within 1%, at least 99% of the reference's
    coincidences found with the same members (segments and template
    numbers), at least 98% also with the reference's average SNR and
    frequency (1e-4), and the leading three in the same order."""
    segs = _gpu_segments(c1, "split")
    got, seginfo = coincidences(CoincOptions(**c1.cc["opts"]["a"]), segs)
    total = same = same_v = 0
    for ish in range(16):
        si, w, vals, cseg, trig, ntrig = c1.expected("a", ish)
        mine = [c for c in got if c.shift == ish]
        assert abs(len(mine) - len(w)) <= max(2, 0.01 * len(w))
        # the same members (segment, template) can form several
        # coincidences (other frequency cells): the reference's values per
        # member set, each used once
        ref = {}
        m = 0
        for k in range(len(w)):
            key = tuple(zip(cseg[m:m + w[k]].tolist(), trig[m:m + w[k]].tolist()))
            ref.setdefault(key, []).append(np.asarray(vals[k][:2], dtype=np.float64))
            m += int(w[k])
        for c in mine:
            key = tuple(zip(np.asarray(c.cseg).tolist(), np.asarray(c.trig).tolist()))
            if key in ref and ref[key]:
                same += 1
                got_v = np.array([c.avg_snr, c.avg_f], dtype=np.float64)
                for i, rv in enumerate(ref[key]):
                    if np.allclose(got_v, rv, rtol=1e-4, atol=0):
                        same_v += 1
                        del ref[key][i]
                        break
        total += len(w)
        for k in range(min(3, len(w))):     # the leading coincidences, in order
            c = mine[k]
            assert c.w == w[k]
            np.testing.assert_allclose([c.avg_snr, c.avg_f], vals[k][:2], rtol=1e-4)
            m = int(np.sum(w[:k]))
            np.testing.assert_array_equal(c.trig, trig[m:m + c.w])
    print("split-form coincidences with the reference's members: %d of %d, of them %d with its average SNR and "
          "frequency (1e-4)" % (same, total, same_v))
    assert same >= 0.99 * total
    assert same_v >= 0.98 * total
