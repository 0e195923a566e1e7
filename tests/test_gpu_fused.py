"""The fused spindown passes against the two-launch path.

With N1 = N2 (nfftf = 2^16: 256 x 256, and 2^18: 512 x 512) the column and
row pass of a chunk run as one ordered launch, k_spinpass: CTAs take tickets,
a template's row blocks follow its column blocks by `lag` templates and wait
(bounded) until all of them have stored their spectra.  The arithmetic is the
two passes' own, in the same order, so the records must equal those of the
two launches (TDF_FUSED_PASSES=0) bit for bit: for chunk sizes that do and do
not divide the template count, lags from 1 to past the chunk, both F
stores (sparse default, full with TDF_FULL_F=1), and an F range past
nfftf/2 (whole rows kept)."""
import shutil
import tempfile

import numpy as np
import pytest

from tdfstat_b200 import synth
from tdfstat_b200.engine import Engine
from tdfstat_b200.workloads import Workload

pytestmark = pytest.mark.gpu


def _day1():
    """H1+L1, one day at dt = 2 s: N = 43082, nfft = nfftf = 2^16."""
    inj = synth.Injection(f=100.1234, fdot=-3e-10, ra=4.0, dec=0.9, iota=0.9, psi=0.4, phase=2.2, snr=12.0)
    case = synth.Case(dt=2.0, nod=1, band=360, dets=("H1", "L1"), seed=606, thr=11.0, fdot_step=1e-10,
                      sky_cells=16.0, injections=(inj,))
    return case, (4, 4), 401, 0.25


@pytest.fixture(scope="module", params=["cfg3", "day1"])
def wl(request):
    root = tempfile.mkdtemp(prefix="tdf_fused_")
    w = Workload(request.param, root, case=_day1() if request.param == "day1" else None)
    yield w
    shutil.rmtree(root, ignore_errors=True)


def _search(w, monkeypatch, fused, tc, lag=3, full_f=False):
    monkeypatch.setenv("TDF_FUSED_PASSES", "1" if fused else "0")
    monkeypatch.setenv("TDF_TEMPLATES_PER_CHUNK", str(tc))
    monkeypatch.setenv("TDF_FUSE_LAG", str(lag))
    monkeypatch.setenv("TDF_FULL_F", "1" if full_f else "0")
    eng = Engine.from_job(w.job, form="split")
    pm, mm, nn = w.patch(4)
    res = eng.search(pm, mm, nn)
    out = (res.hdr.copy(), [p.copy() for p in res.pairs], res.per_point.copy())
    n = eng.launch_count()
    eng.close()
    return out, n


def _same(a, b):
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[2], b[2])
    assert len(a[1]) == len(b[1])
    for x, y in zip(a[1], b[1]):
        np.testing.assert_array_equal(x, y)


@pytest.mark.parametrize("tc,lag", [(48, 3), (7, 1), (96, 5), (20, 200)])
def test_fused_passes_match_two_launches(wl, monkeypatch, tc, lag):
    two, n_two = _search(wl, monkeypatch, False, tc)
    one, n_one = _search(wl, monkeypatch, True, tc, lag)
    assert wl.job.sett.nfftf in (1 << 16, 1 << 18)
    assert n_one < n_two     # the fused launch ran: one launch per chunk instead of two
    assert sum(len(p) for p in two[1]) > 0
    _same(one, two)


def test_fused_passes_full_f_store(wl, monkeypatch):
    two, _ = _search(wl, monkeypatch, False, 32, full_f=True)
    one, _ = _search(wl, monkeypatch, True, 32, full_f=True)
    _same(one, two)


def test_fused_passes_whole_rows(wl, monkeypatch):
    """An F range reaching past nfftf/2: the row blocks keep every output of
    their rows (no half-row pruning)."""
    fr = list(wl.job.range.fr)
    try:
        wl.job.range.fr = [fr[0], wl.job.sett.nfftf // 2 + 4096]
        two, _ = _search(wl, monkeypatch, False, 32)
        one, _ = _search(wl, monkeypatch, True, 32)
    finally:
        wl.job.range.fr = fr
    assert sum(len(p) for p in two[1]) > 0
    _same(one, two)
