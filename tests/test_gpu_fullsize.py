"""Parity at the benchmark sizes: cfg1 (H1 alone, float64 input read as
mods=read_O3, N = 86164), cfg2 (H1L1, N = 86164, nfftf = 2^17) and cfg3
(N = 258492, nfftf = 2^18), through checks the FP64 oracle finishes in
seconds:
  * F spectra of single templates (first and last spindown of two sky points)
    against orc_fstat_spectrum,
  * the records of one sky point x 21 spindowns against orc_search_points,
  * the injected signal (cfg2, cfg3) is the loudest trigger over all 401
    spindowns of the sky point nearest to it.
Tolerances as in test_gpu_parity: FP64 form 1e-10, split form 1e-4
(normalised F error), identical triggers up to threshold/neighbour ties.
"""
import ctypes as C
import shutil
import tempfile

import numpy as np
import pytest

import refkit
from tdfstat_b200 import host
from tdfstat_b200.engine import Engine
from tdfstat_b200.workloads import Workload

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-10, "split": 1e-4}


@pytest.fixture(scope="module")
def workload():
    made = {}

    def get(name):
        if name not in made:
            root = tempfile.mkdtemp(prefix="tdf_full_")
            wl = Workload(name, root)
            # the FP64 (PREC=DOUBLE) reading of the same inputs, same ranges
            j64 = host.Job(wl.ini, float_build=False)
            j64.range.fr = list(wl.job.range.fr)
            j64.sett.bufsize = wl.job.sett.bufsize
            made[name] = (wl, j64, root)
        return made[name][:2]

    yield get
    for _, _, root in made.values():
        shutil.rmtree(root, ignore_errors=True)


def _job(wl, j64, form):
    return j64 if form == "fp64" else wl.job


@pytest.mark.parametrize("form", ["split", "fp64"])
@pytest.mark.parametrize("name", ["cfg1", "cfg2", "cfg3"])
def test_fullsize_spectrum_matches_oracle(workload, oracle, name, form):
    wl, j64 = workload(name)
    seg, opts = j64.segment(), j64.search_opts()
    eng = Engine.from_job(_job(wl, j64, form), form=form)
    for ip in (0, wl.centre):   # a corner of the patch and its centre
        res = eng.search(wl.pm[ip:ip + 1], wl.mm[ip:ip + 1], wl.nn[ip:ip + 1])
        assert len(res) == wl.nspd
        for r in (0, len(res) - 1):
            m, n, s = (float(v) for v in res.hdr[r, :3])
            Fg = eng.fstat(int(wl.pm[ip]), m, n, s)
            Fo = np.zeros_like(Fg)
            st = oracle.orc_fstat_spectrum(C.byref(seg), C.byref(opts), int(wl.pm[ip]), m, n, s,
                                           Fo.ctypes.data_as(C.POINTER(C.c_double)), len(Fo))
            assert st == 0
            err = np.max(np.abs(Fg - Fo) / np.maximum(Fo, 1.0))
            print(name, form, ip, r, "max normalised F err %.3g" % err)
            assert err <= TOL[form], err
    eng.close()


@pytest.mark.parametrize("form", ["split", "fp64"])
@pytest.mark.parametrize("name", ["cfg1", "cfg2", "cfg3"])
def test_fullsize_records_match_oracle(workload, oracle, name, form):
    wl, j64 = workload(name)
    seg, opts = j64.segment(), j64.search_opts()
    ip = wl.centre
    pm, mm, nn = wl.pm[ip:ip + 1], wl.mm[ip:ip + 1], wl.nn[ip:ip + 1]
    sst = np.array([opts.spndr[1] - 20], dtype=np.float32)   # the last 21 spindowns
    eng = Engine.from_job(_job(wl, j64, form), form=form)
    res = eng.search(pm, mm, nn, sst=sst)
    rec = refkit.Records(res.hdr, res.pairs, np.repeat(pm, res.per_point))
    st, ref, _ = refkit.search_points(oracle.orc_search_points, seg, opts, pm, mm, nn, sst=sst)
    assert st == 0 and len(ref) == 21 == len(rec)
    r = refkit.compare_records(rec, ref, f_rtol=2e-6 if form == "split" else 1e-12, F_rtol=TOL[form],
                               thr=float(opts.thr), tie_band=TOL[form])
    print(name, form, {k: v for k, v in r.items() if k != "unmatched"})
    assert not r["unmatched"], r["unmatched"][:10]
    assert r["max_F_rel"] <= TOL[form], r["max_F_rel"]
    assert r["matched"] > 0
    assert r["only_a"] + r["only_b"] <= max(2, 0.002 * r["matched"])
    eng.close()


@pytest.mark.parametrize("name", ["cfg2", "cfg3"])
def test_fullsize_injection_is_loudest(workload, name):
    wl, _ = workload(name)
    ip = wl.centre   # the grid point of the injection
    eng = Engine.from_job(wl.job, form="split")
    res = eng.search(wl.pm[ip:ip + 1], wl.mm[ip:ip + 1], wl.nn[ip:ip + 1])
    assert len(res) == wl.nspd
    allp = np.concatenate([p for p in res.pairs if len(p)]).reshape(-1, 2)
    fbest, Fbest = allp[np.argmax(allp[:, 1])]
    st = wl.job.sett
    f_hz = st.fpo + fbest / np.pi * st.B
    inj = wl.case.injections[0]
    bin_hz = st.B * 2 / st.nfftf
    print(name, "loudest F %.1f at %.6f Hz (injected %.6f Hz, bin %.2e Hz)" % (Fbest, f_hz, inj.f, bin_hz))
    assert Fbest > 40
    assert abs(f_hz - inj.f) < 50 * bin_hz
    eng.close()


def test_trigger_buffer_grows_and_reruns(workload, oracle):
    """More triggers in one batch than the device trigger buffer holds
    (2^21 at first): at thr = 0.5 one cfg2 sky point gives ~21k triggers per
    spindown, 121 spindowns ~2.5M.  The engine grows the buffer and reruns
    the batch; records against the FP64 oracle at the same threshold."""
    wl, j64 = workload("cfg2")
    seg, opts = j64.segment(), j64.search_opts()
    opts.thr = 0.5
    ip = wl.centre
    pm, mm, nn = wl.pm[ip:ip + 1], wl.mm[ip:ip + 1], wl.nn[ip:ip + 1]
    sst = np.array([opts.spndr[1] - 120], dtype=np.float32)
    eng = Engine(seg, opts, form="fp64")
    res = eng.search(pm, mm, nn, sst=sst)
    eng.close()
    assert len(res) == 121 and res.ntrig > (1 << 21)
    rec = refkit.Records(res.hdr, res.pairs, np.repeat(pm, res.per_point))
    st, ref, _ = refkit.search_points(oracle.orc_search_points, seg, opts, pm, mm, nn, sst=sst,
                                      max_pairs=res.pairs_flat.size + (1 << 20))
    assert st == 0 and len(ref) == 121
    r = refkit.compare_records(rec, ref, f_rtol=1e-12, F_rtol=TOL["fp64"], thr=0.5, tie_band=TOL["fp64"])
    assert not r["unmatched"], r["unmatched"][:10]
    assert r["max_F_rel"] <= TOL["fp64"], r["max_F_rel"]
    assert r["only_a"] + r["only_b"] <= 2
