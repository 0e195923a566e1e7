"""Parity at the benchmark configurations test_gpu_fullsize does not cover,
and against the reference build itself at benchmark sizes.

  * The two intermediate segment sizes of the batched workload: nod 3
    (N = 129246, nfft = nfftf = 2^17, Ninterp = 2^18; 1.01 FFT points per
    sample) and nod 4 (N = 172328, nfft = nfftf = 2^18, Ninterp = 2^19; 1.52),
    whose four-step splits and zero-padded tails differ from the 2- and
    6-day segments.
  * The scale configuration: N = 258492, sigma 1.0 (H1) / 1.3 (L1), 10% of
    the samples zeroed in gaps, 801 spindowns.
  For each: F spectra of the first and last spindown of two sky points
  against orc_fstat_spectrum, and the records of one sky point x 21
  spindowns against orc_search_points (the FP64 restatement, pinned bit for
  bit to the reference's FP64 build on the golden cases).
  * A 15-point x 401-spindown patch of the 2-day H1L1 segment (~6000
    templates) and a 1% sample of the scale configuration's 1024-point patch
    (11 points x 801 spindowns) against the reference's own FP64 build
    (oracle/_ref/gwsearch-ref-f64, its unmodified sources) run on the host
    cores on the same INI: the same records, the same trigger set up to
    threshold ties, F within the form's tolerance (jobcore.c:552-603 trigger
    selection).
Tolerances: FP64 form 1e-10, split form 1e-4 (normalised F error).
"""
import ctypes as C
import os
import shutil
import tempfile

import numpy as np
import pytest

import refkit
from tdfstat_b200 import host, synth
from tdfstat_b200.engine import Engine
from tdfstat_b200.workloads import Workload, workload_case

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-10, "split": 1e-4}
# cfg4:2 is the batched workload's nod 3 segment, cfg4:3 its nod 4 segment
NAMES = ["cfg4:2", "cfg4:3", "cfg5"]


@pytest.fixture(scope="module")
def workload():
    made = {}

    def get(name):
        if name not in made:
            root = tempfile.mkdtemp(prefix="tdf_cfg_")
            wl = Workload(name, root)
            j64 = host.Job(wl.ini, float_build=False)
            j64.range.fr = list(wl.job.range.fr)
            j64.sett.bufsize = wl.job.sett.bufsize
            made[name] = (wl, j64, root)
        return made[name][:2]

    yield get
    for _, _, root in made.values():
        shutil.rmtree(root, ignore_errors=True)


def test_configuration_sizes(workload):
    """The segments are the sizes the configurations name."""
    want = {"cfg4:2": (129246, 131072, 131072, 262144, 401), "cfg4:3": (172328, 262144, 262144, 524288, 401),
            "cfg5": (258492, 262144, 262144, 524288, 801)}
    for name, (N, nfft, nfftf, ninterp, nspd) in want.items():
        wl, _ = workload(name)
        s = wl.job.sett
        assert (s.N, s.nfft, s.nfftf, s.Ninterp, wl.nspd) == (N, nfft, nfftf, ninterp, nspd), name
    wl, _ = workload("cfg5")
    x0 = np.asarray(wl.job.dets[0].xdat)
    x1 = np.asarray(wl.job.dets[1].xdat)
    assert 0.08 < np.mean(x0 == 0) < 0.12      # 10% gaps
    assert abs(np.std(x1[x1 != 0]) / np.std(x0[x0 != 0]) - 1.3) < 0.02   # sigma 1.3 on L1, 1.0 on H1


@pytest.mark.parametrize("form", ["split", "fp64"])
@pytest.mark.parametrize("name", NAMES)
def test_config_spectrum_matches_oracle(workload, oracle, name, form):
    wl, j64 = workload(name)
    seg, opts = j64.segment(), j64.search_opts()
    eng = Engine.from_job(j64 if form == "fp64" else wl.job, form=form)
    for ip in (0, wl.centre):
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
@pytest.mark.parametrize("name", NAMES)
def test_config_records_match_oracle(workload, oracle, name, form):
    wl, j64 = workload(name)
    seg, opts = j64.segment(), j64.search_opts()
    ip = wl.centre
    pm, mm, nn = wl.pm[ip:ip + 1], wl.mm[ip:ip + 1], wl.nn[ip:ip + 1]
    sst = np.array([opts.spndr[1] - 20], dtype=np.float32)   # the last 21 spindowns
    eng = Engine.from_job(j64 if form == "fp64" else wl.job, form=form)
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


def _reference_patch(name, g, step, root):
    """The workload's segment with a directed_range grid of 2g+1 sky points
    along nn (step in grid cells) around the first injection, x the
    workload's spindowns, F over the all-sky range; written as the
    reference's input tree.  Returns the INI path and the spindown count."""
    case, _, nspd, _ = workload_case(name)
    inj = case.injections[0]
    st = case.settings()
    case.gtype = "directed_range"
    case.gcenter = (st.fpo + st.B / 2, inj.fdot, inj.ra, inj.dec)
    case.gsizes = (st.nfft // 4 - 1024, float((nspd - 1) // 2), 0.0, g * step)
    case.gsteps = (1, 1.0, 1.0, step)
    return synth.write_case(root, case), nspd


@pytest.fixture(scope="module")
def reference_runs():
    """The reference FP64 build run once per patch (all host threads)."""
    made = {}

    def get(name, g, step):
        key = (name, g, step)
        if key not in made:
            if not os.path.exists(refkit.REF_BIN["f64"]):
                pytest.skip("reference build oracle/_ref/gwsearch-ref-f64 not present")
            root = tempfile.mkdtemp(prefix="tdf_refpatch_")
            ini, nspd = _reference_patch(name, g, step, root)
            ref, meta, _ = refkit.run_reference(ini, "f64", threads=os.cpu_count() or 1, timeout=1800)
            made[key] = (ini, ref, meta, nspd, root)
        return made[key][:4]

    yield get
    for v in made.values():
        shutil.rmtree(v[4], ignore_errors=True)


@pytest.mark.parametrize("form", ["split", "fp64"])
@pytest.mark.parametrize("name,g,step", [("cfg2", 7, 0.25), ("cfg5", 5, 0.1)])
def test_patch_matches_reference_build(reference_runs, name, g, step, form):
    """Many sky points at a benchmark configuration: the GPU's records
    against the reference build's own, on the same INI (the same grid,
    ranges and point enumeration)."""
    ini, ref, meta, nspd = reference_runs(name, g, step)
    job = host.Job(ini, float_build=(form == "split"))
    pm, mm, nn = job.sky_points()
    assert len(pm) >= 2 * g   # 2g+1 up to the float rounding of the range's ends
    eng = Engine.from_job(job, form=form)
    res = eng.search(pm, mm, nn)
    eng.close()
    rec = refkit.Records(res.hdr, res.pairs, np.repeat(pm, res.per_point))
    assert len(rec) == len(ref) == len(pm) * nspd
    np.testing.assert_array_equal(rec.pm, ref.pm)
    if form == "fp64":
        np.testing.assert_array_equal(rec.hdr, ref.hdr)
    r = refkit.compare_records(rec, ref, f_rtol=2e-6 if form == "split" else 1e-12, F_rtol=TOL[form],
                               thr=float(job.search_opts().thr), tie_band=TOL[form])
    print(name, form, "reference walltime %.1f s on %s threads," % (meta["walltime"], meta.get("num_threads")),
          "%d triggers (GPU %d)," % (ref.ntrig, rec.ntrig), {k: v for k, v in r.items() if k != "unmatched"})
    assert not r["unmatched"], r["unmatched"][:10]
    assert r["max_F_rel"] <= TOL[form], r["max_F_rel"]
    assert r["matched"] > 0
    assert r["only_a"] + r["only_b"] <= max(2, 0.002 * r["matched"])
    # trigger counts agree except for threshold ties
    assert abs(rec.ntrig - ref.ntrig) <= r["only_a"] + r["only_b"]
