"""GPU parity: libtdfcuda (through its C ABI) against the reference's own
records (golden fixtures) and the FP64 restatement oracle.

Tolerances:
  FP64 form  : F relative error <= 1e-10, identical trigger set
  split form : F relative error <= 1e-4, identical trigger set except
               triggers whose F lies within 1e-4 (relative) of thr or of a
               neighbouring bin (threshold and local-maximum ties)
F-spectrum error is normalised per bin by max(F_ref, 1): F of pure noise has
mean 2, so this is the relative error wherever F is not close to zero.
"""
import numpy as np
import pytest

import refkit
from golden.cases import CASES

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-10, "split": 1e-4}


def _engine(job, form, **kw):
    # the case's signal file (g4) injected on the device, as main.c does on the host
    return refkit.engine_for(job, form=form, **kw)


def _match(rec, ref, form, thr):
    F_rtol = TOL[form]
    return refkit.compare_records(rec, ref, f_rtol=2e-6 if form == "split" else 1e-12,
                                  F_rtol=F_rtol, thr=thr, tie_band=F_rtol)


def _as_records(res, pm):
    return refkit.Records(res.hdr, res.pairs, np.repeat(np.asarray(pm, np.int32), res.per_point))


@pytest.mark.parametrize("form", ["fp64", "split"])
@pytest.mark.parametrize("name", sorted(CASES))
def test_records_match_reference(golden, name, form):
    g = golden(name)
    job = g.job if form == "fp64" else g.job32
    pm, mm, nn = job.sky_points()
    eng = _engine(job, form)
    res = eng.search(pm, mm, nn)
    rec = _as_records(res, pm)
    ref = g.ref["f64"]
    assert len(rec) == len(ref)
    np.testing.assert_array_equal(rec.pm, ref.pm)
    np.testing.assert_array_equal(rec.hdr[:, :3], ref.hdr[:, :3])
    if form == "fp64":
        np.testing.assert_array_equal(rec.hdr, ref.hdr)
    else:
        np.testing.assert_allclose(rec.hdr, g.ref["f32"].hdr, rtol=1e-6)
    r = _match(rec, ref, form, g.case.thr)
    print(name, form, {k: v for k, v in r.items() if k != "unmatched"})
    assert not r["unmatched"], r["unmatched"][:10]
    assert r["max_F_rel"] <= TOL[form], r["max_F_rel"]
    # tie-explained differences must stay rare
    assert r["only_a"] + r["only_b"] <= max(2, 0.002 * r["matched"])
    eng.close()


@pytest.mark.parametrize("form", ["fp64", "split"])
@pytest.mark.parametrize("name", sorted(CASES))
def test_fstat_spectrum_matches_oracle(golden, oracle, name, form):
    import ctypes as C
    g = golden(name)
    job = g.job
    os_ = refkit.OracleSegment(job, oracle)
    seg, opts = os_.seg, job.search_opts()
    pm, mm, nn = job.sky_points()
    ref = g.ref["f64"]
    eng = _engine(g.job if form == "fp64" else g.job32, form)
    # first and last template of the run
    for r in (0, len(ref) - 1):
        m, n, s = (float(v) for v in ref.hdr[r, :3])
        p = int(ref.pm[r])
        Fg = eng.fstat(p, m, n, s)
        Fo = np.zeros_like(Fg)
        st = oracle.orc_fstat_spectrum(C.byref(seg), C.byref(opts), p, m, n, s,
                                       Fo.ctypes.data_as(C.POINTER(C.c_double)), len(Fo))
        assert st == 0
        err = np.max(np.abs(Fg - Fo) / np.maximum(Fo, 1.0))
        print(name, form, r, "max normalised F err", err)
        assert err <= TOL[form], err
    eng.close()


def test_outside_ellipse_and_empty(golden):
    g = golden("g1_h1_directed")
    eng = _engine(g.job, "split")
    res = eng.search([1], [1e4], [1e4])
    assert len(res) == 0 and res.per_point[0] == 0
    res = eng.search([], [], [])
    assert len(res) == 0
    eng.close()


def test_trigger_overflow_is_an_error(golden):
    from tdfstat_b200.engine import Engine, TdfError
    g = golden("g1_h1_directed")
    opts = g.job.search_opts()
    opts.bufsize = 8
    eng = Engine(g.job.segment(), opts, form="split")
    pm, mm, nn = g.job.sky_points()
    with pytest.raises(TdfError) as ei:
        eng.search(pm, mm, nn)
    assert ei.value.status == 3
    # the engine stays usable after the error
    opts2 = g.job.search_opts()
    eng2 = Engine(g.job.segment(), opts2, form="split")
    assert len(eng2.search(pm, mm, nn)) == len(g.ref["f64"])
    eng.close()
    eng2.close()


def test_restart_spindown(golden, oracle):
    """s_range->sst: the first point starts at a later spindown (restart
    from a checkpoint, jobcore.c:208)."""
    g = golden("g1_h1_directed")
    pm, mm, nn = g.job.sky_points()
    sst = [g.job.range.spndr[0] + 3.0]
    eng = _engine(g.job, "fp64")
    res = eng.search(pm, mm, nn, sst=sst)
    st, orc, per = refkit.search_points(oracle.orc_search_points, g.job.segment(), g.job.search_opts(),
                                        pm, mm, nn, sst=sst)
    assert st == 0 and len(res) == len(orc) == len(g.ref["f64"]) - 3
    r = _match(_as_records(res, pm), orc, "fp64", g.case.thr)
    assert not r["unmatched"] and r["max_F_rel"] <= 1e-10
    eng.close()


def test_device_only_counts(golden):
    g = golden("g2_h1l1_inj")
    pm, mm, nn = g.job32.sky_points()
    eng = _engine(g.job32, "split")
    nrec, ntrig = eng.search_device(pm, mm, nn)
    res = eng.search(pm, mm, nn)
    assert nrec == len(res) and ntrig == res.ntrig
    assert eng.launch_count() > 0
    eng.close()


def test_injection_recovered(golden):
    """The injected signal of g2 (network SNR 40) is the loudest trigger, at
    the injected frequency within a few bins."""
    g = golden("g2_h1l1_inj")
    pm, mm, nn = g.job32.sky_points()
    eng = _engine(g.job32, "split")
    res = eng.search(pm, mm, nn)
    allp = np.concatenate([p for p in res.pairs if len(p)]).reshape(-1, 2)
    fbest, Fbest = allp[np.argmax(allp[:, 1])]
    st = g.job.sett
    f_hz = st.fpo + fbest / np.pi * st.B
    inj = g.case.injections[0]
    assert Fbest > 200
    assert abs(f_hz - inj.f) < 5 * st.B * 2 / st.nfftf * 10
    eng.close()


@pytest.mark.parametrize("form", ["fp64", "split"])
@pytest.mark.parametrize("variant", ["hemi1", "label", "usedet_H1", "overlap"])
def test_option_variants_match_reference(tmp_path, variant, form):
    """The option variants of test_host_options (one hemisphere, a label,
    usedet selecting one detector, a band overlap) through the GPU engine
    against the reference's own FP64 run."""
    import os
    from tdfstat_b200 import host, synth
    from test_host_options import _case
    case, usedet = _case(variant)
    ini = synth.write_case(str(tmp_path), case)
    if usedet:
        with open(ini) as f:
            text = f.read()
        with open(ini, "w") as f:
            f.write(text.replace("usedet = %s" % "".join(case.dets), "usedet = %s" % usedet))
    if not os.path.exists(refkit.REF_BIN["f64"]):
        pytest.skip("reference build not present")
    ref, _, _ = refkit.run_reference(ini, "f64", threads=1)
    job = host.Job(ini, float_build=(form == "split"))
    pm, mm, nn = job.sky_points()
    eng = _engine(job, form)
    rec = _as_records(eng.search(pm, mm, nn), pm)
    assert len(rec) == len(ref) > 0
    np.testing.assert_array_equal(rec.pm, ref.pm)
    np.testing.assert_array_equal(rec.hdr[:, :3], ref.hdr[:, :3])
    r = _match(rec, ref, form, case.thr)
    assert not r["unmatched"], r["unmatched"][:10]
    assert r["max_F_rel"] <= TOL[form], r["max_F_rel"]
    assert r["only_a"] + r["only_b"] <= max(2, 0.002 * r["matched"])
    eng.close()


@pytest.mark.parametrize("form", ["fp64", "split"])
def test_candidate_overflow_falls_back_to_full_scan(golden, oracle, form):
    """At thr = 0.5 about 90% of the bins are candidates (F of noise is
    chi^2_4 / 2), more than the 64 x 4096 entries of a lane's candidate list
    for every full group of 64 templates: the row pass stops appending and
    k_resolve scans every bin instead.  Records against the oracle at the
    same threshold."""
    g = golden("g2_h1l1_inj")
    job = g.job if form == "fp64" else g.job32
    seg = job.segment()
    opts = job.search_opts()
    opts.thr = 0.5
    pm, mm, nn = job.sky_points()
    from tdfstat_b200.engine import Engine
    eng = Engine(seg, opts, form=form)
    rec = _as_records(eng.search(pm, mm, nn), pm)
    eng.close()
    oseg, oopts = g.job.segment(), g.job.search_opts()
    oopts.thr = 0.5
    st, ref, _ = refkit.search_points(oracle.orc_search_points, oseg, oopts, pm, mm, nn)
    assert st == 0 and len(rec) == len(ref) > 64
    assert ref.ntrig > 100 * len(ref)          # the candidate lists overflowed
    r = _match(rec, ref, form, 0.5)
    assert not r["unmatched"], r["unmatched"][:10]
    assert r["max_F_rel"] <= TOL[form], r["max_F_rel"]
    assert r["only_a"] + r["only_b"] <= max(2, 0.002 * r["matched"])
