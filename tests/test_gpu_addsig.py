"""Injection on the GPU (tdf_engine_add_signal) against the oracle's
restatement of add_signal (init.c:365-504), which the golden case g4_addsig
pins to the reference itself (test_oracle.py: the reference injects from its
signal file and searches; the oracle reproduces its records bit for bit).

The device computes sin/cos of ~1e8 rad phases with CUDA's double-precision
functions, which may differ from the host libm in the last bit; after the
sum is rounded to float a sample may differ by at most one float ulp, and
only rarely.  The records of the injected search are checked against the
reference by test_gpu_parity (g4_addsig is one of its cases).
"""
import ctypes as C

import numpy as np
import pytest

import refkit
from tdfstat_b200 import _abi
from tdfstat_b200.engine import Engine

pytestmark = pytest.mark.gpu


def _copy(sig):
    s = _abi.TdfSignal()
    C.memmove(C.byref(s), C.byref(sig), C.sizeof(sig))
    return s


def _check_xdat(eng, job, os_):
    N = job.sett.N
    for n in range(job.sett.nifo):
        xg = eng.xdat(n, N)
        xo = os_.xdat[n]
        diff = xg != xo
        ulp = np.spacing(np.abs(xo).astype(np.float32))
        assert np.all(np.abs(xg.astype(np.float64) - xo) <= ulp), "more than one float ulp apart"
        assert diff.sum() <= max(2, N // 10000), diff.sum()
        # the signal went where the data is nonzero, and only there
        x0 = np.asarray(job.dets[n].xdat, dtype=np.float32)
        assert np.all(xg[x0 == 0] == 0)
        assert (xg != x0).sum() > 0.9 * (x0 != 0).sum()


@pytest.mark.parametrize("form", ["split", "fp64"])
def test_device_injection_matches_oracle(golden, oracle, form):
    g = golden("g4_addsig")
    job = g.job if form == "fp64" else g.job32
    eng = Engine.from_job(job, form=form)
    h0, inband = eng.add_signal(job.signal)
    assert inband and h0 == job.signal.h0
    _check_xdat(eng, job, refkit.OracleSegment(job, oracle))
    eng.close()


def test_snr_form_matches_oracle(golden, oracle):
    g = golden("g4_addsig")
    job = g.job
    sig = _copy(job.signal)
    sig.h0, sig.snr = 0.0, 25.0
    keep = job.signal
    job.signal = sig
    try:
        os_ = refkit.OracleSegment(job, oracle)
        eng = Engine.from_job(job, form="fp64")
        h0, inband = eng.add_signal(sig)
        assert inband
        assert abs(h0 - os_.h0) <= 1e-12 * os_.h0, (h0, os_.h0)
        _check_xdat(eng, job, os_)
        eng.close()
    finally:
        job.signal = keep


def test_out_of_band_signal_adds_nothing(golden):
    g = golden("g4_addsig")
    job = g.job32
    sig = _copy(job.signal)
    sig.freq = job.sett.fpo - 0.5          # below the band (init.c:389-395)
    eng = Engine.from_job(job, form="split")
    h0, inband = eng.add_signal(sig)
    assert not inband
    for n in range(job.sett.nifo):
        np.testing.assert_array_equal(eng.xdat(n, job.sett.N), np.asarray(job.dets[n].xdat, dtype=np.float32))
    eng.close()


def test_upload_replaces_the_injection(golden):
    g = golden("g4_addsig")
    job = g.job32
    eng = Engine.from_job(job, form="split")
    eng.add_signal(job.signal)
    eng.upload(job.segment())
    np.testing.assert_array_equal(eng.xdat(0, job.sett.N), np.asarray(job.dets[0].xdat, dtype=np.float32))
    eng.close()


def test_write_signal_matches_reference(tmp_path):
    """mods=write_signal: Engine.inject writes the injected signal as the
    reference's FP64 build does (init.c:475-497).  CUDA's and libm's sin/cos
    of ~1e8-rad phases may differ in the last bit, which can move a "%e"
    value by one unit in its last digit, rarely."""
    import dataclasses
    import os
    from golden.cases import CASES
    from tdfstat_b200 import host, synth
    from tdfstat_b200.engine import TdfError
    case = dataclasses.replace(CASES["g4_addsig"], mods_extra="write_signal")
    ref = refkit.reference_signal_files(synth.write_case(str(tmp_path / "ref"), case))
    for form in ("fp64", "split"):
        job = host.Job(synth.write_case(str(tmp_path / form), case), float_build=(form == "split"))
        eng = Engine.from_job(job, form=form)
        h0, inband = eng.inject(job)
        assert inband and h0 == job.signal.h0
        d = os.path.join(job.outdir, "injections")
        assert sorted(os.listdir(d)) == sorted(ref)
        for fn in ref:
            with open(os.path.join(d, fn)) as f:
                mine = f.read().splitlines()
            theirs = ref[fn].splitlines()
            assert len(mine) == len(theirs) == job.sett.N
            diff = [k for k, (a, b) in enumerate(zip(mine, theirs)) if a != b]
            assert len(diff) <= 2, diff[:5]
            a = np.array([float(x) for x in mine])
            b = np.array([float(x) for x in theirs])
            assert np.all(np.abs(a - b) <= 1e-6 * np.abs(b) + 1e-300)
        # the engine reuses that memory: no signal is held after a search
        eng.search(*job.sky_points())
        with pytest.raises(TdfError):
            eng.signal(0, job.sett.N)
        eng.close()
