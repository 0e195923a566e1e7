"""CPU tests of the checker itself: the FFT core against numpy.fft, the spline
against scipy's natural cubic spline, and the C restatement of job_core()
(fed by the host mirror) against the reference's own outputs stored in the
golden fixtures."""
import ctypes as C

import numpy as np
import pytest

import refkit
from golden.cases import CASES


@pytest.mark.parametrize("n", [8, 64, 4096, 1 << 15])
@pytest.mark.parametrize("sign", [-1, 1])
def test_fft_core_matches_numpy(oracle, n, sign):
    rng = np.random.default_rng(n)
    x = (rng.normal(size=n) + 1j * rng.normal(size=n)).astype(np.complex128)
    out = np.zeros_like(x)
    assert oracle.orc_fft(n, sign, x.ctypes.data, out.ctypes.data) == 0
    ref = np.fft.fft(x) if sign < 0 else np.fft.ifft(x) * n
    err = np.abs(out - ref).max() / np.abs(ref).max()
    assert err < 1e-13, err


def test_fft_core_rejects_non_power_of_two(oracle):
    x = np.zeros(12, np.complex128)
    assert oracle.orc_fft(12, -1, x.ctypes.data, x.ctypes.data) != 0


def test_splintpad_matches_natural_cubic_spline(oracle):
    from scipy.interpolate import CubicSpline
    rng = np.random.default_rng(5)
    N, pad = 500, 2
    n = pad * N
    ya = (rng.normal(size=n) + 1j * rng.normal(size=n)).astype(np.complex128)
    shftf = rng.uniform(-3, 3, size=N)
    shftf[0] = 0.0
    out = np.zeros(N, np.complex128)
    oracle.orc_splintpad(ya.ctypes.data, shftf.ctypes.data_as(C.POINTER(C.c_double)), N, pad, out.ctypes.data)
    xs = np.arange(n, dtype=np.float64)
    cr = CubicSpline(xs, ya.real, bc_type="natural")
    ci = CubicSpline(xs, ya.imag, bc_type="natural")
    x = pad * (np.arange(N) - shftf)
    inside = (x >= 0) & (x <= n - 1)
    exp = np.where(inside, cr(np.clip(x, 0, n - 1)) + 1j * ci(np.clip(x, 0, n - 1)), 0)
    assert np.abs(out - exp).max() < 1e-10


@pytest.mark.parametrize("name", sorted(CASES))
def test_inputs_regenerate_identically(golden, name):
    g = golden(name)
    assert g.checksum == g.expected_checksum, "synthetic inputs differ from the ones the fixture was made from"


@pytest.mark.parametrize("name", sorted(CASES))
def test_host_mirror_reproduces_reference_grid(golden, name):
    """The host set-up mirror yields exactly the reference's templates:
    every record header (m, n, s, ra, dec, fdot) and hemisphere."""
    g = golden(name)
    pm, mm, nn = g.job.sky_points()
    ref = g.ref["f64"]
    st, rec, per = refkit.search_points(refkit.load_oracle().orc_search_points, g.job.segment(),
                                        g.job.search_opts(), pm, mm, nn)
    assert st == 0
    np.testing.assert_array_equal(rec.hdr, ref.hdr)
    np.testing.assert_array_equal(rec.pm, ref.pm)


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_bit_identical_to_reference_f64(golden, oracle, name):
    """The C restatement reproduces the reference FP64 build's triggers bit
    for bit (same (f, F) float pairs in the same order)."""
    g = golden(name)
    pm, mm, nn = g.job.sky_points()
    os_ = refkit.OracleSegment(g.job, oracle)   # the signal file injected, as main.c does
    st, rec, per = refkit.search_points(oracle.orc_search_points, os_.seg, g.job.search_opts(), pm, mm, nn)
    assert st == 0
    ref = g.ref["f64"]
    assert len(rec) == len(ref)
    assert rec.ntrig == ref.ntrig
    for a, b in zip(rec.pairs, ref.pairs):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("name", sorted(CASES))
def test_reference_f32_build_close_to_f64(golden, name):
    """How far the reference's own default (FLOAT) build is from its DOUBLE
    build on the same inputs: the scale of precision the FP32 form must
    stay within (identical trigger set except threshold/neighbour ties)."""
    g = golden(name)
    r = refkit.compare_records(g.ref["f32"], g.ref["f64"], f_rtol=1e-6, F_rtol=1e-3, thr=g.case.thr, tie_band=2e-3)
    assert not r["unmatched"], r["unmatched"][:5]
    assert r["max_F_rel"] < 1e-2


def test_oracle_overflow_status(golden, oracle):
    """bufsize/2 triggers per spindown at most (jobcore.c:586-590)."""
    g = golden("g1_h1_directed")
    opts = g.job.search_opts()
    opts.bufsize = 8
    pm, mm, nn = g.job.sky_points()
    st, _, _ = refkit.search_points(oracle.orc_search_points, g.job.segment(), opts, pm, mm, nn)
    assert st == 3   # TDF_ERR_TRIGGER_OVERFLOW


def test_oracle_outside_ellipse_gives_no_records(golden, oracle):
    g = golden("g1_h1_directed")
    st, rec, per = refkit.search_points(oracle.orc_search_points, g.job.segment(), g.job.search_opts(),
                                        [1], [1e4], [1e4])
    assert st == 0 and len(rec) == 0 and per[0] == 0
