"""The largest transforms the engine takes: nfft = 2^19 (N = 516985, 12
sidereal days at dt = 2 s; Ninterp = 2^20, the limit of the sky stage) with
fftpad 1 and 2 (nfftf = 2^19 and 2^20), the 1024-point passes of the
four-step FFT.  Split form against the FP64 oracle (orc_fstat_spectrum) on
single templates, at the split tolerance (1e-4 normalised F error), and the
records of one sky point x 3 spindowns against orc_search_points.  The FP64
form is limited to nfftf <= 2^18 and refuses these sizes with a status."""
import ctypes as C
import shutil
import tempfile

import numpy as np
import pytest

import refkit
from tdfstat_b200 import _abi, host, synth
from tdfstat_b200.engine import Engine, TdfError

pytestmark = pytest.mark.gpu

TOL = 1e-4


@pytest.fixture(scope="module")
def jobs():
    made = {}

    def get(fftpad):
        if fftpad not in made:
            root = tempfile.mkdtemp(prefix="tdf_max_")
            inj = synth.Injection(f=100.1234, fdot=-3e-10, ra=4.0, dec=0.9, iota=0.9, psi=0.4, phase=2.2,
                                  snr=15.0)
            c = synth.Case(dt=2.0, nod=12, band=360, dets=("H1", "L1"), seed=1212, thr=14.5, fdot_step=1e-10,
                           sky_cells=16.0, fftpad=fftpad, injections=(inj,))
            st = c.settings()
            c.gtype = "directed_range"
            c.gcenter = (st.fpo + st.B / 2, inj.fdot, inj.ra, inj.dec)
            c.gsizes = (st.nfft // 4 - 1024, 1.0, 0.0, 0.0)
            ini = synth.write_case(root, c)
            out = []
            for fb in (True, False):
                j = host.Job(ini, float_build=fb)
                j.range.fr = [j.sett.nmin, j.sett.nmax]
                j.sett.bufsize = j.sett.nfftf
                out.append(j)
            made[fftpad] = (out[0], out[1], root)
        return made[fftpad][:2]

    yield get
    for _, _, root in made.values():
        shutil.rmtree(root, ignore_errors=True)


@pytest.mark.parametrize("fftpad", [1, 2])
def test_largest_transforms_match_oracle(jobs, oracle, fftpad):
    j32, j64 = jobs(fftpad)
    assert j32.sett.nfft == 1 << 19 and j32.sett.Ninterp == 1 << 20 and j32.sett.nfftf == fftpad << 19
    seg, opts = j64.segment(), j64.search_opts()
    pm, mm, nn = j32.sky_points()
    eng = Engine.from_job(j32, form="split")
    res = eng.search(pm[:1], mm[:1], nn[:1])
    assert len(res) == 3
    for r in range(3):
        m, n, s = (float(v) for v in res.hdr[r, :3])
        Fg = eng.fstat(int(pm[0]), m, n, s)
        Fo = np.zeros_like(Fg)
        st = oracle.orc_fstat_spectrum(C.byref(seg), C.byref(opts), int(pm[0]), m, n, s,
                                       Fo.ctypes.data_as(C.POINTER(C.c_double)), len(Fo))
        assert st == 0
        err = np.max(np.abs(Fg - Fo) / np.maximum(Fo, 1.0))
        print("nfftf 2^%d template %d: max normalised F err %.3g" % (int(np.log2(j32.sett.nfftf)), r, err))
        assert err <= TOL, err
    rec = refkit.Records(res.hdr, res.pairs, np.repeat(pm[:1], res.per_point))
    st, ref, _ = refkit.search_points(oracle.orc_search_points, seg, opts, pm[:1], mm[:1], nn[:1])
    assert st == 0 and len(ref) == 3
    cmp = refkit.compare_records(rec, ref, f_rtol=2e-6, F_rtol=TOL, thr=float(opts.thr), tie_band=TOL)
    assert not cmp["unmatched"], cmp["unmatched"][:10]
    assert cmp["only_a"] + cmp["only_b"] <= max(2, 0.002 * cmp["matched"])
    eng.close()


def test_fp64_form_refuses_transforms_above_2_18(jobs):
    _, j64 = jobs(1)
    with pytest.raises(TdfError) as ei:
        Engine.from_job(j64, form="fp64")
    assert ei.value.status == _abi.TDF_ERR_UNSUPPORTED
