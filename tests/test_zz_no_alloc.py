"""The allocation-free entry point tdf_fstat_operands_static(): for callers
that cannot allocate device memory while they run (the memory belongs to
another allocator or was reserved up front, or cudaMalloc's implicit
synchronisation is not acceptable on that path).  It keeps its scratch in a
static device array of the library, so it takes only caller-owned buffers.

The test builds the spindown operands of a sky point on the CPU (the FP64
oracle's sky stage), places them in device memory the test itself allocates
(the caller's buffers), calls the entry point through the C ABI for two
templates in a row, then at another transform length, detector count and
row stride, and checks each F spectrum against the engine entry point
tdf_fstat_spectrum() for the same template and against the FP64 oracle's
orc_fstat_spectrum(), at the split form's tolerance (1e-4, normalised per
bin by max(F, 1)).  This file is collected
last so that a failure here stops a -x run only after every other test ran.
"""
import ctypes as C
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-4


def _operands(oracle, job, pm, mm, nn):
    seg = job.segment()
    N, nifo = job.sett.N, job.sett.nifo
    xa = np.zeros(N * nifo, np.complex128)
    xb = np.zeros(N * nifo, np.complex128)
    t1 = np.zeros(N * nifo, np.float64)
    sh = np.zeros(N * nifo, np.float64)
    aa, bb = C.c_double(), C.c_double()
    oracle.orc_sky_stage.restype = C.c_int
    oracle.orc_sky_stage.argtypes = [C.c_void_p, C.c_int32, C.c_float, C.c_float, C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    st = oracle.orc_sky_stage(C.addressof(seg), pm, mm, nn, xa.ctypes.data, xb.ctypes.data, t1.ctypes.data,
                              sh.ctypes.data, C.byref(aa), C.byref(bb))
    assert st == 0
    i = np.tile(np.arange(N, dtype=np.float64), nifo)
    xab = np.stack([xa.real, xa.imag, xb.real, xb.imag], axis=1).astype(np.float32)   # [nifo*N, 4]
    s2 = (2.0 * i * sh).astype(np.float32)
    return xab, s2


def _split_sums(oracle, job, pm, mm, nn):
    """aa, bb as float accumulations over detectors (jobcore.c:373-386)."""
    seg = job.segment()
    N = job.sett.N
    tot_a, tot_b = np.float32(0), np.float32(0)
    orc = oracle
    orc.orc_modvir.restype = None
    orc.orc_modvir.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                               C.c_void_p, C.c_void_p]
    M = job.sett.M
    al1 = nn * M[10] + mm * M[14]
    al2 = nn * M[11] + mm * M[15]
    cof = job.sett.oms
    be1, be2 = al1 / cof, al2 / cof
    sindel = be1 * job.sett.sepsm - (2 * pm - 3) * math.sqrt(1. - be1 * be1 - be2 * be2) * job.sett.cepsm
    cosdel = math.sqrt(1. - sindel * sindel)
    sinal = (be1 - job.sett.sepsm * sindel) / (job.sett.cepsm * cosdel)
    cosal = be2 / cosdel
    for d in range(job.sett.nifo):
        a = np.zeros(N)
        b = np.zeros(N)
        orc.orc_modvir(C.addressof(seg), d, sinal, cosal, sindel, cosdel, a.ctypes.data, b.ctypes.data)
        s2 = job.dets[d].sig2
        tot_a = np.float32(float(tot_a) + float(np.cumsum(a * a)[-1]) / s2)
        tot_b = np.float32(float(tot_b) + float(np.cumsum(b * b)[-1]) / s2)
    return float(tot_a), float(tot_b)


def _call_case(lib, oracle, golden, name, nk, pad):
    """nk calls in a row for consecutive spindowns of the first sky point of
    golden case `name`, operands in caller buffers of row stride N + pad;
    each F spectrum checked against the engine's tdf_fstat_spectrum and the
    FP64 oracle's orc_fstat_spectrum."""
    import torch
    from tdfstat_b200 import _abi
    from tdfstat_b200.engine import Engine

    g = golden(name)
    job = g.job32
    pm, mm, nn = job.sky_points()
    p, m, n = int(pm[0]), float(mm[0]), float(nn[0])
    xab, s2 = _operands(oracle, job, p, m, n)
    aa, bb = _split_sums(oracle, job, p, m, n)
    N, nifo, nfftf = job.sett.N, job.sett.nifo, job.sett.nfftf
    Nal = N + pad
    if pad:
        xp = np.zeros((nifo, Nal, 4), np.float32)
        sp = np.zeros((nifo, Nal), np.float32)
        xp[:, :N] = xab.reshape(nifo, N, 4)
        sp[:, :N] = s2.reshape(nifo, N)
        xab, s2 = xp.reshape(-1, 4), sp.reshape(-1)
    fr0, fr1 = job.range.fr
    dev = torch.device("cuda", 0)
    d_xab = torch.from_numpy(xab).to(dev).contiguous()     # the caller's buffers
    d_s2 = torch.from_numpy(s2).to(dev).contiguous()
    d_F = torch.zeros(fr1 - fr0 + 1, dtype=torch.float32, device=dev)
    eng = Engine.from_job(job, form="split")
    seg64, opts64 = g.job.segment(), g.job.search_opts()
    M = job.sett.M
    ss0 = float(job.range.spndr[0])
    for k in range(nk):
        ss = float(np.float32(ss0 + k * job.range.sstep))
        spnd = ss * M[5] + n * M[9] + m * M[13]
        het1 = math.fmod(ss * M[4], M[0])
        if het1 < 0:
            het1 += M[0]
        d_F.fill_(-1.0)
        st = lib.tdf_fstat_operands_static(d_xab.data_ptr(), d_s2.data_ptr(), nifo, N, Nal, nfftf, het1, spnd,
                                           aa, bb, fr0, fr1, d_F.data_ptr(), None)
        assert st == _abi.TDF_OK, lib.tdf_last_error()
        torch.cuda.synchronize()
        F_static = d_F.double().cpu().numpy()
        F_engine = eng.fstat(p, m, n, ss)
        F_oracle = np.zeros_like(F_engine)
        assert oracle.orc_fstat_spectrum(C.byref(seg64), C.byref(opts64), p, m, n, ss,
                                         F_oracle.ctypes.data_as(C.POINTER(C.c_double)), len(F_oracle)) == 0
        e_eng = np.max(np.abs(F_static - F_engine) / np.maximum(F_engine, 1.0))
        e_orc = np.max(np.abs(F_static - F_oracle) / np.maximum(F_oracle, 1.0))
        print(name, "nfftf", nfftf, "Nal-N", pad, "call", k, "max normalised F difference: engine %.3g, "
              "oracle %.3g" % (e_eng, e_orc))
        assert e_eng <= TOL, e_eng
        assert e_orc <= TOL, e_orc
    eng.close()


def test_static_scratch_entry_matches_engine(golden, oracle):
    """Two calls in a row at one transform length (nfftf 2^14, two
    detectors), then a second length (nfftf 2^13, one detector) with
    operand rows padded beyond N, a three-detector network, and the first
    length again: the tables of every length stay valid side by side."""
    from tdfstat_b200.engine import load_library

    lib = load_library()
    _call_case(lib, oracle, golden, "g2_h1l1_inj", 2, 0)
    _call_case(lib, oracle, golden, "g1_h1_directed", 1, 1000)
    _call_case(lib, oracle, golden, "g6_h1l1v1", 1, 0)
    _call_case(lib, oracle, golden, "g2_h1l1_inj", 1, 0)


def test_static_scratch_entry_rejects_oversize():
    import torch
    from tdfstat_b200 import _abi
    from tdfstat_b200.engine import load_library

    lib = load_library()
    buf = torch.zeros(16, device="cuda")
    st = lib.tdf_fstat_operands_static(buf.data_ptr(), buf.data_ptr(), 1, 1000, 1000, 1 << 19, 0.0, 0.0,
                                       1.0, 1.0, 0, 10, buf.data_ptr(), None)
    assert st == _abi.TDF_ERR_UNSUPPORTED
    assert b"2^18" in lib.tdf_last_error()
