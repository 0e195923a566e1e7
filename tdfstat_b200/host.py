"""Host-side set-up of a search, mirroring TDFstat's C host (main.c:33-126).

This is the part of the reference that runs once per search, before the hot
path: reading the INI file, the grid matrix, the input time series and
ephemerides, the search settings, the search range and the veto lines.  It
produces the ``tdf_segment`` / ``tdf_search_opts`` descriptors of
include/tdfcuda.h.  Each function cites the reference lines it mirrors
(paths relative to the TDFstat tree).

C float/double semantics are kept explicit: values the reference stores in
``float`` fields are rounded with :func:`f32`; everything else is Python
float (IEEE double).
"""
from __future__ import annotations

import ctypes as C
import math
import os
import re
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np

from . import _abi
from . import vlines as vlines_mod

# common.h:14-31
RAD_TO_DEG = 180.0 / math.pi
C_EPSMA = 84381.448 / 3600.0 / RAD_TO_DEG
C_OMEGA_R = 7.2921151467064e-5
C_SIDDAY = 2.0 * math.pi / C_OMEGA_R
C_TAIDAY = 86400.0
C_YEARSEC = 365.25 * C_TAIDAY
NAV = 4096          # settings.h:12
NAVFSTAT = 4096     # auxi.h:12
MAXL = 512          # struct.h:14


def f32(x: float) -> float:
    """Round to IEEE single precision (a C store to a ``float``)."""
    return float(np.float32(x))


def cround(x: float) -> float:
    """The ``round`` macro of auxi.h:15: floor(x + 0.5)."""
    return math.floor(x + 0.5)


def ctrunc_int(x: float) -> int:
    """C conversion of a floating value to int (truncation toward zero)."""
    return int(math.trunc(x))


# ---------------------------------------------------------------- settings

def fpo(band: int, overlap: float, dt: float) -> float:
    """common.c:14-18"""
    return 10.0 + (1.0 - overlap) * band / (2 * dt)


def get_fdot_range(fpo_: float, dt: float):
    """common.c:22-33 -> (fdot_min, fdot_max)"""
    B = 1.0 / (2 * dt)
    if fpo_ < 200.0:
        return 2.0 * (fpo_ + B) / (2.0 * 1000.0 * C_YEARSEC), 0.0
    return 2e-10, 2e-11


@dataclass
class Settings:
    """Search_settings (struct.h:105-145), filled as search_settings()
    (settings.c:20-105) and read_grid() (init.c:148-197) do."""
    fpo: float
    dt: float
    nod: int
    fftpad: int
    M: List[float]
    B: float = 0.0
    oms: float = 0.0
    omr: float = 0.0
    N: int = 0
    nfft: int = 0
    Smin: float = 0.0
    Smax: float = 0.0
    interpftpad: int = 2
    Ninterp: int = 0
    nfftf: int = 0
    nmin: int = 0
    nmax: int = 0
    dd: int = 0
    nifo: int = 0
    sepsm: float = 0.0
    cepsm: float = 0.0
    bufsize: int = 0
    numlines_band: int = 0
    nvlines_all_inband: int = 0
    lines: List[List[float]] = field(default_factory=list)

    def compute(self):
        dt = self.dt
        self.B = 0.5 / dt
        self.oms = 2.0 * math.pi * self.fpo * dt
        self.omr = C_OMEGA_R * dt
        self.N = int(cround(self.nod * C_SIDDAY / dt))
        self.nfft = 1 << int(math.ceil(math.log(self.N) / math.log(2.0)))
        fdotmin, fdotmax = get_fdot_range(self.fpo, dt)
        self.Smax = math.pi * fdotmin * dt * dt
        self.Smin = math.pi * fdotmax * dt * dt
        self.interpftpad = 2
        self.Ninterp = self.interpftpad * self.nfft
        self.nfftf = self.fftpad * self.nfft
        self.nmin = ctrunc_int(self.fftpad * NAV * self.B)
        self.nmax = ctrunc_int((self.nfft / 2 - NAV * self.B) * self.fftpad)
        dayfbins = ctrunc_int(1.0 / C_SIDDAY * self.nfftf / (2 * self.B))
        self.dd = dayfbins - 1
        return self


# ---------------------------------------------------------------- detectors

def detector_geometry(name: str):
    """settings.c:178-213 -> (ephi, elam, eheight, egam)"""
    if name == "V1":
        return ((43. + 37. / 60. + 53.0880 / 3600.) / RAD_TO_DEG,
                (10. + 30. / 60. + 16.1885 / 3600.) / RAD_TO_DEG, 51.884,
                (135. - (19.0 + 25. / 60.0 + 57.96 / 3600.)) / RAD_TO_DEG)
    if name == "H1":
        return ((46 + (27 + 18.528 / 60.) / 60.) / RAD_TO_DEG,
                -(119 + (24 + 27.5657 / 60.) / 60.) / RAD_TO_DEG, 142.554,
                170.9994 / RAD_TO_DEG)
    if name == "L1":
        return ((30 + (33 + 46.4196 / 60.) / 60.) / RAD_TO_DEG,
                -(90 + (46 + 27.2654 / 60.) / 60.) / RAD_TO_DEG, -6.574,
                242.7165 / RAD_TO_DEG)
    raise ValueError("unknown detector " + name)


def rogcvir(ephi: float, egam: float) -> List[float]:
    """settings.c:226-248 -> [c1..c9]"""
    s2g, c2g = math.sin(2. * egam), math.cos(2. * egam)
    sp, cp = math.sin(ephi), math.cos(ephi)
    return [
        .25 * s2g * (1 + sp * sp),
        -.5 * c2g * sp,
        .5 * s2g * math.sin(2. * ephi),
        -c2g * cp,
        .75 * s2g * (cp * cp),
        c2g * sp,
        .5 * s2g * (1. + sp * sp),
        c2g * cp,
        .5 * s2g * math.sin(2. * ephi),
    ]


def seq_sum(x: np.ndarray) -> float:
    """Left-to-right double sum, as a C for-loop accumulates."""
    return float(np.cumsum(np.asarray(x, dtype=np.float64))[-1]) if len(x) else 0.0


def var(x: np.ndarray) -> float:
    """auxi.c:245-260"""
    n = len(x)
    xd = np.asarray(x, dtype=np.float64)
    mean = seq_sum(xd) / n
    return seq_sum((xd - mean) ** 2) / (n - 1)


@dataclass
class Detector:
    name: str
    xdat: np.ndarray            # float32 [N]
    detssb: np.ndarray          # float64 [3N]
    phir: float
    epsm: float
    start_time: float = 0.0
    Nzeros: int = 0
    crf0: float = 1.0
    sig2: float = 1.0
    amod: List[float] = field(default_factory=list)

    def finish(self):
        """read_xdat variance (common.c:68-78), read_detssb sines
        (common.c:123-126), rogcvir (settings.c:226-248)."""
        N = len(self.xdat)
        self.Nzeros = int(np.count_nonzero(self.xdat == 0))
        self.crf0 = float(N) / (N - self.Nzeros)
        self.sig2 = self.crf0 * var(self.xdat)
        self.sphir, self.cphir = math.sin(self.phir), math.cos(self.phir)
        self.sepsm, self.cepsm = math.sin(self.epsm), math.cos(self.epsm)
        ephi, _, _, egam = detector_geometry(self.name)
        self.amod = rogcvir(ephi, egam)
        return self


def aux_arrays(N: int, omr: float):
    """init_aux_array (init.c:222-239): cos/sin(omr*i) with the C library's
    cos/sin (math.cos/sin call the same libm)."""
    cosm = np.empty(N)
    sinm = np.empty(N)
    for i in range(N):
        a = omr * i
        cosm[i] = math.cos(a)
        sinm[i] = math.sin(a)
    return cosm, sinm


# ---------------------------------------------------------------- file readers

def read_ini(path: str) -> Dict[str, str]:
    """Key/value pairs of an INI file as iniparser reads them
    (section:key, lower case; inline '#' / ';' comments removed)."""
    out: Dict[str, str] = {}
    sec = ""
    with open(path) as f:
        for raw in f:
            line = raw.strip()
            if not line or line[0] in "#;":
                continue
            m = re.match(r"^\[(.*)\]$", line)
            if m:
                sec = m.group(1).strip().lower()
                continue
            if "=" not in line:
                continue
            k, v = line.split("=", 1)
            v = re.split(r"[#;]", v, maxsplit=1)[0].strip()
            if len(v) >= 2 and v[0] == v[-1] and v[0] in "\"'":
                v = v[1:-1]
            out[f"{sec}:{k.strip().lower()}"] = v
    return out


def read_grid(path: str):
    """init.c:180-191 -> (fftpad, M[16])"""
    with open(path, "rb") as f:
        fftpad = int(np.frombuffer(f.read(4), dtype=np.int32)[0])
        M = np.frombuffer(f.read(16 * 8), dtype=np.float64).tolist()
    return fftpad, M


def read_xdat(path: str, N: int, read_o3: bool) -> np.ndarray:
    """common.c:50-61"""
    if read_o3:
        x = np.fromfile(path, dtype=np.float64, count=N).astype(np.float32)
    else:
        x = np.fromfile(path, dtype=np.float32, count=N)
    out = np.zeros(N, dtype=np.float32)
    out[: len(x)] = x
    return out


def read_detssb(path: str, N: int):
    """common.c:103-114 -> (DetSSB[3N], phir, epsm)"""
    a = np.fromfile(path, dtype=np.float64, count=3 * N + 2)
    return a[: 3 * N].copy(), float(a[3 * N]), float(a[3 * N + 1])


# ---------------------------------------------------------------- search range

@dataclass
class SearchRange:
    """Search_range (struct.h:69-82); float fields hold f32-rounded values."""
    pmr: List[int]
    fr: List[int]
    mr: List[float]
    nr: List[float]
    spndr: List[float]
    mstep: float = 1.0
    nstep: float = 1.0
    sstep: float = 1.0


def ast2lin(alfa: float, delta: float, epsm: float):
    """auxi.c:32-58 -> (pm, be[2])"""
    be0 = math.cos(epsm) * math.sin(alfa) * math.cos(delta) + math.sin(epsm) * math.sin(delta)
    be1 = math.cos(alfa) * math.cos(delta)
    d1 = math.asin(be0 * math.sin(epsm) + math.sqrt(1. - be0 * be0 - be1 * be1) * math.cos(epsm)) - delta
    pm = 1 if abs(d1) < 10. * 2.220446049250313e-16 else 2
    return pm, [be0, be1]


def _lu_solve4(A: List[List[float]], b: List[float]) -> List[float]:
    """4x4 solve by Doolittle elimination with partial pivoting, the method
    gsl_linalg_LU_decomp / LU_solve document (dimless_to_code, auxi.c:63-90)."""
    n = 4
    a = [row[:] for row in A]
    perm = list(range(n))
    for j in range(n - 1):
        ip, mx = j, abs(a[j][j])
        for i in range(j + 1, n):
            if abs(a[i][j]) > mx:
                mx, ip = abs(a[i][j]), i
        if ip != j:
            a[j], a[ip] = a[ip], a[j]
            perm[j], perm[ip] = perm[ip], perm[j]
        piv = a[j][j]
        if piv != 0.0:
            for i in range(j + 1, n):
                f = a[i][j] / piv
                a[i][j] = f
                for k in range(j + 1, n):
                    a[i][k] -= f * a[j][k]
    x = [b[perm[i]] for i in range(n)]
    for i in range(n):
        s = x[i]
        for k in range(i):
            s -= a[i][k] * x[k]
        x[i] = s
    for i in range(n - 1, -1, -1):
        s = x[i]
        for k in range(i + 1, n):
            s -= a[i][k] * x[k]
        x[i] = s / a[i][i]
    return x


def dimless_to_code(M: List[float], pos: List[float]) -> List[float]:
    """auxi.c:63-90: solve M^T x = pos (M stored as 4 rows of 4, transposed
    in place before the LU), results rounded to float."""
    rows = [[M[4 * i + j] for j in range(4)] for i in range(4)]
    At = [[rows[j][i] for j in range(4)] for i in range(4)]
    return [f32(v) for v in _lu_solve4(At, pos)]


def _ludcmp(a: List[float], n: int):
    """auxi.c:366-432 (Numerical Recipes LU with implicit pivoting)."""
    indx = [0] * n
    vv = [0.0] * n
    for i in range(n):
        big = max(abs(a[n * i + j]) for j in range(n))
        vv[i] = 1.0 / big
    imax = -1
    for j in range(n):
        for i in range(j):
            s = a[n * i + j]
            for k in range(i):
                s -= a[n * i + k] * a[n * k + j]
            a[n * i + j] = s
        big = 0.0
        for i in range(j, n):
            s = a[n * i + j]
            for k in range(j):
                s -= a[n * i + k] * a[n * k + j]
            a[n * i + j] = s
            dum = vv[i] * abs(s)
            if dum >= big:
                big, imax = dum, i
        if j != imax:
            for k in range(n):
                a[n * imax + k], a[n * j + k] = a[n * j + k], a[n * imax + k]
            vv[imax] = vv[j]
        indx[j] = imax
        if a[n * j + j] == 0.0:
            a[n * j + j] = 1.0e-20
        if j != n:
            dum = 1.0 / a[n * j + j]
            for i in range(j + 1, n):
                a[n * i + j] *= dum
    return indx


def _lubksb(a: List[float], n: int, indx: List[int], b: List[float]):
    """auxi.c:435-470"""
    ii = -1
    for i in range(n):
        ip = indx[i]
        s = b[ip]
        b[ip] = b[i]
        if ii >= 0:
            for j in range(ii, i):
                s -= a[n * i + j] * b[j]
        elif s:
            ii = i
        b[i] = s
    for i in range(n - 1, -1, -1):
        s = b[i]
        for j in range(i + 1, n):
            s -= a[n * i + j] * b[j]
        b[i] = s / a[n * i + i]


def gridr(M: List[float], oms: float, Smax: float):
    """auxi.c:264-332 -> (spndr, nr, mr) as f32 values"""
    Ob = math.pi
    cof = oms + Ob
    Mp = [0.0] * 16
    for i in range(4):
        for j in range(4):
            Mp[4 * i + j] = M[4 * j + i]
    indx = _ludcmp(Mp, 4)
    smx = [0.0] * 64
    for i in range(8):
        smx[8 * i + 2] = cof
        smx[8 * i + 6] = -cof
    for i in range(4):
        smx[16 * i + 3] = smx[16 * i + 7] = cof
        smx[16 * i + 11] = smx[16 * i + 15] = -cof
    for i in range(8):
        smx[4 * i] = Ob
        smx[4 * i + 32] = -Ob
    for i in range(2):
        for j in range(4):
            smx[32 * i + 4 * j + 1] = -Smax
            smx[32 * i + 4 * j + 17] = 0.
    for i in range(16):
        b = smx[4 * i: 4 * i + 4]
        _lubksb(Mp, 4, indx, b)
        smx[4 * i: 4 * i + 4] = b
    spndr = [16384.0, -16384.0]
    nr = [16384.0, -16384.0]
    mr = [16384.0, -16384.0]
    for i in range(16):
        for rng, k in ((spndr, 1), (nr, 2), (mr, 3)):
            v = smx[4 * i + k]
            if math.floor(v) < rng[0]:
                rng[0] = f32(math.floor(v))
            if math.ceil(v) > rng[1]:
                rng[1] = f32(math.ceil(v))
    return spndr, nr, mr


def set_search_range(sett: Settings, ini: Dict[str, str], float_build: bool = True) -> SearchRange:
    """init.c:510-705.  float_build selects FLOAT_TYPE of the reference build
    whose arithmetic is mirrored (PREC=FLOAT is the reference default)."""
    hemi = int(ini.get("search:hemi", "0") or 0)
    pmr = [hemi, hemi] if hemi else [1, 2]
    gtype = ini.get("grid:gtype", "allsky")
    if gtype == "allsky":
        spndr, nr, mr = gridr(sett.M, sett.oms, sett.Smax)
        return SearchRange(pmr=pmr, fr=[sett.nmin, sett.nmax], mr=mr, nr=nr, spndr=spndr)
    gc = ini["grid:gcenter"].split()
    fr, sr, alphar, deltar = (f32(float(v)) for v in gc[:4])
    gs = ini["grid:gsizes"].split()
    fr_gsize = int(float(gs[0]))
    sr_gsize, mr_gsize, nr_gsize = (f32(float(v)) for v in gs[1:4])
    st = ini["grid:gsteps"].split()
    sr_step, mr_step, nr_step = (f32(float(v)) for v in st[1:4])
    M = sett.M
    sgnlol = [0.0, math.pi * sr * sett.dt * sett.dt, 0.0, 0.0]
    cof = sett.oms
    pm, be = ast2lin(alphar, deltar, C_EPSMA)
    pmr = [pm, pm]
    sgnlol[2] = be[0] * cof
    sgnlol[3] = be[1] * cof
    code = dimless_to_code(M, sgnlol)
    het0 = math.fmod(code[2] * M[8] + code[3] * M[12], M[0])
    het1 = math.fmod(code[1] * M[4], M[0])
    if float_build:
        het1 = f32(het1)
    if het1 < 0:
        het1 = het1 + M[0]
        if float_build:
            het1 = f32(het1)
    sgnl0 = het0 + het1
    if float_build:
        sgnl0 = f32(sgnl0)
        t = f32(sgnl0 * f32(sett.nfftf))
    else:
        t = sgnl0 * sett.nfftf
    code0 = f32((fr - sett.fpo) / sett.B * sett.nfftf / 2 - t / (2 * math.pi))
    fr_gsize = int(cround(fr_gsize))
    sr_gsize = f32(cround(f32(sr_gsize / sr_step)) * sr_step)
    nr_gsize = f32(cround(f32(nr_gsize / nr_step)) * nr_step)
    mr_gsize = f32(cround(f32(mr_gsize / mr_step)) * mr_step)
    if gtype == "allsky_range":
        fmid = int(cround(code0))
        smid, nmid, mmid = (f32(cround(c)) for c in code[1:4])
    elif gtype == "directed_range":
        fmid = ctrunc_int(code0)
        smid, nmid, mmid = code[1], code[2], code[3]
    else:
        raise ValueError("Unknown grid type " + gtype)
    return SearchRange(
        pmr=pmr,
        fr=[fmid - fr_gsize, fmid + fr_gsize],
        spndr=[f32(smid - sr_gsize), f32(smid + sr_gsize)],
        nr=[f32(nmid - nr_gsize), f32(nmid + nr_gsize)],
        mr=[f32(mmid - mr_gsize), f32(mmid + mr_gsize)],
        mstep=mr_step, nstep=nr_step, sstep=sr_step)


def sky_points(rng: SearchRange):
    """The (pm, mm, nn) enumeration of search() (jobcore.c:88-111), without
    checkpoint restart.  Returns three lists."""
    pms, mms, nns = [], [], []
    for pm in range(rng.pmr[0], rng.pmr[1] + 1):
        imm_size = ctrunc_int(f32(f32(f32(rng.mr[1] - rng.mr[0]) / rng.mstep) + 1))
        for imm in range(imm_size):
            mm = f32(rng.mr[0] + f32(imm * rng.mstep))
            inn_size = ctrunc_int(f32(f32(f32(rng.nr[1] - rng.nr[0]) / rng.nstep) + 1))
            for inn in range(inn_size):
                nn = f32(rng.nr[0] + f32(inn * rng.nstep))
                pms.append(pm)
                mms.append(mm)
                nns.append(nn)
    return pms, mms, nns


# ---------------------------------------------------------------- [gpu] section

@dataclass
class GpuOptions:
    """The INI's [gpu] section, read by this library only (the reference's
    iniparser-based host ignores sections it does not ask for):
    form = split | fp64, device = CUDA device, sky_batch = sky points per
    batch (0: the library's default), templates_per_chunk = templates per
    pass launch (0: the library's default, or what tdf_engine_autotune
    picks)."""
    form: str = "split"
    device: int = 0
    sky_batch: int = 0
    templates_per_chunk: int = 0


def gpu_options(ini: Dict[str, str]) -> GpuOptions:
    g = GpuOptions(form=(ini.get("gpu:form", "") or "split").lower(),
                   device=int(ini.get("gpu:device", "") or 0),
                   sky_batch=int(ini.get("gpu:sky_batch", "") or 0),
                   templates_per_chunk=int(ini.get("gpu:templates_per_chunk", "") or 0))
    if g.form not in ("split", "fp64"):
        raise ValueError("[gpu] form must be split or fp64, not %r" % g.form)
    if g.device < 0 or g.sky_batch < 0 or not (0 <= g.templates_per_chunk <= 48):
        raise ValueError("[gpu] device/sky_batch >= 0 and templates_per_chunk in 0..48")
    return g


# ---------------------------------------------------------------- veto lines
# narrow_down_band, read_band_vlines, extract_band_vlines: tdfstat_b200/vlines.py


# ---------------------------------------------------------------- injection output

def write_signal_files(job, signals) -> List[str]:
    """mods=write_signal (init.c:475-497): per detector the injected signal
    h0*s_n[i], i < N, one "%e" value per line, into
    <outdir>/injections/signal_<seg>_<band>_<det><label>; returns the paths."""
    d = os.path.join(job.outdir, "injections")
    os.makedirs(d, exist_ok=True)
    paths = []
    for det, sig in zip(job.dets, signals):
        p = os.path.join(d, "signal_%03d_%04d_%s%s" % (job.seg, job.band, det.name, job.label))
        with open(p, "w") as f:
            f.write("".join("%e\n" % v for v in np.asarray(sig, dtype=np.float64)))
        paths.append(p)
    return paths


# ---------------------------------------------------------------- the job

def read_signal_file(path: str) -> Dict[str, float]:
    """read_signal_file (init.c:300-358): skips tokens up to 'amp' or 'snr',
    then reads h0 (or snr), reffr, freq, fdot, ra, dec, iota, psi, phase."""
    with open(path) as f:
        tok = f.read().split()
    k = 0
    while k < len(tok) and tok[k] not in ("amp", "snr"):
        k += 1
    if k == len(tok):
        raise ValueError("%s: no 'amp' or 'snr' line" % path)
    form = tok[k]
    v = tok[k + 1:k + 10]
    out = {"form": form, "reffr": int(v[1])}
    out["h0" if form == "amp" else "snr"] = float(v[0])
    for name, s in zip(("freq", "fdot", "ra", "dec", "iota", "psi", "phase"), v[2:]):
        out[name] = float(s)
    return out


class Job:
    """Everything the reference's main() prepares before search(), built from
    an INI file (main.c:33-116), plus the descriptors of include/tdfcuda.h.
    A signal file named by search:addsig is read (job.signal, a tdf_signal)
    but not applied: the engine applies it on the device
    (Engine.add_signal), as main.c:101-104 does on the host."""

    def __init__(self, ini_path: str, float_build: bool = True, vlines: str = "auto"):
        """`vlines`: "auto" reads <outdir>/vlines_<band><label>.dat when it
        exists and otherwise extracts the band's veto lines from
        <indir>/lines/ and writes that file (main.c:84-94); "extract" always
        extracts and writes it (vlinegen.c:66-78)."""
        if vlines not in ("auto", "extract"):
            raise ValueError("vlines must be 'auto' or 'extract'")
        self.ini_path = ini_path
        ini = read_ini(ini_path)
        self.ini = ini
        indir = ini["search:indir"]
        indir_ini = indir
        base = os.path.dirname(os.path.abspath(ini_path))
        if not os.path.isabs(indir):
            indir = os.path.join(base, indir)
        self.indir = indir
        self.band = int(ini["search:band"])
        self.seg = int(ini["search:seg"])
        self.thr = float(ini.get("search:thr", "20") or 20)
        nod = int(ini["search:nod"])
        dt = float(ini["search:dt"])
        overlap = float(ini.get("search:overlap", "0") or 0)
        narrowdown = float(ini.get("search:narrowdown", "-1") or -1)
        if narrowdown < 0.:
            narrowdown = (1. - overlap) / 2.
        narrowdown *= math.pi
        self.narrowdown = narrowdown          # opts->narrowdown [rad] (init.c:134-139)
        self.usedet = ini.get("search:usedet", "")
        self.mods = ini.get("search:mods", "")
        self.fstat_norm = ini.get("search:fstat_norm", "")
        self.veto_flag = int(ini.get("search:veto_flag", "0") or 0)
        self.gpu = gpu_options(ini)
        self.gtype = ini.get("grid:gtype", "allsky")
        outdir = ini.get("search:outdir", ".")
        if not os.path.isabs(outdir):
            outdir = os.path.join(base, outdir)
        self.outdir = outdir
        label = ini.get("search:label", "")
        self.label = "_" + label if label else ""
        read_o3 = "read_O3" in self.mods
        self.write_signal = "write_signal" in self.mods   # init.c:476
        segdir = os.path.join(indir, "%03d" % self.seg)
        names = []
        for d in ("H1", "L1", "V1"):   # detectors_settings, settings.c:136-169
            if (not self.usedet or d in self.usedet) and os.path.isdir(os.path.join(segdir, d)):
                names.append(d)
        grid_file = ini.get("search:grid_file", "")
        if grid_file.startswith("/"):
            gpath = grid_file
        elif grid_file:
            gpath = os.path.join(indir, grid_file)
        elif len(self.usedet) == 2 and len(names) == 1:
            gpath = os.path.join(segdir, names[0], "grid.bin")
        else:
            gpath = os.path.join(segdir, "grids", "grid_%03d_%04d_%s.bin" % (self.seg, self.band, "".join(names)))
        fftpad, M = read_grid(gpath)
        self.sett = Settings(fpo=fpo(self.band, overlap, dt), dt=dt, nod=nod, fftpad=fftpad, M=M).compute()
        N = self.sett.N
        self.dets: List[Detector] = []
        for d in names:
            fn = ("xdatsc_%03d_%04d.bin" if read_o3 else "xdat_%03d_%04d.bin") % (self.seg, self.band)
            x = read_xdat(os.path.join(segdir, d, fn), N, read_o3)
            ssb, phir, epsm = read_detssb(os.path.join(segdir, d, "DetSSB.bin"), N)
            self.dets.append(Detector(name=d, xdat=x, detssb=ssb, phir=phir, epsm=epsm).finish())
        self.sett.nifo = len(self.dets)
        self.sett.sepsm = self.dets[-1].sepsm
        self.sett.cepsm = self.dets[-1].cepsm
        # main.c:78-94
        narrow = vlines_mod.narrow_down_lines(narrowdown) if narrowdown < 0.5 * math.pi else []
        os.makedirs(outdir, exist_ok=True)                 # main.c:53-64
        self.vlines_file = os.path.join(outdir, "vlines_%04d%s.dat" % (self.band, self.label))
        if vlines == "auto" and os.access(self.vlines_file, os.R_OK):
            bv = vlines_mod.read_band_vlines(self.vlines_file, narrow, self.veto_flag)
        else:
            bv = vlines_mod.extract_band_vlines(
                self.sett.fpo, self.sett.B, N, self.sett.dt, [d.detssb for d in self.dets],
                [d.name for d in self.dets], indir_ini, narrow, self.veto_flag, self.vlines_file, base=base)
        self.vlines = bv
        self.lines = bv.lines
        self.numlines = bv.numlines_band
        self.cosmodf, self.sinmodf = aux_arrays(N, self.sett.omr)
        self.range = set_search_range(self.sett, ini, float_build=float_build)
        self.sett.bufsize = self.sett.nfftf // 16 if self.gtype == "allsky" else self.sett.nfftf
        self.signal = None
        addsig = ini.get("search:addsig", "")
        if addsig:
            p = addsig if os.path.isabs(addsig) else os.path.join(base, addsig)
            sp = read_signal_file(p)
            sig = _abi.TdfSignal()
            sig.h0 = sp.get("h0", 0.0)
            sig.snr = sp.get("snr", 0.0)
            for name in ("freq", "fdot", "ra", "dec", "iota", "psi", "phase"):
                setattr(sig, name, sp[name])
            sig.fpo, sig.B = self.sett.fpo, self.sett.B
            sig.reffr, sig.seg = sp["reffr"], self.seg
            self.signal = sig
        self._keep = []

    # descriptors ---------------------------------------------------------
    def segment(self) -> _abi.TdfSegment:
        s = _abi.TdfSegment()
        st = self.sett
        s.N, s.nfft, s.nfftf, s.Ninterp = st.N, st.nfft, st.nfftf, st.Ninterp
        s.interpftpad, s.nifo = st.interpftpad, st.nifo
        s.dt, s.oms, s.sepsm, s.cepsm, s.Smin, s.Smax = st.dt, st.oms, st.sepsm, st.cepsm, st.Smin, st.Smax
        for i in range(16):
            s.M[i] = st.M[i]
        self._cos = np.ascontiguousarray(self.cosmodf, dtype=np.float64)
        self._sin = np.ascontiguousarray(self.sinmodf, dtype=np.float64)
        s.cosmodf = self._cos.ctypes.data_as(C.POINTER(C.c_double))
        s.sinmodf = self._sin.ctypes.data_as(C.POINTER(C.c_double))
        for i, d in enumerate(self.dets):
            x = np.ascontiguousarray(d.xdat, dtype=np.float32)
            e = np.ascontiguousarray(d.detssb, dtype=np.float64)
            self._keep += [x, e]
            s.det[i].xdat = x.ctypes.data_as(C.POINTER(C.c_float))
            s.det[i].detssb = e.ctypes.data_as(C.POINTER(C.c_double))
            s.det[i].sig2 = d.sig2
            s.det[i].sphir = d.sphir
            s.det[i].cphir = d.cphir
            for k in range(9):
                s.det[i].amod[k] = d.amod[k]
        return s

    def search_opts(self) -> _abi.TdfSearchOpts:
        o = _abi.TdfSearchOpts()
        o.thr = self.thr
        o.fr[0], o.fr[1] = self.range.fr
        o.allsky = 1 if self.gtype == "allsky" else 0
        o.blocks_avg = 1 if self.fstat_norm == "blocks_avg" else 0
        o.spndr[0], o.spndr[1] = self.range.spndr
        o.sstep = self.range.sstep
        o.bufsize = self.sett.bufsize
        o.numlines = self.numlines
        ln = np.ascontiguousarray(np.array(self.lines if self.lines else [[0.0, 0.0]], dtype=np.float64).reshape(-1))
        self._keep.append(ln)
        o.lines = ln.ctypes.data_as(C.POINTER(C.c_double))
        return o

    def sky_points(self):
        return sky_points(self.range)


def vlinegen(ini_path: str) -> str:
    """vlinegen.c: extracts the veto lines of the INI's band from the line
    lists under <indir>/lines/ and (over)writes <outdir>/vlines_<band><label>.dat,
    the file a later search reads; returns its path."""
    return Job(ini_path, vlines="extract").vlines_file

