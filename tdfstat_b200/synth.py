"""Seeded synthetic inputs in the reference's on-disk formats.

The reference reads a directory tree (docs/input_data.md:306-356):
``indir/SSS/DD/xdat_SSS_BBBB.bin`` (float32, or ``xdatsc_`` float64 with
mods=read_O3, common.c:50-61), ``DetSSB.bin`` (3N float64 detector positions
w.r.t. the solar-system barycentre in units of light-seconds/dt, then phir and
epsm: common.c:103-114, genseg/get_barycenter.c:65-81) and ``starting_date``
(common.c:141-150), plus a grid file (int32 fftpad, 16 float64 M, 16 float64
Fisher: init.c:180-186) and an INI file (init.c:30-143).

No public data set is reproduced: the time series is seeded Gaussian noise
with zeroed gaps, the ephemeris is a circular 1 AU orbit in the ecliptic plus
Earth rotation, and the grid matrix is a seeded lower-triangular matrix with
the magnitudes of the example in docs/grid_generation.md.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from . import host

AU_LIGHT_S = 499.00478383615643      # 1 astronomical unit in light-seconds
R_EARTH_LIGHT_S = 6378.140 / 299792.458


def _cos(x: np.ndarray) -> np.ndarray:
    """Element-wise cos through the C library (math.cos), so that generated
    inputs do not depend on which SIMD path numpy picks on a given CPU."""
    return np.fromiter((math.cos(v) for v in np.asarray(x, dtype=np.float64).ravel()), dtype=np.float64,
                       count=np.size(x)).reshape(np.shape(x))


def _sin(x: np.ndarray) -> np.ndarray:
    return np.fromiter((math.sin(v) for v in np.asarray(x, dtype=np.float64).ravel()), dtype=np.float64,
                       count=np.size(x)).reshape(np.shape(x))


@dataclass
class Injection:
    """A CW signal in add_signal()'s model (init.c:365-504), 'amp' form."""
    f: float
    fdot: float
    ra: float
    dec: float
    iota: float
    psi: float
    phase: float
    snr: Optional[float] = None     # network SNR; sets h0 when given
    h0: float = 0.0
    reffr: int = 1


@dataclass
class Case:
    seg: int = 1
    band: int = 2880            # fpo = 10 + band/(2 dt) (common.c:14-18)
    dt: float = 2.0
    nod: int = 2
    overlap: float = 0.0
    dets: Sequence[str] = ("H1",)
    sigma: Sequence[float] = (1.0,)
    gap_frac: float = 0.05
    ngaps: int = 3
    read_o3: bool = False       # float64 xdatsc_ files (mods=read_O3)
    seed: int = 1
    fftpad: int = 1
    fdot_step: float = 1e-10    # spindown grid spacing [Hz/s] -> M[5]
    sky_cells: float = 16.0     # sky grid cells across oms -> M[10]
    thr: float = 14.5
    gtype: str = "directed_range"
    gcenter: Optional[Sequence[float]] = None   # f, fdot, ra, dec
    gsizes: Sequence[float] = (0, 0.0, 0.0, 0.0)   # fr_gsize, s, mm, nn
    gsteps: Sequence[float] = (1, 1.0, 1.0, 1.0)
    hemi: int = 0
    fstat_norm: str = ""
    narrowdown: float = -1.0
    veto_flag: int = 0
    vlines_hz: Sequence[Sequence[float]] = ()   # veto intervals [Hz]
    line_files: Sequence[Sequence[str]] = ()    # (name, text) of line lists under <indir>/lines/
    injections: Sequence[Injection] = ()
    addsig: Optional[Injection] = None          # written as the reference's signal file, not applied
    noise_seed: Optional[int] = None            # set: noise from its own generator (segments sharing a grid)
    label: str = ""
    mods_extra: str = ""                        # further search:mods words (e.g. write_signal)

    def settings(self) -> host.Settings:
        fpo = host.fpo(self.band, self.overlap, self.dt)
        return host.Settings(fpo=fpo, dt=self.dt, nod=self.nod, fftpad=self.fftpad,
                             M=[0.0] * 16).compute()


def grid_matrix(case: Case, rng: np.random.Generator) -> List[float]:
    """Lower-triangular generator (stored in M[] as jobcore.c:230-240 reads
    it: M[1]=M[2]=M[3]=M[6]=M[7]=M[11]=0), magnitudes relative to M[0] and
    M[5] as in the example of docs/grid_generation.md:31-35."""
    st = case.settings()
    M = [0.0] * 16
    M[0] = 2.0 * math.pi / st.nfftf
    M[5] = math.pi * case.dt * case.dt * case.fdot_step
    j = lambda: 1.0 + 0.05 * rng.uniform(-1, 1)
    M[4] = -3.63 * M[0] * j()
    M[8] = -517.0 * M[0] * j()
    M[12] = 200.0 * M[0] * j()
    M[9] = -0.78 * M[5] * j()
    M[13] = 1.44 * M[5] * j()
    M[10] = st.oms / case.sky_cells * j()
    M[14] = -0.516 * M[10] * j()
    M[15] = 0.759 * M[10] * j()
    return M


def detssb(N: int, dt: float, name: str, phir: float, orbit_phase: float) -> np.ndarray:
    """Detector position w.r.t. the SSB in light-seconds/dt, equatorial
    axes: circular 1 AU orbit in the ecliptic (obliquity C_EPSMA) plus the
    detector on a rotating spherical Earth (rate C_OMEGA_R)."""
    ephi = host.detector_geometry(name)[0]
    t = np.arange(N, dtype=np.float64) * dt
    om_y = 2.0 * math.pi / host.C_YEARSEC
    th = orbit_phase + om_y * t
    eps = host.C_EPSMA
    ex = AU_LIGHT_S * _cos(th)
    ey = AU_LIGHT_S * _sin(th) * math.cos(eps)
    ez = AU_LIGHT_S * _sin(th) * math.sin(eps)
    ro = phir + host.C_OMEGA_R * t
    rx = R_EARTH_LIGHT_S * math.cos(ephi) * _cos(ro)
    ry = R_EARTH_LIGHT_S * math.cos(ephi) * _sin(ro)
    rz = R_EARTH_LIGHT_S * math.sin(ephi) * np.ones_like(t)
    out = np.empty(3 * N)
    out[0::3] = (ex + rx) / dt
    out[1::3] = (ey + ry) / dt
    out[2::3] = (ez + rz) / dt
    return out


def noise(N: int, sigma: float, gap_frac: float, ngaps: int, rng: np.random.Generator) -> np.ndarray:
    """Gaussian white noise with `ngaps` contiguous zeroed gaps covering
    about gap_frac of the samples (the gap model of
    genseg/gauss-xdat-mask.c:32-75: zeros copied from a mask)."""
    x = rng.normal(0.0, sigma, N)
    if ngaps > 0 and gap_frac > 0:
        glen = max(1, int(N * gap_frac / ngaps))
        starts = np.sort(rng.choice(np.arange(1, N - glen - 1), size=ngaps, replace=False))
        for s in starts:
            x[s: s + glen] = 0.0
    return x


def modvir_np(det: host.Detector, cosmodf, sinmodf, sinal, cosal, sindel, cosdel, xdat):
    """Vectorised modvir (settings.c:254-294) for the injection."""
    c1, c2, c3, c4, c5, c6, c7, c8, c9 = det.amod
    cosalfr = cosal * det.cphir + sinal * det.sphir
    sinalfr = sinal * det.cphir - cosal * det.sphir
    c2d = cosdel ** 2
    c2sd = sindel * cosdel
    c = cosalfr * cosmodf + sinalfr * sinmodf
    s = sinalfr * cosmodf - cosalfr * sinmodf
    c2s = 2. * c * c
    cs = c * s
    aa = c1 * (2. - c2d) * c2s + c2 * (2. - c2d) * 2. * cs + c3 * c2sd * c + c4 * c2sd * s - c1 * (2. - c2d) + c5 * c2d
    bb = c6 * sindel * c2s + c7 * sindel * 2. * cs + c8 * cosdel * c + c9 * cosdel * s - c6 * sindel
    nz = np.abs(xdat.astype(np.float64)) > 2.2250738585072014e-308
    return np.where(nz, aa, 0.0), np.where(nz, bb, 0.0)


def inject(case: Case, sett: host.Settings, dets: List[host.Detector], xdats: List[np.ndarray],
           inj: Injection, cosmodf, sinmodf):
    """add_signal() (init.c:365-504) applied to float64 series; h0 from the
    network SNR when inj.snr is set (sum over detectors of s^2/sig2)."""
    N = sett.N
    freqo0 = 2 * math.pi * inj.f * sett.dt
    freqo1 = math.pi * inj.fdot * sett.dt * sett.dt
    freqo0 += 2. * freqo1 * N * (case.seg - inj.reffr)
    sa, ca = math.sin(inj.ra), math.cos(inj.ra)
    sd, cd = math.sin(inj.dec), math.cos(inj.dec)
    cosi = math.cos(inj.iota)
    psi, phi = inj.psi, inj.phase
    cosip = (1. + cosi * cosi) / 2.
    amp = [math.cos(2 * psi) * cosip * math.cos(phi) - math.sin(2 * psi) * cosi * math.sin(phi),
           math.sin(2 * psi) * cosip * math.cos(phi) + math.cos(2 * psi) * cosi * math.sin(phi),
           -math.cos(2 * psi) * cosip * math.sin(phi) - math.sin(2 * psi) * cosi * math.cos(phi),
           -math.sin(2 * psi) * cosip * math.sin(phi) + math.cos(2 * psi) * cosi * math.cos(phi)]
    phaseshift = freqo0 * N * (case.seg - inj.reffr) - freqo1 * (N * (case.seg - inj.reffr)) ** 2
    i = np.arange(N, dtype=np.float64)
    sigs = []
    for det, x in zip(dets, xdats):
        aa, bb = modvir_np(det, cosmodf, sinmodf, sa, ca, sd, cd, x)
        e = det.detssb
        sh = ca * cd * e[0::3] + sa * cd * e[1::3] + sd * e[2::3]
        ph = freqo0 * (i + sh) + freqo1 * (2. * sh * i + i * i + sh * sh) + phaseshift
        ph -= 2 * math.pi * sett.dt * sett.fpo * i
        cph, sph = _cos(ph), _sin(ph)
        s = amp[0] * aa * cph + amp[1] * bb * cph + amp[2] * aa * sph + amp[3] * bb * sph
        sigs.append(s)
    h0 = inj.h0
    if inj.snr is not None:
        tot = sum(float(np.sum(s * s)) / d.sig2 for s, d in zip(sigs, dets))
        h0 = inj.snr / math.sqrt(tot)
    for x, s in zip(xdats, sigs):
        nz = x != 0
        x[nz] += h0 * s[nz]
    return h0


def write_case(root: str, case: Case) -> str:
    """Write the input tree, grid, veto-line file and INI of `case` under
    `root`; returns the INI path."""
    rng = np.random.default_rng(case.seed)
    sett = case.settings()
    N = sett.N
    indir = os.path.join(root, "in")
    outdir = os.path.join(root, "out")
    segdir = os.path.join(indir, "%03d" % case.seg)
    os.makedirs(outdir, exist_ok=True)
    M = grid_matrix(case, rng)
    sett.M = M
    gpath = os.path.join(indir, "grid.bin")
    os.makedirs(indir, exist_ok=True)
    with open(gpath, "wb") as f:
        f.write(np.array([case.fftpad], dtype=np.int32).tobytes())
        f.write(np.array(M, dtype=np.float64).tobytes())
        f.write(np.zeros(16, dtype=np.float64).tobytes())
    orbit_phase = rng.uniform(0, 2 * math.pi)
    gmst0 = rng.uniform(0, 2 * math.pi)
    dets, xs = [], []
    nrng = rng if case.noise_seed is None else np.random.default_rng(case.noise_seed)
    for k, name in enumerate(case.dets):
        elam = host.detector_geometry(name)[1]
        phir = math.fmod(gmst0 + elam + 2 * math.pi, 2 * math.pi)
        e = detssb(N, case.dt, name, phir, orbit_phase)
        sigma = case.sigma[k] if k < len(case.sigma) else case.sigma[-1]
        x = noise(N, sigma, case.gap_frac, case.ngaps, nrng)
        d = host.Detector(name=name, xdat=x.astype(np.float32), detssb=e, phir=phir, epsm=host.C_EPSMA).finish()
        dets.append(d)
        xs.append(x)
    if case.injections:
        cosm, sinm = host.aux_arrays(N, sett.omr)
        for inj in case.injections:
            inject(case, sett, dets, xs, inj, cosm, sinm)
    for k, name in enumerate(case.dets):
        ddir = os.path.join(segdir, name)
        os.makedirs(ddir, exist_ok=True)
        if case.read_o3:
            xs[k].astype(np.float64).tofile(os.path.join(ddir, "xdatsc_%03d_%04d.bin" % (case.seg, case.band)))
        else:
            xs[k].astype(np.float32).tofile(os.path.join(ddir, "xdat_%03d_%04d.bin" % (case.seg, case.band)))
        np.concatenate([dets[k].detssb, [dets[k].phir, host.C_EPSMA]]).astype(np.float64).tofile(
            os.path.join(ddir, "DetSSB.bin"))
        with open(os.path.join(ddir, "starting_date"), "w") as f:
            f.write("1.2000000000e+09\n")
    label = ("_" + case.label) if case.label else ""
    if case.line_files:
        ldir = os.path.join(indir, "lines")
        os.makedirs(ldir, exist_ok=True)
        for name, text in case.line_files:
            with open(os.path.join(ldir, name), "w") as f:
                f.write(text)
    if case.vlines_hz:
        with open(os.path.join(outdir, "vlines_%04d%s.dat" % (case.band, label)), "w") as f:
            f.write("# fl[rad]  fr[rad]   fl[Hz]  fr[Hz]   line info\n")
            for fl, fr in case.vlines_hz:
                a = (fl - sett.fpo) / sett.B * math.pi
                b = (fr - sett.fpo) / sett.B * math.pi
                f.write("   %.15f  %.15f  %.15f  %.15f  synthetic\n" % (a, b, fl, fr))
            f.write("#band_veto_fraction= %6.4f\n" % 0.0)
    gc = case.gcenter
    if gc is None:
        gc = (sett.fpo + sett.B / 2, 0.0, 1.2, 0.3)
    lines = [
        "[search]",
        "indir = in",
        "outdir = out",
        "band = %d" % case.band,
        "seg = %d" % case.seg,
        "hemi = %d" % case.hemi,
        "thr = %r" % case.thr,
        "nod = %d" % case.nod,
        "dt = %r" % case.dt,
        "overlap = %r" % case.overlap,
        "narrowdown = %r" % case.narrowdown,
        "fstat_norm = %s" % case.fstat_norm,
        "grid_file = grid.bin",
        "usedet = %s" % "".join(case.dets),
        "addsig = %s" % (os.path.join(root, "in", "signal.txt") if case.addsig else ""),
        "mods = %s" % " ".join(w for w in ("read_O3" if case.read_o3 else "", case.mods_extra) if w),
        "label = %s" % case.label,
        "veto_flag = %d" % case.veto_flag,
        "checkp_flag = 0",
        "",
        "[grid]",
        "gtype = %s" % case.gtype,
        "gcenter = %.17g %.17g %.17g %.17g" % tuple(gc),
        "gsizes = %d %.9g %.9g %.9g" % tuple(case.gsizes),
        "gsteps = %d %.9g %.9g %.9g" % tuple(case.gsteps),
        "",
    ]
    if case.addsig:
        # the reference's signal file (read_signal_file, init.c:300-358), 'amp' form
        s = case.addsig
        with open(os.path.join(indir, "signal.txt"), "w") as f:
            f.write("amp %.17g %d %.17g %.17g %.17g %.17g %.17g %.17g %.17g\n"
                    % (s.h0, s.reffr, s.f, s.fdot, s.ra, s.dec, s.iota, s.psi, s.phase))
    ini = os.path.join(root, "search.ini")
    with open(ini, "w") as f:
        f.write("\n".join(lines))
    return ini
