"""The synthetic workloads of the benchmark and of the full-size GPU tests.

  cfg1  H1, N = 86164 (2 sidereal days at dt = 2 s), float64 input
        (mods=read_O3), one sky point x 64 spindowns
  cfg2  H1+L1, N = 86164, nfft = nfftf = 2^17, Ninterp = 2^18, Gaussian noise
        (sigma 1, 5% gaps) + a CW injection (network SNR 12, 100.1234 Hz,
        -3e-10 Hz/s), a 32 x 32 sky patch around the injection (step 0.25
        grid cells) x 401 spindowns = 410,624 templates
  cfg3  as cfg2 with N = 258492 (6 days), nfft = 2^18, Ninterp = 2^19,
        four injections (network SNR 20, 8, 12, 16 at 100.12, 100.05, 100.18,
        100.22 Hz), a 128 x 64 patch (step 0.1 cells) around the first x 401
        spindowns = 3,284,992 templates
  cfg4  64 segments, nod cycling through 2, 3, 4, 6 (N = 86164, 129246,
        172328, 258492; nfft 2^17, 2^17, 2^18, 2^18), per-segment seeds, noise
        and gaps, H1+L1; a 16 x 16 patch x 401 spindowns per segment =
        6,569,984 templates (MultiWorkload)
  cfg5  the scale configuration: H1+L1, N = 258492, sigma 1.0 / 1.3, 10% gaps,
        801 spindowns; a 32 x 32 patch (2^10 points) = 820,224 templates
        (larger skies scale the count, not the per-template work)
All are seeded; the F range is the all-sky one, [nmin, nmax] (settings.c:83-84).
"""
from __future__ import annotations

import numpy as np

from . import host, synth
from .shard import shard_points


def workload_case(name: str):
    if name == "cfg1":
        # directed_range gives 2g+1 spindowns: 65 for the 64 of the reference's single-point case
        return synth.Case(dt=2.0, nod=2, band=360, dets=("H1",), read_o3=True, seed=101, thr=14.5,
                          fdot_step=1e-10, sky_cells=16.0), (1, 1), 65, 0.25
    if name == "cfg5":
        inj = synth.Injection(f=100.1234, fdot=-3e-10, ra=4.0, dec=0.9, iota=0.9, psi=0.4, phase=2.2, snr=12.0)
        return synth.Case(dt=2.0, nod=6, band=360, dets=("H1", "L1"), sigma=(1.0, 1.3), gap_frac=0.10, seed=505,
                          thr=14.5, fdot_step=1e-10, sky_cells=16.0, injections=(inj,)), (32, 32), 801, 0.1
    if name.startswith("cfg4:"):
        # one segment of cfg4: cfg4:<k>, k = 1..64
        k = int(name.split(":")[1])
        nod = (2, 3, 4, 6)[(k - 1) % 4]
        inj = synth.Injection(f=100.1234, fdot=-3e-10, ra=4.0, dec=0.9, iota=0.9, psi=0.4, phase=2.2, snr=12.0)
        return synth.Case(seg=k, dt=2.0, nod=nod, band=360, dets=("H1", "L1"), seed=4000 + k, thr=14.5,
                          fdot_step=1e-10, sky_cells=16.0, injections=(inj,)), (16, 16), 401, 0.1
    # the injections (and the patches centred on them) lie well inside the
    # sky grid's ellipse: every patch point is searched (job_core skips
    # points outside it, jobcore.c:248)
    if name == "cfg3":
        # four signals at network SNR 20, 8, 12, 16; the patch is centred on
        # the first, the others lie elsewhere in the sky and the band
        injs = (synth.Injection(f=100.1234, fdot=-3e-10, ra=4.0, dec=0.9, iota=0.9, psi=0.4, phase=2.2, snr=20.0),
                synth.Injection(f=100.0517, fdot=-1e-10, ra=1.1, dec=-0.4, iota=0.3, psi=1.2, phase=0.7, snr=8.0),
                synth.Injection(f=100.1788, fdot=-6e-10, ra=2.6, dec=0.2, iota=1.4, psi=0.1, phase=4.1, snr=12.0),
                synth.Injection(f=100.2231, fdot=-2e-10, ra=5.3, dec=-1.1, iota=2.0, psi=0.8, phase=5.5, snr=16.0))
        return synth.Case(dt=2.0, nod=6, band=360, dets=("H1", "L1"), seed=303, thr=14.5, fdot_step=1e-10,
                          sky_cells=16.0, injections=injs), (128, 64), 401, 0.1
    inj = synth.Injection(f=100.1234, fdot=-3e-10, ra=4.0, dec=0.9, iota=0.9, psi=0.4, phase=2.2, snr=12.0)
    return synth.Case(dt=2.0, nod=2, band=360, dets=("H1", "L1"), seed=202, thr=14.5, fdot_step=1e-10,
                      sky_cells=16.0, injections=(inj,)), (32, 32), 401, 0.25


class Workload:
    """The benchmark search: one sky patch x nspd spindowns per rank.  With
    `world` ranks the point list holds world patches of the same region,
    patch r shifted by r/world of a grid step in mm (distinct sky points,
    all inside the grid), so that each rank's contiguous shard is one full
    patch: the work per GPU is fixed as the GPU count grows."""

    def __init__(self, name: str, root: str, world: int = 1, case=None):
        # case: (synth.Case, patch shape, spindowns, step) instead of the named workload's
        case, (nm, nn_), nspd, step = case if case is not None else workload_case(name)
        self.name, self.case = name, case
        inj = case.injections[0] if case.injections else None
        c = case
        # a directed_range INI centred on the injection (or a fixed point)
        ra, dec = (inj.ra, inj.dec) if inj else (1.2, 0.3)
        fdot = inj.fdot if inj else 0.0
        st = c.settings()
        c.gtype = "directed_range"
        c.gcenter = (st.fpo + st.B / 2, fdot, ra, dec)
        half = (nspd - 1) // 2
        c.gsizes = (st.nfft // 4 - 1024, float(half), 0.0, 0.0)
        c.gsteps = (1, 1.0, 1.0, 1.0)
        ini = synth.write_case(root, c)
        self.ini = ini
        job = host.Job(ini, float_build=True)
        self.job = job
        # the F range of an all-sky run: [nmin, nmax]
        job.range.fr = [job.sett.nmin, job.sett.nmax]
        job.sett.bufsize = job.sett.nfftf
        pm0, mm0, nn0 = job.sky_points()
        m0, n0 = mm0[0], nn0[0]
        pms, mms, nns = [], [], []
        for r in range(world):
            mg, ng = np.meshgrid((np.arange(nm) - nm // 2 + r / world) * step, (np.arange(nn_) - nn_ // 2) * step,
                                 indexing="ij")
            pms.append(np.full(nm * nn_, pm0[0], dtype=np.int32))
            mms.append((m0 + mg.ravel()).astype(np.float32))
            nns.append((n0 + ng.ravel()).astype(np.float32))
        self.pm, self.mm, self.nn = np.concatenate(pms), np.concatenate(mms), np.concatenate(nns)
        self.m0, self.n0, self.pm0 = m0, n0, pm0[0]
        self.nspd = nspd
        self.shape = (nm, nn_)
        self.centre = (nm // 2) * nn_ + nn_ // 2   # index of the patch centre (the injection's grid point)
        self.templates = nm * nn_ * nspd
        self.config = {"workload": name, "detectors": "".join(c.dets), "N": job.sett.N, "nfft": job.sett.nfft,
                       "nfftf": job.sett.nfftf, "Ninterp": job.sett.Ninterp, "sky_points": nm * nn_,
                       "spindowns": nspd, "templates_per_step": self.templates,
                       "fr": list(job.range.fr), "thr": c.thr}

    def patch(self, npts: int, extent: float = 3.2):
        """A square-ish patch of npts = 2^k sky points around the same centre,
        spanning `extent` grid cells in mm and nn (the spacing shrinks as
        the patch grows, so that every point stays inside the grid's
        ellipse).  Returns (pm, mm, nn)."""
        k = int(round(np.log2(npts)))
        assert 1 << k == npts
        a, b = 1 << (k // 2), 1 << (k - k // 2)
        step = extent / max(a, b)
        mg, ng = np.meshgrid((np.arange(a) - a // 2) * step, (np.arange(b) - b // 2) * step, indexing="ij")
        pm = np.full(npts, self.pm0, dtype=np.int32)
        return pm, (self.m0 + mg.ravel()).astype(np.float32), (self.n0 + ng.ravel()).astype(np.float32)

    def shard(self, rank: int, world: int):
        return shard_points(self.pm, self.mm, self.nn, rank, world)


class MultiWorkload:
    """cfg4: `nseg` segments (Workload "cfg4:<k>" each, under root/seg<k>),
    grouped by their sizes so that one engine per size can take the
    segments in turn."""

    def __init__(self, root: str, nseg: int = 64, world: int = 1):
        import os
        self.segments = [Workload("cfg4:%d" % k, os.path.join(root, "seg%02d" % k), world)
                         for k in range(1, nseg + 1)]
        self.nspd = self.segments[0].nspd
        self.templates = sum(w.templates for w in self.segments)
        sizes = sorted({w.job.sett.N for w in self.segments})
        self.config = {"workload": "cfg4", "detectors": "H1L1", "segments": nseg, "N": sizes,
                       "nfft": sorted({w.job.sett.nfft for w in self.segments}),
                       "sky_points_per_segment": len(self.segments[0].pm) // world, "spindowns": self.nspd,
                       "templates_per_step": self.templates, "thr": self.segments[0].case.thr}
