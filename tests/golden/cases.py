"""The golden cases: seeded synthetic searches small enough for the CPU
reference to run in seconds.  make_golden.py runs the reference build on each
and stores its records; the tests regenerate the inputs from these
definitions (checked against the stored input checksums) and compare.
"""
from __future__ import annotations

import hashlib
import os

from tdfstat_b200 import synth

GOLDEN_DIR = os.path.dirname(os.path.abspath(__file__))

CASES = {
    # one detector, float64 input (mods=read_O3), directed_range: one sky
    # point, 9 spindowns, low threshold so that many triggers are compared
    "g1_h1_directed": synth.Case(
        dt=16.0, nod=1, band=2880, dets=("H1",), read_o3=True, seed=11, thr=6.0,
        gtype="directed_range", gcenter=(100.0152, -2e-10, 1.2, 0.3),
        gsizes=(1800, 4.0, 0.0, 0.0), gsteps=(1, 1.0, 1.0, 1.0)),
    # H1+L1 network with an injected signal, allsky_range 3x3 sky patch x 11
    # spindowns, veto lines applied and the band narrowed down
    "g2_h1l1_inj": synth.Case(
        dt=8.0, nod=1, band=1440, dets=("H1", "L1"), sigma=(1.0, 1.3), seed=22, thr=8.0,
        fdot_step=2e-10, sky_cells=12.0,
        gtype="allsky_range", gcenter=(100.031, -4e-10, 2.1, -0.4),
        gsizes=(3600, 5.0, 1.0, 1.0), gsteps=(1, 1.0, 1.0, 1.0),
        narrowdown=0.45, veto_flag=1, vlines_hz=((100.010, 100.0105), (100.0400, 100.0412)),
        injections=(synth.Injection(f=100.031, fdot=-4e-10, ra=2.1, dec=-0.4, iota=0.7, psi=0.3,
                                    phase=1.1, snr=40.0),)),
    # the signal comes from a signal file (search:addsig) that the reference
    # injects itself with add_signal() before its search; the data files hold
    # noise only
    "g4_addsig": synth.Case(
        dt=8.0, nod=1, band=1440, dets=("H1", "L1"), sigma=(1.0, 1.2), seed=44, thr=8.0,
        fdot_step=2e-10, sky_cells=12.0,
        gtype="allsky_range", gcenter=(100.0412, -2e-10, 2.1, -0.4),
        gsizes=(3600, 5.0, 1.0, 1.0), gsteps=(1, 1.0, 1.0, 1.0),
        addsig=synth.Injection(f=100.0412, fdot=-2e-10, ra=2.1, dec=-0.4, iota=0.5, psi=0.8,
                               phase=0.3, h0=0.3)),
    # all-sky grid (spindown range from Smin/Smax per sky point, both
    # hemispheres) with blocks_avg F-statistic normalisation
    "g3_allsky_blocks": synth.Case(
        dt=8.0, nod=1, band=1440, dets=("H1", "L1"), sigma=(1.0, 1.0), seed=33, thr=9.0,
        fdot_step=1e-9, sky_cells=3.0, gtype="allsky", fstat_norm="blocks_avg"),
}


# Coincidences between segments (coincidences/coincidences.c): segments 1-4
# of one search (same grid and range, one INI per segment, noise per
# segment) with a signal (network SNR 14 per segment) whose frequency moves
# with its spindown; the reference's coincidence program runs on the
# reference's trigger files with each option set
COINC_CASES = {
    "c1_4seg": {
        "base": synth.Case(
            dt=8.0, nod=1, band=1440, dets=("H1", "L1"), sigma=(1.0, 1.1), seed=55, thr=6.5,
            fdot_step=2e-10, sky_cells=12.0, gtype="allsky_range",
            gcenter=(100.031, -4e-10, 2.1, -0.4), gsizes=(3600, 5.0, 1.0, 1.0), gsteps=(1, 1.0, 1.0, 1.0),
            injections=(synth.Injection(f=100.031, fdot=-4e-10, ra=2.1, dec=-0.4, iota=0.6, psi=0.2, phase=0.9,
                                        snr=14.0),)),
        "segs": (1, 2, 3, 4),
        "noise_seed": 5500,          # segment k: noise_seed + k
        "hemi": 2,                   # the hemisphere whose trigger files are compared
        "opts": {
            "a": dict(refr=2, cthr=7.0, scalef=4, scales=1, scalem=1, scalen=1, mincoin=2),
            "b": dict(refr=1, cthr=7.0, scalef=8, scales=2, scalem=2, scalen=2, mincoin=3),
        },
    },
}


def write_coinc_case(root: str, name: str):
    """Writes the segments of a coincidence case under `root` (one INI per
    segment, search_<seg>.ini); returns [(seg, ini path)]."""
    import dataclasses
    import shutil
    cc = COINC_CASES[name]
    out = []
    for seg in cc["segs"]:
        c = dataclasses.replace(cc["base"], seg=seg, noise_seed=cc["noise_seed"] + seg)
        ini = synth.write_case(root, c)
        segini = os.path.join(root, "search_%03d.ini" % seg)
        shutil.copy(ini, segini)
        out.append((seg, segini))
    return out


def input_checksum(root: str) -> str:
    """sha256 over the input files of a written case (sorted paths)."""
    h = hashlib.sha256()
    base = os.path.join(root, "in")
    for dp, _, fs in sorted(os.walk(base)):
        for f in sorted(fs):
            p = os.path.join(dp, f)
            h.update(os.path.relpath(p, base).encode())
            with open(p, "rb") as fh:
                h.update(fh.read())
    return h.hexdigest()
