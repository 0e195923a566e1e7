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
