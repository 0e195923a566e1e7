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

# Instrumental line lists (<indir>/lines/<det>lines*.csv, columns of
# common.c:226-234) for a band of [100, 100.0625] Hz: singlets, a comb of
# fixed width and one of scaling width, harmonics in and out of the band,
# overlapping veto intervals, comment lines, white space around fields.  The
# demodulation widens every line by ~0.01 Hz at 100 Hz (the detector's
# velocity, v/c ~ 1e-4), so the band keeps [~100.017, ~100.052] Hz unvetoed.
LINE_FILES_100HZ = (
    ("H1lines.csv",
     "% f [Hz], type, offset [Hz], first harmonic, last harmonic, left width [Hz], right width [Hz], comment\n"
     "100.006,0,0,0,0,0.0002,0.0003,singlet in the band\n"
     "60.0,0,0,0,0,0.01,0.01,mains: below the band\n"
     "0.5,1,0.0,198,202,0.0001,0.0001,fixed comb: harmonic 200 at 100 Hz\n"),
    ("H1lines_O3.csv",
     "% a second list of the same detector\n"
     "120.0,0,0,0,0,0.05,0.05,out of the band\n"
     "100.0615,0,0,0,0,0.0,0.0,singlet at the upper edge\n"),
    ("L1lines.csv",
     "% L1\n"
     "16.677,2,0.0,5,7,0.00002,0.00001,scaling comb: harmonic 6 at 100.062 Hz\n"
     " 1.0, 1, 0.5, 99, 100, 0.0, 0.0, fixed comb with an offset: 99.5 and 100.5 Hz\n"),
)

# The same kind of lists for a band at 250 Hz, where the spindown range
# (fdotmax = 2e-11 Hz/s above 200 Hz, common.c:22-33) adds to the widening.
LINE_FILES_250HZ = (
    ("H1lines.csv",
     "% H1\n"
     "250.021,0,0,0,0,0.0001,0.0001,singlet\n"
     "50.0,2,0.0,4,6,0.00001,0.00002,scaling comb: harmonic 5 at 250 Hz\n"),
    ("L1lines_a.csv",
     "% L1\n"
     "0.25,1,0.0,1000,1001,0.0005,0.0005,fixed comb: 250 and 250.25 Hz\n"
     "250.05,0,0,0,0,0.0,0.0,singlet\n"),
)

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
    # no veto file in the output directory: the search extracts the band's
    # veto lines from the line lists of both detectors (extract_band_vlines,
    # main.c:84-94), writes the veto file and applies the lines (veto_flag)
    "g5_vlines": synth.Case(
        dt=8.0, nod=1, band=1440, dets=("H1", "L1"), sigma=(1.0, 1.1), seed=66, thr=8.0,
        fdot_step=2e-10, sky_cells=12.0,
        gtype="allsky_range", gcenter=(100.035, -2e-10, 2.1, -0.4),
        gsizes=(3600, 3.0, 1.0, 1.0), gsteps=(1, 1.0, 1.0, 1.0),
        narrowdown=0.45, veto_flag=1, line_files=LINE_FILES_100HZ,
        injections=(synth.Injection(f=100.035, fdot=-2e-10, ra=2.1, dec=-0.4, iota=0.7, psi=0.3,
                                    phase=1.1, snr=30.0),)),
    # a three-detector network (H1, L1, V1: the general detector loop of the
    # demodulation and the sky stage) with an injection
    "g6_h1l1v1": synth.Case(
        dt=8.0, nod=1, band=1440, dets=("H1", "L1", "V1"), sigma=(1.0, 1.2, 1.5), seed=88, thr=8.0,
        fdot_step=2e-10, sky_cells=12.0,
        gtype="allsky_range", gcenter=(100.031, -2e-10, 0.7, 0.9),
        gsizes=(3600, 3.0, 1.0, 1.0), gsteps=(1, 1.0, 1.0, 1.0),
        injections=(synth.Injection(f=100.031, fdot=-2e-10, ra=0.7, dec=0.9, iota=0.4, psi=1.2,
                                    phase=2.0, snr=30.0),)),
    # fftpad = 2 in the grid file: spindown FFTs of nfftf = 2 nfft and the
    # F-statistic range scaled by it (settings.c:83-84)
    "g7_fftpad2": synth.Case(
        dt=16.0, nod=1, band=2880, dets=("H1",), seed=99, thr=7.0, fftpad=2,
        gtype="directed_range", gcenter=(100.0152, -2e-10, 1.2, 0.3),
        gsizes=(1800, 3.0, 0.0, 0.0), gsteps=(1, 1.0, 1.0, 1.0),
        injections=(synth.Injection(f=100.0152, fdot=-2e-10, ra=1.2, dec=0.3, iota=0.2, psi=0.5,
                                    phase=0.4, snr=25.0),)),
    # all-sky grid (spindown range from Smin/Smax per sky point, both
    # hemispheres) with blocks_avg F-statistic normalisation
    "g3_allsky_blocks": synth.Case(
        dt=8.0, nod=1, band=1440, dets=("H1", "L1"), sigma=(1.0, 1.0), seed=33, thr=9.0,
        fdot_step=1e-9, sky_cells=3.0, gtype="allsky", fstat_norm="blocks_avg"),
}


# Veto-line generation alone (the reference's vlinegen program): the veto
# file each case's band gets from its line lists
VLINE_CASES = {
    "v1_band100": CASES["g5_vlines"],
    # no narrow-down (narrowdown = pi/2), one detector's lists in two files
    "v2_band250": synth.Case(
        dt=8.0, nod=1, band=3840, dets=("H1", "L1"), seed=77, narrowdown=0.5, veto_flag=0,
        line_files=LINE_FILES_250HZ, gtype="directed_range"),
    # no line lists at all: an empty veto file with fraction 0
    "v3_nolists": synth.Case(dt=8.0, nod=1, band=1440, dets=("H1",), seed=78, narrowdown=0.3),
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
