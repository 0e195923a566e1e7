"""Veto lines of a band, mirroring TDFstat's host code for them
(search/network/openmp/common.c:155-553, main.c:78-94, vlinegen.c).

A search vetoes a trigger whose frequency falls inside one of the first
``numlines_band`` intervals of ``sett->lines`` (jobcore.c:576-583).  The
intervals are, in this order:

* the two narrow-down intervals at the band edges (narrow_down_band,
  common.c:433-445), when narrowdown < pi/2;
* the instrumental lines of the band, either read from
  ``<outdir>/vlines_<band><label>.dat`` when that file exists
  (read_band_vlines, common.c:477-553), or extracted from the line lists
  ``<indir>/lines/<det>lines*.csv`` of every detector and written to that
  file (extract_band_vlines, common.c:166-413).

The veto lines count in ``numlines_band`` only with ``veto_flag`` set.
Extraction widens every line by the largest frequency excursion the
demodulation can give it: the spindown range over the segment plus the
detector's velocity and its time derivative, both taken from DetSSB.

Floating-point expressions follow the reference's in order and in type
(doubles, except the veto fraction, which the reference keeps in a float),
so the file written here is the reference's text, character for character.
"""
from __future__ import annotations

import glob as _glob
import math
import os
import re
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

MAXL = 512          # struct.h:14, veto intervals in a band
MAXVFILEL = 8192    # struct.h:15, data lines of all veto files together
MAXLINE = 1024      # struct.h:16, fgets buffer of the readers
VF_TAG = "#band_veto_fraction="
HEADER = "# fl[rad]  fr[rad]   fl[Hz]  fr[Hz]   line info\n"


class VlinesError(ValueError):
    """A condition on which the reference prints a message and exits."""


def narrow_down_lines(narrowdown: float) -> List[List[float]]:
    """narrow_down_band (common.c:433-445): [0, pi/2 - nd] and [pi/2 + nd, pi]."""
    return [[0.0, math.pi / 2 - narrowdown], [math.pi / 2 + narrowdown, math.pi]]


# ------------------------------------------------------------ C text parsing

_FLOAT = re.compile(r"[ \t\n\v\f\r]*([+-]?(?:inf(?:inity)?|nan|(?:\d+\.?\d*|\.\d+)(?:[eE][+-]?\d+)?))",
                    re.IGNORECASE)
_INT = re.compile(r"[ \t\n\v\f\r]*([+-]?\d+)")


def c_atof(s: str) -> float:
    """atof: the longest decimal prefix after white space, else 0."""
    m = _FLOAT.match(s)
    return float(m.group(1)) if m else 0.0


def c_atoi(s: str) -> int:
    """atoi: the longest integer prefix after white space, else 0."""
    m = _INT.match(s)
    return int(m.group(1)) if m else 0


def fgets_lines(path: str, size: int = MAXLINE):
    """The successive buffers `fgets(line, size, f)` returns: each text line,
    cut into pieces of at most size-1 characters."""
    with open(path, "r", newline="", encoding="latin-1") as f:
        text = f.read()
    for ln in re.split(r"(?<=\n)", text):
        while len(ln) > size - 1:
            yield ln[:size - 1]
            ln = ln[size - 1:]
        if ln:
            yield ln


# ------------------------------------------------------------ line lists

@dataclass
class VetoLine:
    """One data line of a veto file (common.c:173-183, columns :226-234):
    spacing or frequency [Hz], type (0 singlet, 1 comb of fixed width,
    2 comb of scaling width), offset of the first harmonic [Hz], first and
    last harmonic index, left and right width [Hz]."""
    f: float
    type: int
    offset: float
    iharm1: int
    iharm2: int
    lwidth: float
    rwidth: float
    det: int
    nline: int
    vfile: str


def read_veto_files(indir: str, det_names: Sequence[str], base: str = ".") -> List[VetoLine]:
    """The line lists of every detector, in the reference's order
    (common.c:213-269): detectors in network order, the files of the
    pattern ``<indir>/lines/<det>lines*.csv`` in glob's sorted order, data
    lines in file order; lines starting with '%' are comments.  Fields are
    cut as strtok(line, ",") cuts them (empty fields vanish) and converted
    with atof/atoi.  `indir` is the INI's string, relative to `base` when
    not absolute; `vfile` keeps the glob's path as the reference prints it."""
    out: List[VetoLine] = []
    for det, name in enumerate(det_names):
        pattern = "%s/lines/%slines*.csv" % (indir, name)
        full = pattern if os.path.isabs(pattern) else os.path.join(base, pattern)
        files = sorted(_glob.glob(full))
        for fp in files:
            # glob keeps the pattern's directory part as written
            vfile = pattern[:pattern.rfind("/") + 1] + os.path.basename(fp)
            nline = 0
            for line in fgets_lines(fp):
                nline += 1
                if line.startswith("%"):
                    continue
                tok = [t for t in line.split(",") if t]
                if len(tok) < 7:
                    raise VlinesError("%s:%d: %d fields, 7 needed" % (fp, nline, len(tok)))
                out.append(VetoLine(f=c_atof(tok[0]), type=c_atoi(tok[1]), offset=c_atof(tok[2]),
                                    iharm1=c_atoi(tok[3]), iharm2=c_atoi(tok[4]), lwidth=c_atof(tok[5]),
                                    rwidth=c_atof(tok[6]), det=det, nline=nline, vfile=vfile))
                if len(out) > MAXVFILEL - 1:
                    raise VlinesError("Too many lines in file %s, increase MAXVFILEL!" % fp)
    return out


def demodulation_broadening(detssb: np.ndarray, N: int, dt: float) -> Tuple[float, float]:
    """(normdEmax, normdtEmax) of one detector (common.c:196-211): the
    largest squared step of DetSSB between consecutive samples, and of
    DetSSB[i]*i*dt, over i < N-1."""
    e = np.asarray(detssb, dtype=np.float64)[:3 * N].reshape(N, 3)
    d = np.abs(e[1:] - e[:-1])
    dE = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
    i = np.arange(N - 1, dtype=np.float64)[:, None]
    t = np.abs(e[1:] * (i + 1.0) - e[:-1] * i) * dt
    dtE = (t[:, 0] * t[:, 0] + t[:, 1] * t[:, 1]) + t[:, 2] * t[:, 2]
    return float(max(0.0, dE.max(initial=0.0))), float(max(0.0, dtE.max(initial=0.0)))


def line_in_band(fl: float, fr: float, fpo: float, B: float) -> Optional[Tuple[float, float]]:
    """line_in_band (common.c:416-430): the interval clipped to [fpo, fpo+B],
    or None when it misses the band."""
    bs, be = fpo, fpo + B
    if not (fr < bs or fl > be):
        return (bs if fl < bs else fl), (be if fr > be else fr)
    return None


def lines_veto_fraction(lines: List[List[float]]) -> Tuple[float, List[List[float]]]:
    """lines_veto_fraction (common.c:448-474): sorts the intervals [rad] by
    (left, right) and returns the fraction of [0, pi] they cover, rounded to
    float as the reference stores it, with the sorted list."""
    srt = sorted(([a, b] for a, b in lines), key=lambda x: (x[0], x[1]))
    ll, gap = 0.0, 0.0
    for a, b in srt:
        if a >= ll:
            gap += a - ll
            ll = b
        elif ll < b:
            ll = b
    if ll < math.pi:
        gap += math.pi - ll
    vf = float(np.float32(float(np.float32(math.pi - gap)) / math.pi))
    return vf, srt


@dataclass
class BandVlines:
    """The result of extract_band_vlines/read_band_vlines: all intervals
    [rad] (narrow-down first), how many of them the search applies, the
    band's veto fraction and, for an extraction, the text written."""
    lines: List[List[float]]
    numlines_band: int
    nvlines_all_inband: int
    veto_fraction: float
    text: str = ""
    info: List[str] = field(default_factory=list)


def extract_band_vlines(fpo: float, B: float, N: int, dt: float, detssb: Sequence[np.ndarray],
                        det_names: Sequence[str], indir: str, narrow: List[List[float]],
                        veto_flag: int, out_path: Optional[str], base: str = ".") -> BandVlines:
    """extract_band_vlines (common.c:166-413).  `narrow` holds the
    narrow-down intervals already in the list (empty when narrowdown >= pi/2);
    `detssb[k]` is detector k's DetSSB (3N doubles).  Writes the band's veto
    file to `out_path` (when given) and returns the intervals."""
    from .host import get_fdot_range
    _, fdotmax = get_fdot_range(fpo, dt)
    brd = [demodulation_broadening(e, N, dt) for e in detssb]
    vls = read_veto_files(indir, det_names, base)
    hz: List[Tuple[float, float, str]] = []

    def add(fl, fr, info):
        c = line_in_band(fl, fr, fpo, B)
        if c is not None:
            hz.append((c[0], c[1], info))
            if len(narrow) + len(hz) > MAXL - 1:
                raise VlinesError("Too many lines, increase MAXL!")

    for v in vls:
        nde, ndte = brd[v.det]
        if v.type == 0:
            D = 2. * fdotmax * (N * dt + math.sqrt(ndte)) + v.f * math.sqrt(nde)
            add(v.f - v.lwidth - D, v.f + v.rwidth + D, "singlet          [l.%d]%s" % (v.nline, v.vfile))
        elif v.type in (1, 2):
            for k in range(v.iharm1, v.iharm2 + 1):
                lf = v.offset + k * v.f
                D = 2. * fdotmax * (N * dt + math.sqrt(ndte)) + lf * math.sqrt(nde)
                if v.type == 1:
                    add(lf - v.lwidth - D, lf + v.rwidth + D, "fcomb rank %4d  [l.%d]%s" % (k, v.nline, v.vfile))
                else:
                    add(lf - k * v.lwidth - D, lf + k * v.rwidth + D,
                        "scomb rank %4d  [l.%d]%s" % (k, v.nline, v.vfile))
    rad = [[(fl - fpo) / B * math.pi, (fr - fpo) / B * math.pi] for fl, fr, _ in hz]
    body = "".join("   %.15f  %.15f  %.15f  %.15f  %s\n" % (r[0], r[1], h[0], h[1], h[2])
                   for r, h in zip(rad, hz))
    vf, srt = lines_veto_fraction(rad)
    text = HEADER + body + "%s %6.4f\n" % (VF_TAG, vf)
    if out_path is not None:
        with open(out_path, "w", encoding="latin-1") as f:
            f.write(text)
    lines = [list(x) for x in narrow] + srt
    nall = len(lines)
    return BandVlines(lines=lines, numlines_band=nall if veto_flag else len(narrow), nvlines_all_inband=nall,
                      veto_fraction=vf, text=text, info=[h[2] for h in hz])


_TWO = re.compile(r"[ \t\n\v\f\r]*([+-]?(?:inf(?:inity)?|nan|(?:\d+\.?\d*|\.\d+)(?:[eE][+-]?\d+)?))"
                  r"[ \t\n\v\f\r]*([+-]?(?:inf(?:inity)?|nan|(?:\d+\.?\d*|\.\d+)(?:[eE][+-]?\d+)?))",
                  re.IGNORECASE)


def read_band_vlines(path: str, narrow: List[List[float]], veto_flag: int) -> BandVlines:
    """read_band_vlines (common.c:477-553): the veto file an extraction
    wrote.  Lines starting with the veto-fraction tag carry the fraction;
    other '#' lines are comments; every other line must start with two
    numbers (fl, fr in radians).  A missing fraction, an unparsable line or
    more than MAXL intervals are errors, as in the reference."""
    lines = [list(x) for x in narrow]
    vf = -1.0
    for lnum, line in enumerate(fgets_lines(path), 1):
        if line.startswith(VF_TAG):
            m = _FLOAT.match(line[len(VF_TAG):])
            if not m:
                raise VlinesError("Can't parse veto fraction in line %d of %s" % (lnum, path))
            vf = float(np.float32(float(m.group(1))))
            continue
        if line.startswith("#"):
            continue
        m = _TWO.match(line)
        if not m:
            raise VlinesError("Can't parse line %d of %s" % (lnum, path))
        lines.append([float(m.group(1)), float(m.group(2))])
        if len(lines) > MAXL - 1:
            raise VlinesError("Too many lines, increase MAXL!")
    if vf < 0.0:
        raise VlinesError("veto fraction missing in %s" % path)
    nall = len(lines)
    return BandVlines(lines=lines, numlines_band=nall if veto_flag else len(narrow), nvlines_all_inband=nall,
                      veto_fraction=vf)
