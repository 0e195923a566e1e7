"""Coincidences between segments (tdf_coincidences, include/tdfcuda.h): the
coincidence search of the reference's coincidences/coincidences.c over the
records of several segments' searches of the same templates."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import _abi
from .engine import _REC_DTYPE, _check, load_library


@dataclass
class CoincOptions:
    """[coincidences] options (coincidences/io.c:86-154)."""
    refr: int
    cthr: float
    scalef: int = 1
    scales: int = 1
    scalem: int = 1
    scalen: int = 1
    mincoin: int = 4
    shift: Optional[int] = None     # None: all 16 cell shifts; else 0..15 (bits m,n,s,f = 8,4,2,1)


@dataclass
class Segment:
    """One segment's search: its records (as Engine.search returns them or as
    read from a trigger file) and the settings the reference reads with them."""
    seg: int
    N: int
    nfftf: int
    dt: float
    narrowdown: float
    hdr: np.ndarray                 # (nrec, 6) float32: m, n, s, ra, dec, fdot
    pairs: List[np.ndarray]         # per record: interleaved (f, F) float32
    lines: np.ndarray = field(default_factory=lambda: np.zeros((0, 2)))


@dataclass
class Coincidence:
    shift: int
    w: int
    avg_snr: float
    avg_f: float
    avg_fdot: float
    avg_ra: float
    avg_dec: float
    cseg: np.ndarray                # segment indices (0-based, into the segment list)
    trig: np.ndarray                # template indices
    ntrig: np.ndarray               # triggers in the cell per segment


def coincidences(opts: CoincOptions, segments: Sequence[Segment]):
    """Runs tdf_coincidences; returns (coincidences in output order, seginfo
    array [nshift][nseg][3])."""
    lib = load_library()
    o = _abi.TdfCoincOpts(opts.refr, opts.cthr, opts.scalef, opts.scales, opts.scalem, opts.scalen, opts.mincoin,
                          -1 if opts.shift is None else opts.shift)
    keep = []
    segs = (_abi.TdfCoincSegment * len(segments))()
    for k, s in enumerate(segments):
        n = len(s.hdr)
        lens = np.array([len(p) for p in s.pairs], dtype=np.int64)
        offs = np.zeros(n, dtype=np.int64)
        if n:
            offs[1:] = np.cumsum(lens)[:-1]
        flat = np.concatenate([np.asarray(p, np.float32) for p in s.pairs]) if n and lens.sum() else np.zeros(1, np.float32)
        rec = np.zeros(max(n, 1), dtype=_REC_DTYPE)
        for i, name in enumerate(("m", "n", "s", "ra", "dec", "fdot")):
            rec[name][:n] = s.hdr[:, i]
        rec["len"][:n] = lens
        rec["offset"][:n] = offs
        lines = np.ascontiguousarray(s.lines, dtype=np.float64).reshape(-1, 2)
        keep += [rec, flat, lines]
        segs[k].seg, segs[k].N, segs[k].nfftf = s.seg, s.N, s.nfftf
        segs[k].dt, segs[k].narrowdown = s.dt, s.narrowdown
        segs[k].nlines = len(lines)
        segs[k].lines = lines.ctypes.data_as(C.POINTER(C.c_double)) if len(lines) else None
        segs[k].nrec = n
        segs[k].recs = C.cast(rec.ctypes.data, C.POINTER(_abi.TdfRecord))
        segs[k].pairs = flat.ctypes.data_as(C.POINTER(C.c_float))
    nshift = 16 if opts.shift is None else 1
    seginfo = np.zeros((nshift, len(segments), 3), dtype=np.int32)
    ncoi, nmem = C.c_int64(0), C.c_int64(0)
    st = lib.tdf_coincidences(C.byref(o), len(segments), segs, None, 0, C.byref(ncoi), None, None, None, 0,
                              C.byref(nmem), seginfo.ctypes.data_as(C.POINTER(C.c_int32)))
    if st not in (_abi.TDF_OK, _abi.TDF_ERR_CAPACITY):
        _check(lib, st)
    coi = (_abi.TdfCoincidence * max(ncoi.value, 1))()
    cseg = np.zeros(max(nmem.value, 1), dtype=np.int16)
    trig = np.zeros(max(nmem.value, 1), dtype=np.int32)
    ntrig = np.zeros(max(nmem.value, 1), dtype=np.int16)
    _check(lib, lib.tdf_coincidences(C.byref(o), len(segments), segs, coi, ncoi.value, C.byref(ncoi),
                                     cseg.ctypes.data_as(C.POINTER(C.c_int16)),
                                     trig.ctypes.data_as(C.POINTER(C.c_int32)),
                                     ntrig.ctypes.data_as(C.POINTER(C.c_int16)), nmem.value, C.byref(nmem),
                                     seginfo.ctypes.data_as(C.POINTER(C.c_int32))))
    out = []
    for i in range(ncoi.value):
        c = coi[i]
        a, b = c.member, c.member + c.w
        out.append(Coincidence(c.shift, c.w, np.float32(c.avg_snr), np.float32(c.avg_f), np.float32(c.avg_fdot),
                               np.float32(c.avg_ra), np.float32(c.avg_dec), cseg[a:b].copy(), trig[a:b].copy(),
                               ntrig[a:b].copy()))
    return out, seginfo
