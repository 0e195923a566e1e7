"""Python binding of libtdfcuda (include/tdfcuda.h) through ctypes.

There is no CPU fallback: if the library is missing or no CUDA device is
present, construction raises.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional, Tuple

import numpy as np

from . import _abi

_LIB = None
_REC_DTYPE = np.dtype([("m", "<f4"), ("n", "<f4"), ("s", "<f4"), ("ra", "<f4"), ("dec", "<f4"), ("fdot", "<f4"),
                       ("len", "<u4"), ("pad", "<u4"), ("offset", "<i8")])
assert _REC_DTYPE.itemsize == C.sizeof(_abi.TdfRecord)


def load_library(path: Optional[str] = None):
    """Loads (once) the in-tree libtdfcuda.so and binds its ABI."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    p = path or _abi.LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError("libtdfcuda.so not built: run python -m tdfstat_b200.build (%s missing)" % p)
    lib = _abi.bind(C.CDLL(p))
    if path is None:
        _LIB = lib
    return lib


class TdfError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__("tdfcuda status %d: %s" % (status, msg))
        self.status = status


def _check(lib, st: int):
    if st != _abi.TDF_OK:
        raise TdfError(st, lib.tdf_last_error().decode() or lib.tdf_status_string(st).decode())


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


def device_count() -> int:
    lib = load_library()
    n = C.c_int32(0)
    st = lib.tdf_device_count(C.byref(n))
    return n.value if st == 0 else 0


class Result:
    """Records of a search call: headers (m, n, s, ra, dec, fdot), per-record
    (f, F) pairs and the per-point record counts (the *FNum increments)."""

    def __init__(self, hdr: np.ndarray, lens: np.ndarray, offsets: np.ndarray, pairs: np.ndarray, per_point: np.ndarray):
        self.hdr = hdr
        self.lens = lens
        self.offsets = offsets
        self.pairs_flat = pairs
        self.per_point = per_point

    def __len__(self):
        return len(self.hdr)

    @property
    def pairs(self):
        return [self.pairs_flat[o: o + n] for o, n in zip(self.offsets, self.lens)]

    @property
    def ntrig(self) -> int:
        return int(self.lens.sum() // 2)


class Engine:
    """One data segment resident on one GPU (tdf_engine_create)."""

    def __init__(self, segment: _abi.TdfSegment, opts: _abi.TdfSearchOpts, form: str = "split",
                 device: int = 0, max_sky_batch: int = 0):
        self.lib = load_library()
        self.form = form
        h = C.c_void_p()
        st = self.lib.tdf_engine_create(C.byref(segment), C.byref(opts), _abi.FORMS[form], device,
                                        max_sky_batch, C.byref(h))
        _check(self.lib, st)
        self.h = h
        self.nF = opts.fr[1] - opts.fr[0] + 1

    @classmethod
    def from_job(cls, job, form: Optional[str] = None, device: Optional[int] = None,
                 max_sky_batch: Optional[int] = None) -> "Engine":
        """An engine for a host.Job; arguments left out come from the job's
        INI [gpu] section (host.GpuOptions), else split form on device 0."""
        g = getattr(job, "gpu", None)
        form = form if form is not None else (g.form if g else "split")
        device = device if device is not None else (g.device if g else 0)
        max_sky_batch = max_sky_batch if max_sky_batch is not None else (g.sky_batch if g else 0)
        e = cls(job.segment(), job.search_opts(), form=form, device=device, max_sky_batch=max_sky_batch)
        e.job = job
        if g and g.templates_per_chunk:
            e.templates_per_chunk = g.templates_per_chunk
        return e

    def close(self):
        if getattr(self, "h", None):
            self.lib.tdf_engine_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload(self, segment: _abi.TdfSegment):
        _check(self.lib, self.lib.tdf_engine_upload(self.h, C.byref(segment)))

    def search(self, pm, mm, nn, sst=None, max_recs: Optional[int] = None, max_pairs: Optional[int] = None) -> Result:
        pm = np.ascontiguousarray(pm, dtype=np.int32)
        mm = np.ascontiguousarray(mm, dtype=np.float32)
        nn = np.ascontiguousarray(nn, dtype=np.float32)
        sp = None if sst is None else _p(np.ascontiguousarray(sst, dtype=np.float32), C.c_float)
        npts = len(pm)
        per = np.zeros(max(npts, 1), dtype=np.int32)
        nrec, npairs = C.c_int64(0), C.c_int64(0)
        if max_recs is None:
            _check(self.lib, self.lib.tdf_count_templates(self.h, npts, _p(pm, C.c_int32), _p(mm, C.c_float),
                                                          _p(nn, C.c_float), sp, C.byref(nrec), None))
            mr = nrec.value
        else:
            mr = max_recs
        mp = max_pairs if max_pairs is not None else 8 * mr + 4096
        recs = (_abi.TdfRecord * max(mr, 1))()
        pairs = np.empty(max(mp, 1), dtype=np.float32)
        st = self.lib.tdf_search_points(self.h, npts, _p(pm, C.c_int32), _p(mm, C.c_float), _p(nn, C.c_float), sp,
                                        recs, mr, C.byref(nrec), _p(pairs, C.c_float), mp, C.byref(npairs),
                                        _p(per, C.c_int32))
        if st == _abi.TDF_ERR_CAPACITY and (max_recs is None or max_pairs is None):
            # the engine kept the results: fetch them into arrays of the right size
            mr, mp = nrec.value, npairs.value
            recs = (_abi.TdfRecord * max(mr, 1))()
            pairs = np.empty(max(mp, 1), dtype=np.float32)
            st = self.lib.tdf_last_results(self.h, recs, mr, C.byref(nrec), _p(pairs, C.c_float), mp,
                                           C.byref(npairs), _p(per, C.c_int32))
        _check(self.lib, st)
        n = nrec.value
        a = np.frombuffer(memoryview(recs), dtype=_REC_DTYPE)[:n]
        hdr = np.stack([a["m"], a["n"], a["s"], a["ra"], a["dec"], a["fdot"]], axis=1) if n else np.zeros((0, 6), np.float32)
        return Result(hdr.astype(np.float32), a["len"].astype(np.int64), a["offset"].astype(np.int64),
                      pairs[: npairs.value].copy(), per[:npts].copy())

    def search_device(self, pm, mm, nn, sst=None) -> Tuple[int, int]:
        """Device-only pass; returns (records, triggers)."""
        pm = np.ascontiguousarray(pm, dtype=np.int32)
        mm = np.ascontiguousarray(mm, dtype=np.float32)
        nn = np.ascontiguousarray(nn, dtype=np.float32)
        sp = None if sst is None else _p(np.ascontiguousarray(sst, dtype=np.float32), C.c_float)
        nrec, ntrig = C.c_int64(0), C.c_int64(0)
        st = self.lib.tdf_search_points_device(self.h, len(pm), _p(pm, C.c_int32), _p(mm, C.c_float), _p(nn, C.c_float),
                                               sp, C.byref(nrec), C.byref(ntrig))
        _check(self.lib, st)
        return nrec.value, ntrig.value

    def add_segment(self, segment: _abi.TdfSegment) -> int:
        """Uploads another segment of the engine's sizes; returns its slot."""
        slot = C.c_int32(0)
        _check(self.lib, self.lib.tdf_engine_add_segment(self.h, C.byref(segment), C.byref(slot)))
        return slot.value

    def upload_segment(self, slot: int, segment: _abi.TdfSegment):
        _check(self.lib, self.lib.tdf_engine_upload_segment(self.h, int(slot), C.byref(segment)))

    def search_segments_device(self, slots, npts, pm, mm, nn) -> Tuple[int, int]:
        """Device-only pass over several resident segments (slot k searches
        npts[k] of the points, in order); returns (records, triggers)."""
        slots = np.ascontiguousarray(slots, dtype=np.int32)
        npts = np.ascontiguousarray(npts, dtype=np.int32)
        pm = np.ascontiguousarray(pm, dtype=np.int32)
        mm = np.ascontiguousarray(mm, dtype=np.float32)
        nn = np.ascontiguousarray(nn, dtype=np.float32)
        assert int(npts.sum()) == len(pm) == len(mm) == len(nn)
        nrec, ntrig = C.c_int64(0), C.c_int64(0)
        st = self.lib.tdf_search_segments_device(self.h, len(slots), _p(slots, C.c_int32), _p(npts, C.c_int32),
                                                 _p(pm, C.c_int32), _p(mm, C.c_float), _p(nn, C.c_float),
                                                 C.byref(nrec), C.byref(ntrig))
        _check(self.lib, st)
        return nrec.value, ntrig.value

    def fstat(self, pm: int, mm: float, nn: float, ss: float) -> np.ndarray:
        F = np.zeros(self.nF, dtype=np.float64)
        st = self.lib.tdf_fstat_spectrum(self.h, int(pm), float(mm), float(nn), float(ss), _p(F, C.c_double), len(F))
        _check(self.lib, st)
        return F

    def add_signal(self, sig: _abi.TdfSignal) -> Tuple[float, bool]:
        """Injects a CW signal into the resident data (add_signal, init.c:365-504);
        returns (h0 used, whether the signal was in band)."""
        h0, inb = C.c_double(0.0), C.c_int32(0)
        _check(self.lib, self.lib.tdf_engine_add_signal(self.h, C.byref(sig), C.byref(h0), C.byref(inb)))
        return h0.value, bool(inb.value)

    def signal(self, det: int, N: int) -> np.ndarray:
        """h0*s_n[i] (N values) of the signal the last add_signal() injected
        into detector `det`, before the next search or upload."""
        out = np.zeros(N, dtype=np.float64)
        _check(self.lib, self.lib.tdf_engine_get_signal(self.h, int(det), _p(out, C.c_double), N))
        return out

    def inject(self, job) -> Tuple[float, bool]:
        """main.c:101-104 for a host.Job: injects job.signal (search:addsig)
        and, with mods=write_signal, writes the injected signal of every
        detector as the reference does (init.c:475-497)."""
        h0, inband = self.add_signal(job.signal)
        if inband and job.write_signal:
            from . import host
            host.write_signal_files(job, [self.signal(n, job.sett.N) for n in range(job.sett.nifo)])
        return h0, inband

    def xdat(self, det: int, n: int) -> np.ndarray:
        """The resident xDat of detector `det` (first n samples)."""
        x = np.zeros(n, dtype=np.float32)
        _check(self.lib, self.lib.tdf_engine_get_xdat(self.h, int(det), _p(x, C.c_float), n))
        return x

    def stream(self) -> int:
        s = C.c_void_p()
        _check(self.lib, self.lib.tdf_engine_get_stream(self.h, C.byref(s)))
        return s.value or 0

    def set_stream(self, stream_ptr: int):
        _check(self.lib, self.lib.tdf_engine_set_stream(self.h, C.c_void_p(stream_ptr)))

    def autotune(self, pm, mm, nn) -> int:
        """Times chunk sizes on these points and keeps the fastest."""
        pm = np.ascontiguousarray(pm, dtype=np.int32)
        mm = np.ascontiguousarray(mm, dtype=np.float32)
        nn = np.ascontiguousarray(nn, dtype=np.float32)
        best = C.c_int32(0)
        _check(self.lib, self.lib.tdf_engine_autotune(self.h, len(pm), _p(pm, C.c_int32), _p(mm, C.c_float),
                                                      _p(nn, C.c_float), C.byref(best)))
        return best.value

    def tuning(self) -> dict:
        """The launch configuration in use: templates per chunk, lanes,
        templates per resolve group."""
        tc, ln, gt = C.c_int32(0), C.c_int32(0), C.c_int32(0)
        _check(self.lib, self.lib.tdf_engine_get_tuning(self.h, C.byref(tc), C.byref(ln), C.byref(gt)))
        return {"templates_per_chunk": tc.value, "lanes": ln.value, "group_templates": gt.value}

    @property
    def templates_per_chunk(self) -> int:
        tc = C.c_int32(0)
        _check(self.lib, self.lib.tdf_engine_get_templates_per_chunk(self.h, C.byref(tc)))
        return tc.value

    @templates_per_chunk.setter
    def templates_per_chunk(self, tc: int):
        _check(self.lib, self.lib.tdf_engine_set_templates_per_chunk(self.h, int(tc)))

    def enable_kernel_timing(self, on: bool = True):
        _check(self.lib, self.lib.tdf_engine_set_kernel_timing(self.h, 1 if on else 0))

    def kernel_times(self) -> dict:
        k = _abi.TdfKernelTimes()
        _check(self.lib, self.lib.tdf_engine_get_kernel_times(self.h, C.byref(k)))
        return {f: getattr(k, f) for f, _ in _abi.TdfKernelTimes._fields_}

    def launch_count(self) -> int:
        n = C.c_int64(0)
        _check(self.lib, self.lib.tdf_engine_launch_count(self.h, C.byref(n)))
        return n.value
