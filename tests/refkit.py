"""Test-side helpers: run the reference build, read its trigger files, load
the CPU oracle restatement, compare record sets.

Only tests/ (and the smoke check / bench CPU leg) use this module; it is the
checker side of the parity tests.
"""
from __future__ import annotations

import ctypes as C
import glob
import os
import struct
import re
import subprocess
from typing import Dict, List, Optional, Tuple

import numpy as np

from tdfstat_b200 import _abi

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(REPO, "oracle")
REF_BIN = {
    "f64": os.path.join(ORACLE_DIR, "_ref", "gwsearch-ref-f64"),
    "f32": os.path.join(ORACLE_DIR, "_ref", "gwsearch-ref-f32"),
    "dropin": os.path.join(ORACLE_DIR, "_ref", "gwsearch-dropin"),
    "coinc": os.path.join(ORACLE_DIR, "_ref", "coinc-ref"),
    "vlinegen": os.path.join(ORACLE_DIR, "_ref", "vlinegen-ref"),
}
ORACLE_LIB = os.path.join(ORACLE_DIR, "libtdforacle.so")


# ------------------------------------------------------------------ records

class Records:
    """A set of trigger records: header arrays plus per-record (f, F) pairs."""

    def __init__(self, hdr: np.ndarray, pairs: List[np.ndarray], pm: Optional[np.ndarray] = None):
        self.hdr = np.asarray(hdr, dtype=np.float32).reshape(-1, 6)   # m n s ra dec fdot
        self.pairs = pairs
        self.pm = pm if pm is not None else np.zeros(len(self.hdr), dtype=np.int32)

    def __len__(self):
        return len(self.hdr)

    @property
    def ntrig(self) -> int:
        return sum(len(p) // 2 for p in self.pairs)

    @staticmethod
    def from_abi(recs, nrec: int, pairs: np.ndarray, pm: Optional[np.ndarray] = None) -> "Records":
        hdr = np.zeros((nrec, 6), dtype=np.float32)
        pl = []
        for i in range(nrec):
            r = recs[i]
            hdr[i] = (r.m, r.n, r.s, r.ra, r.dec, r.fdot)
            pl.append(np.array(pairs[r.offset: r.offset + r.len], dtype=np.float32))
        return Records(hdr, pl, pm)

    def triggers(self) -> np.ndarray:
        """All triggers as rows (record index, f, F)."""
        rows = []
        for i, p in enumerate(self.pairs):
            for k in range(0, len(p), 2):
                rows.append((i, p[k], p[k + 1]))
        return np.array(rows, dtype=np.float64).reshape(-1, 3)


def read_trigger_file(path: str) -> Tuple[Records, Dict]:
    """Reads the flat trigger file written by oracle/ref_io.c."""
    with open(path, "rb") as f:
        data = f.read()
    assert data[:8] in (b"TDFTRIG2", b"TDFTRIG3"), path
    ver, nifo = struct.unpack_from("<ii", data, 8)
    off = 16
    hdrs, pairs = [], []
    meta = {"format_version": ver, "nifo": nifo}
    if ver >= 3:
        band, seg, hemi = struct.unpack_from("<3i", data, off)
        overlap, narrowdown = struct.unpack_from("<2d", data, off + 12)
        gl = struct.unpack_from("<I", data, off + 28)[0]
        grid_file = data[off + 32: off + 32 + gl].decode()
        off += 32 + gl
        fpo, dt, B = struct.unpack_from("<3d", data, off)
        nod, N, nfftf, numlines_band, nvl = struct.unpack_from("<5i", data, off + 24)
        off += 44
        meta.update(band=band, seg=seg, hemi=hemi, overlap=overlap, narrowdown=narrowdown, grid_file=grid_file,
                    fpo=fpo, dt=dt, B=B, nod=nod, N=N, nfftf=nfftf, numlines_band=numlines_band,
                    nvlines_all_inband=nvl)
    while off < len(data):
        h = struct.unpack_from("<6f", data, off)
        ln = struct.unpack_from("<I", data, off + 24)[0]
        off += 28
        if ln == 0xFFFFFFFF:
            ts, wt, nt = struct.unpack_from("<idi", data, off)
            meta.update(totsgnl=ts, walltime=wt, num_threads=nt)
            break
        p = np.frombuffer(data, dtype="<f4", count=ln, offset=off).copy()
        off += 4 * ln
        hdrs.append(h)
        pairs.append(p)
    return Records(np.array(hdrs, dtype=np.float32).reshape(-1, 6), pairs), meta


def read_coin_file(path: str) -> Dict[int, Dict]:
    """Reads the flat coincidence file of oracle/coinc_io.c: per shift (as
    the integer of its 'mnsf' bit string) its seginfo [nseg][3] and its
    coincidences (w, avg_snr, avg_f, avg_fdot, avg_ra, avg_dec, cseg, trig,
    ntrig) in file order."""
    with open(path, "rb") as f:
        data = f.read()
    assert data[:8] == b"TDFCOIN1", path
    nseg = struct.unpack_from("<i", data, 8)[0]
    off = 12
    out = {}
    while off < len(data):
        shift = int(data[off:off + 4].decode(), 2)
        icoi = struct.unpack_from("<i", data, off + 5)[0]
        off += 9
        seginfo = np.frombuffer(data, dtype="<i4", count=3 * nseg, offset=off).reshape(nseg, 3).copy()
        off += 12 * nseg
        cois = []
        for _ in range(icoi):
            w = struct.unpack_from("<h", data, off)[0]
            vals = struct.unpack_from("<5f", data, off + 2)
            off += 22
            cseg = np.frombuffer(data, dtype="<i2", count=w, offset=off).copy()
            off += 2 * w
            trig = np.frombuffer(data, dtype="<i4", count=w, offset=off).copy()
            off += 4 * w
            ntrig = np.frombuffer(data, dtype="<i2", count=w, offset=off).copy()
            off += 2 * w
            cois.append((w,) + tuple(np.float32(v) for v in vals) + (cseg, trig, ntrig))
        out[shift] = {"seginfo": seginfo, "coi": cois}
    return out


def _big_stack():
    """extract_band_vlines() keeps ~17 MB of arrays on the stack
    (common.c:172-182) and job_core() a [nifo][N] VLA (jobcore.c:211):
    raise the soft stack limit for the reference process."""
    import resource
    soft, hard = resource.getrlimit(resource.RLIMIT_STACK)
    want = 256 << 20
    if hard != resource.RLIM_INFINITY:
        want = min(want, hard)
    resource.setrlimit(resource.RLIMIT_STACK, (want, hard))


def run_reference(ini: str, which: str = "f64", threads: int = 1, timeout: float = 3600,
                  env: Optional[Dict[str, str]] = None) -> Tuple[Records, Dict, str]:
    """Runs a reference build on `ini` (cwd = the INI's directory); returns
    the records of all hemisphere files (in pm order), meta and stdout."""
    wd = os.path.dirname(os.path.abspath(ini))
    e = dict(os.environ)
    e["OMP_NUM_THREADS"] = str(threads)
    if env:
        e.update(env)
    out = subprocess.run([REF_BIN[which], os.path.basename(ini)], cwd=wd, env=e,
                         capture_output=True, text=True, timeout=timeout, preexec_fn=_big_stack)
    if out.returncode != 0:
        raise RuntimeError("reference failed (%d):\n%s\n%s" % (out.returncode, out.stdout[-3000:], out.stderr[-3000:]))
    files = sorted(glob.glob(os.path.join(wd, "out", "triggers_*.h5")))
    hdrs, pairs, pms = [], [], []
    meta = {"walltime": 0.0, "totsgnl": 0}
    for fn in files:
        pm = int(fn.rsplit("_", 1)[1].split(".")[0])
        r, m = read_trigger_file(fn)
        hdrs.append(r.hdr)
        pairs += r.pairs
        pms.append(np.full(len(r), pm, dtype=np.int32))
        meta["walltime"] += m.get("walltime", 0.0)
        meta["totsgnl"] += m.get("totsgnl", 0)
        meta["num_threads"] = m.get("num_threads", 0)
    hdr = np.concatenate(hdrs) if hdrs else np.zeros((0, 6), np.float32)
    pm = np.concatenate(pms) if pms else np.zeros(0, np.int32)
    return Records(hdr, pairs, pm), meta, out.stdout


def run_vlinegen(ini: str, timeout: float = 600) -> str:
    """Runs the reference's veto-line generator (vlinegen.c) on `ini`
    (cwd = the INI's directory); returns the text of the veto file it wrote."""
    wd = os.path.dirname(os.path.abspath(ini))
    out = subprocess.run([REF_BIN["vlinegen"], os.path.basename(ini)], cwd=wd, capture_output=True,
                         text=True, timeout=timeout, preexec_fn=_big_stack)
    if out.returncode != 0:
        raise RuntimeError("vlinegen failed (%d):\n%s" % (out.returncode, out.stdout[-3000:]))
    m = re.search(r"Wrote veto lines in band to: (\S+)", out.stdout)
    with open(os.path.join(wd, m.group(1)), encoding="latin-1") as f:
        return f.read()


# ------------------------------------------------------------------ oracle

def build_oracle(ref: bool = False):
    targets = ["restatement"] + (["ref"] if ref else [])
    subprocess.run(["make", "-s", "-C", ORACLE_DIR] + targets, check=True)


def load_oracle():
    if not os.path.exists(ORACLE_LIB):
        build_oracle()
    lib = C.CDLL(ORACLE_LIB)
    lib.orc_search_points.restype = C.c_int
    lib.orc_search_points.argtypes = [C.POINTER(_abi.TdfSegment), C.POINTER(_abi.TdfSearchOpts), C.c_int,
                                      _abi.I32P, _abi.F32P, _abi.F32P, _abi.F32P,
                                      _abi.RECP, C.c_int64, _abi.I64P, _abi.F32P, C.c_int64, _abi.I64P, _abi.I32P]
    lib.orc_fstat_spectrum.restype = C.c_int
    lib.orc_fstat_spectrum.argtypes = [C.POINTER(_abi.TdfSegment), C.POINTER(_abi.TdfSearchOpts), C.c_int32,
                                       C.c_float, C.c_float, C.c_float, _abi.F64P, C.c_int64]
    lib.orc_fft.restype = C.c_int
    lib.orc_fft.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p]
    lib.orc_splintpad.restype = None
    lib.orc_splintpad.argtypes = [C.c_void_p, _abi.F64P, C.c_int, C.c_int, C.c_void_p]
    lib.orc_add_signal.restype = C.c_int
    lib.orc_add_signal.argtypes = [C.c_void_p, C.POINTER(_abi.TdfSignal), C.POINTER(C.c_double)]
    lib.orc_add_signal_out.restype = C.c_int
    lib.orc_add_signal_out.argtypes = [C.c_void_p, C.POINTER(_abi.TdfSignal), C.POINTER(C.c_double), _abi.F64P]
    return lib


class OracleSegment:
    """job.segment() for the oracle, with the job's signal file (if any)
    injected by orc_add_signal into copies of the xDat arrays, as the
    reference's main() does before its search (main.c:101-104).  Keep the
    object alive while the segment is used."""

    def __init__(self, job, oracle):
        self.seg = job.segment()
        self.h0 = None
        self.xdat = []
        if job.signal is not None:
            for n in range(self.seg.nifo):
                x = np.array(job.dets[n].xdat, dtype=np.float32, copy=True)
                self.xdat.append(x)
                self.seg.det[n].xdat = x.ctypes.data_as(C.POINTER(C.c_float))
            h0 = C.c_double(0.0)
            self.signal = np.zeros((self.seg.nifo, self.seg.N), dtype=np.float64)
            assert oracle.orc_add_signal_out(C.byref(self.seg), C.byref(job.signal), C.byref(h0),
                                             self.signal.ctypes.data_as(C.POINTER(C.c_double))) == 0
            self.h0 = h0.value


def reference_signal_files(ini: str):
    """Runs the reference FP64 build on `ini` (its mods holding write_signal)
    and returns {file name: text} of what it wrote to out/injections."""
    run_reference(ini, "f64", threads=1)
    d = os.path.join(os.path.dirname(os.path.abspath(ini)), "out", "injections")
    out = {}
    for fn in sorted(os.listdir(d)):
        with open(os.path.join(d, fn)) as f:
            out[fn] = f.read()
    return out


def engine_for(job, form="split", **kw):
    """Engine.from_job plus the job's signal injected on the device."""
    from tdfstat_b200.engine import Engine
    eng = Engine.from_job(job, form=form, **kw)
    if job.signal is not None:
        h0, inband = eng.add_signal(job.signal)
        assert inband
    return eng


def _ptr(a, t):
    return a.ctypes.data_as(C.POINTER(t))


def search_points(fn, seg, opts, pm, mm, nn, sst=None, max_recs=None, max_pairs=None, engine=None):
    """Calls orc_search_points / tdf_search_points with numpy inputs;
    returns (status, Records, nrec_per_point)."""
    pm = np.ascontiguousarray(pm, dtype=np.int32)
    mm = np.ascontiguousarray(mm, dtype=np.float32)
    nn = np.ascontiguousarray(nn, dtype=np.float32)
    npts = len(pm)
    sp = None if sst is None else _ptr(np.ascontiguousarray(sst, dtype=np.float32), C.c_float)
    if max_recs is None:
        max_recs = max(1, npts * 4096)
    if max_pairs is None:
        max_pairs = 1 << 22
    recs = (_abi.TdfRecord * max_recs)()
    pairs = np.zeros(max_pairs, dtype=np.float32)
    nrec = C.c_int64(0)
    npairs = C.c_int64(0)
    per = np.zeros(npts, dtype=np.int32)
    head = [engine] if engine is not None else [C.byref(seg), C.byref(opts)]
    st = fn(*head, npts, _ptr(pm, C.c_int32), _ptr(mm, C.c_float), _ptr(nn, C.c_float), sp,
            recs, max_recs, C.byref(nrec), _ptr(pairs, C.c_float), max_pairs, C.byref(npairs),
            _ptr(per, C.c_int32))
    n = min(nrec.value, max_recs)
    rpm = np.repeat(pm, per) if st == 0 else None
    return st, Records.from_abi(recs, n, pairs, rpm), per


# ------------------------------------------------------------------ comparison

def compare_records(a: Records, b: Records, f_rtol: float, F_rtol: float, thr: float,
                    tie_band: float = 1e-4) -> Dict:
    """Compares two record sets of the same templates.  Headers must agree
    exactly for m, n, s and to f32 rounding for ra, dec, fdot.  Triggers are
    matched per record by frequency; a trigger present in one set only must
    lie within tie_band (relative) of thr, or be a neighbour-tie case (its F
    within tie_band of the other set's local maximum structure).  Returns a
    summary dict with 'unmatched' listing unexplained differences."""
    assert len(a) == len(b), (len(a), len(b))
    out = {"max_F_rel": 0.0, "max_f_rel": 0.0, "matched": 0, "only_a": 0, "only_b": 0, "unmatched": []}
    np.testing.assert_array_equal(a.hdr[:, :3], b.hdr[:, :3])
    np.testing.assert_allclose(a.hdr[:, 3:], b.hdr[:, 3:], rtol=2e-6, atol=1e-30)
    for i in range(len(a)):
        pa = a.pairs[i].reshape(-1, 2).astype(np.float64)
        pb = b.pairs[i].reshape(-1, 2).astype(np.float64)
        used = np.zeros(len(pb), dtype=bool)
        for fa, Fa in pa:
            if len(pb):
                d = np.abs(pb[:, 0] - fa)
                d[used] = np.inf
                k = int(np.argmin(d))
                if d[k] <= f_rtol * max(abs(fa), 1.0):
                    used[k] = True
                    out["matched"] += 1
                    out["max_F_rel"] = max(out["max_F_rel"], abs(pb[k, 1] - Fa) / abs(Fa))
                    out["max_f_rel"] = max(out["max_f_rel"], d[k] / max(abs(fa), 1e-30))
                    continue
            out["only_a"] += 1
            if abs(Fa - thr) > tie_band * thr:
                out["unmatched"].append(("a", i, fa, Fa))
        for k in np.nonzero(~used)[0]:
            out["only_b"] += 1
            fb, Fb = pb[k]
            if abs(Fb - thr) > tie_band * thr:
                out["unmatched"].append(("b", i, fb, Fb))
    return out
