"""Benchmark of the coherent-search hot path (job_core chain) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl tdf|reference]
                    [--form split|fp64] [--workload cfg3|cfg2|cfg1|cfg4|cfg5]
                    [--sweep]

Workload (default cfg3, the precision form): H1+L1, 6-sidereal-day segment
at dt = 2 s (N = 258492, nfft = nfftf = 2^18, Ninterp = 2^19), seeded
Gaussian noise (sigma 1, 5% gaps) plus four injected CW signals, a 128 x 64
sky patch around the first injection x 401 spindowns = 3,284,992 templates,
F over bins [1024, 130048], thr 14.5.  A step searches one 1024-point slice
of the patch (410,624 templates); consecutive steps take the slices in turn,
so 8 steps cover the whole patch.  (cfg2: the 2-day segment, N = 86164,
nfftf = 2^17, a 32 x 32 patch searched whole in every step.)  Inputs are
synthetic (no public data set is used).

  value : templates/s with the segment resident in HBM (device-only pass:
          sky stage + spindown stage + trigger compaction), CUDA events on
          the engine's stream, barrier + synchronize around the K steps,
          max over ranks.
  e2e   : the same through the C ABI with host buffers: upload of the
          segment's inputs (xdat, DetSSB, aux arrays) and download of the
          records inside every step.
  fp64  : the plain FP64 form (the reference's PREC=DOUBLE arithmetic on the
          GPU) on the same slices, its own warm-up, timing and clock record.
  --impl reference: the reference's own C search (its unmodified sources,
          PREC=FLOAT, built by oracle/Makefile) on the host cores, each step
          a bounded sample (1 sky point x the spindowns) of the workload.
  --sweep (cfg5): one line per sky-patch size 2^10 .. 2^18 points x 801
          spindowns; sizes above --sweep-cap points are timed on their first
          --sweep-cap points (every template counted is searched).
Under torchrun (N > 1) every rank searches its own patch (the same region,
shifted by a fraction of a grid step per rank) as a contiguous shard of one
point list: weak scaling, no collective on the data path; the whole-job
value counts all ranks' templates; rank 0 prints the JSON line.
"""
from __future__ import annotations

import argparse
import csv
import json
import math
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "templates/s (sky x spindown) on 1 B200, split-prec vs plain FP64 @<=1e-4 F err"
UNIT = "templates/s"


# ------------------------------------------------------------------ workload

from tdfstat_b200.workloads import MultiWorkload, Workload, workload_case  # noqa: E402


# ------------------------------------------------------------------ clocks

class ClockSampler:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        if not shutil.which("nvidia-smi"):
            return
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        self.f = open(self.path, "w")
        self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                                      "--format=csv,noheader,nounits", "-lms", "200"],
                                     stdout=self.f, stderr=subprocess.DEVNULL)

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.f.close()
        rows = []
        with open(self.path) as f:
            for r in csv.reader(f):
                if len(r) >= 9:
                    rows.append([x.strip() for x in r])
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ------------------------------------------------------------------ helpers

def measured_peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def cpu_reference_sample(wl: Workload, root: str, npts: int, threads: int):
    """Runs the reference FLOAT build on `npts` sky points of the workload
    (directed_range patch of the same segment); returns (templates, seconds,
    binary kind)."""
    sys.path.insert(0, os.path.join(REPO, "tests"))
    import refkit
    from tdfstat_b200 import synth
    binp = refkit.REF_BIN["f32"]
    if not os.path.exists(binp):
        return None
    c = wl.case
    half = (wl.nspd - 1) // 2
    c.gsizes = (wl.job.sett.nfft // 4 - 1024, float(half), 0.0, float((npts - 1) // 2))
    c.gsteps = (1, 1.0, 1.0, 0.25)
    ini = synth.write_case(root, c)
    shutil.rmtree(os.path.join(root, "out"), ignore_errors=True)
    os.makedirs(os.path.join(root, "out"), exist_ok=True)
    recs, meta, _ = refkit.run_reference(ini, "f32", threads=threads)
    return len(recs), float(meta["walltime"])


def cpu_fft_proxy(nfftf: int, threads: int, ntmpl: int, secs: float):
    """The FFT share of a reference sample and the sample's rate with a
    library-grade FFT in place of the project shim (FFTW is absent here):
    2 single-precision transforms of nfftf per template (jobcore.c:477-478)
    timed with the shim as the reference binary has it (oracle/_ref/
    fft-time-f32: same flags, `threads` OpenMP threads, own process, half a
    second of warm-up, ~1 s timed) and with scipy.fft (pocketfft) batched
    the way a threaded host search would issue them: the 2 transforms of
    each of `threads` templates in one call with workers = threads.  The
    per-sky-point interpolation transforms (FP64, 4 per detector per point)
    are left in.  When the isolated shim time exceeds the sample's own time
    the share is reported as measured and no substituted rate is derived."""
    import time as _t
    import numpy as _np
    try:
        import scipy.fft as sfft
    except ImportError:
        return None
    exe = os.path.join(REPO, "oracle", "_ref", "fft-time-f32")
    if not os.path.exists(exe):
        return None
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    reps = max(20, int(1.0 / max(secs / max(ntmpl, 1) / 2, 1e-5)))   # ~1 s at the sample's pace
    r = subprocess.run([exe, str(nfftf), str(min(reps, 5000))], capture_output=True, text=True, env=env,
                       timeout=300)
    if r.returncode != 0:
        return None
    t_shim = float(r.stdout.split()[0])
    nb = 2 * max(1, threads)
    rng = _np.random.default_rng(0)
    x = (rng.standard_normal((nb, nfftf)) + 1j * rng.standard_normal((nb, nfftf))).astype(_np.complex64)
    t0 = _t.perf_counter()
    while _t.perf_counter() - t0 < 0.3:
        sfft.fft(x, axis=-1, workers=threads)
    n = 0
    t0 = _t.perf_counter()
    while _t.perf_counter() - t0 < 1.0:
        sfft.fft(x, axis=-1, workers=threads)
        n += 1
    t_sp = (_t.perf_counter() - t0) / (n * nb)   # seconds per transform, amortised over the batch
    fft_s = 2 * ntmpl * t_shim
    rest = secs - fft_s
    out = {"fft_share": round(fft_s / secs, 3), "shim_ms_per_fft": round(1e3 * t_shim, 3),
           "scipy_ms_per_fft": round(1e3 * t_sp, 4),
           "scipy_batch": "%d transforms per call, workers=%d" % (nb, threads)}
    if rest > 0:
        out["value_with_scipy_fft"] = round(ntmpl / (rest + 2 * ntmpl * t_sp), 2)
    else:
        out["value_with_scipy_fft"] = None
        out["note"] = "isolated shim FFT slower than inside the sample; no substituted rate"
    return out


# ------------------------------------------------------------------ arms

def _slices(pm, mm, nn, size):
    """The point list cut into consecutive slices of `size` points (the last
    may be shorter); step k searches slice k mod len."""
    size = len(pm) if size <= 0 else min(size, len(pm))
    return [(pm[i:i + size], mm[i:i + size], nn[i:i + size]) for i in range(0, len(pm), size)]


def _timed_steps(eng, stream, flush, slices, k0, steps, barrier, device):
    """`steps` device-only steps (slices k0, k0+1, ...) between CUDA events
    on the engine's stream, the 256 MiB L2 flush before each, clocks
    sampled during the region.  Returns (ms, templates, triggers, launches,
    clocks)."""
    import torch
    launches0 = eng.launch_count()
    clocks = ClockSampler(device)
    clocks.start()
    barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ntrig = nsearched = 0
    ev0.record(stream)
    for k in range(steps):
        with torch.cuda.stream(stream):
            flush.zero_()   # 256 MiB (> L2) written between steps, on the engine's stream
        pm, mm, nn = slices[(k0 + k) % len(slices)]
        nrec, nt = eng.search_device(pm, mm, nn)
        ntrig += nt
        nsearched += nrec
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    return ev0.elapsed_time(ev1), nsearched, ntrig, eng.launch_count() - launches0, clk


def run_tdf(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from tdfstat_b200.engine import Engine

    torch.cuda.set_device(local_rank)
    root = tempfile.mkdtemp(prefix="tdfbench_")
    try:
        wl = Workload(args.workload, root, world)
        job = wl.job
        pm, mm, nn = wl.shard(rank, world)
        if args.sky_points:
            pm, mm, nn = pm[:args.sky_points], mm[:args.sky_points], nn[:args.sky_points]
            wl.config["sky_points"] = len(pm)
            wl.config["templates_per_step"] = len(pm) * wl.nspd
        slice_pts = args.slice_points if args.slice_points is not None else (1024 if args.workload == "cfg3" else 0)
        slices = _slices(pm, mm, nn, slice_pts)
        seg, opts = job.segment(), job.search_opts()
        flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

        def barrier():
            if world > 1:
                dist.barrier()

        def reduce(vals, op):
            t = torch.tensor(vals, dtype=torch.float64, device="cuda")
            if world > 1:
                dist.all_reduce(t, op=op)
            return [float(v) for v in t]

        eng = Engine(seg, opts, form=args.form, device=local_rank, max_sky_batch=args.sky_batch)
        stream = torch.cuda.ExternalStream(eng.stream(), device=local_rank)
        # chunk size by the engine's autotuner on a 16-point sample (untimed)
        if not args.no_autotune:
            eng.autotune(pm[:16], mm[:16], nn[:16])
        tuned = eng.tuning()
        # warm-up steps are the timed step exactly (the flush included: its
        # first launch loads torch's fill kernel)
        for k in range(args.warmup):
            with torch.cuda.stream(stream):
                flush.zero_()
            eng.search_device(*slices[k % len(slices)])
        torch.cuda.synchronize()
        # ---- value: device-resident inputs, K steps
        ms, nsearched, ntrig, launches, clk = _timed_steps(eng, stream, flush, slices, 0, args.steps, barrier,
                                                           local_rank)
        if nsearched != sum(len(slices[k % len(slices)][0]) for k in range(args.steps)) * wl.nspd:
            print("bench: some patch points lie outside the sky grid", file=sys.stderr)
        # ---- per-kernel durations: one or two steps again at the run's own
        # chunk size, CUDA events recorded on the engine's stream around every
        # launch (kernels one after another: one lane)
        tc_run = eng.templates_per_chunk
        eng.enable_kernel_timing(True)
        for k in range(max(1, min(args.steps, 2))):
            with torch.cuda.stream(stream):
                flush.zero_()
            eng.search_device(*slices[k % len(slices)])
        torch.cuda.synchronize()
        ktimes = eng.kernel_times()
        eng.enable_kernel_timing(False)
        # ---- e2e: host buffers through the C ABI
        eng.upload(seg)
        eng.search(*slices[0])
        torch.cuda.synchronize()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        nsearched_e2e = 0
        d2h = 0
        for k in range(args.steps):
            eng.upload(seg)
            res = eng.search(*slices[k % len(slices)])
            nsearched_e2e += len(res)
            d2h += len(res) * 40 + res.pairs_flat.nbytes
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        ms_e2e = e0.elapsed_time(e1)
        h2d = sum(d.xdat.nbytes + d.detssb.nbytes for d in job.dets) + job.cosmodf.nbytes + job.sinmodf.nbytes \
            + sum(a.nbytes for a in slices[0])
        eng.close()
        # ---- the plain FP64 form on the same slices (its own engine)
        fp64 = None
        if args.form == "split" and not args.no_fp64:
            e64 = Engine(seg, opts, form="fp64", device=local_rank, max_sky_batch=args.sky_batch)
            s64 = torch.cuda.ExternalStream(e64.stream(), device=local_rank)
            # 48 templates per chunk: the autotuner's choice for this form at every size measured
            # (timing the candidates in FP64 would take minutes)
            e64.templates_per_chunk = t64 = 48
            k64 = max(1, min(args.steps, args.fp64_steps))
            for k in range(max(1, min(args.warmup, 2))):
                with torch.cuda.stream(s64):
                    flush.zero_()
                e64.search_device(*slices[k % len(slices)])
            torch.cuda.synchronize()
            ms64, n64, _, _, clk64 = _timed_steps(e64, s64, flush, slices, 0, k64, barrier, local_rank)
            e64.close()
            ms64, = reduce([ms64], dist.ReduceOp.MAX)
            n64, = reduce([n64], dist.ReduceOp.SUM)
            fp64 = {"value": round(n64 / (ms64 / 1e3), 1), "unit": UNIT, "steps": k64,
                    "ms_per_step": round(ms64 / k64, 3), "templates_per_chunk": t64, "clocks": clk64}
        # times: max over ranks; templates searched: sum over ranks
        ms, ms_e2e = reduce([ms, ms_e2e], dist.ReduceOp.MAX)
        nsum, nsum_e2e = reduce([nsearched, nsearched_e2e], dist.ReduceOp.SUM)
        value = nsum / (ms / 1e3)
        e2e = nsum_e2e / (ms_e2e / 1e3)
        out = None
        if rank == 0:
            peak, peak_kind = measured_peaks()
            nifo = len(job.dets)
            N = job.sett.N
            bt = nifo * N * (24 if args.form == "split" else 40)   # algorithmic bytes per template
            col_ms, col_n, col_t = ktimes["colpass_ms"], ktimes["colpass_launches"], ktimes["colpass_templates"]
            roof = None
            if col_n:
                per_launch_bytes = bt * col_t / col_n
                avg_s = col_ms / col_n / 1e3
                achieved = per_launch_bytes / avg_s / 1e9
                roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                        "frac": round(achieved / peak, 4), "traffic": None,
                        "kernel": ("k_spinpass (demodulation + both FFT passes + F, one ordered launch)"
                                   if col_n and not ktimes.get("rowpass_launches")
                                   else "k_colpass (demodulation + first FFT pass)"),
                        "peak_kind": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind,
                        "algorithmic_bytes_per_template": bt,
                        "kernel_ms": {k: round(v, 3) for k, v in ktimes.items() if k.endswith("_ms")},
                        "avg_launch_ms": round(col_ms / col_n, 4), "templates_per_launch": col_t / col_n,
                        "timed": "CUDA events on the engine stream around each launch, one lane, the run's "
                                 "%d templates per launch" % tc_run,
                        "traffic_note": "DRAM bytes are not counted in this run (no profiler in the timed "
                                        "process); ncu figures of the same kernel are kept under profiles/"}
            cpu = None
            if not args.no_cpu_baseline and world == 1:   # the CPU baseline is an N = 1 figure
                r = cpu_reference_sample(wl, tempfile.mkdtemp(prefix="tdfcpu_"), 1, os.cpu_count() or 1)
                if r:
                    nrec_c, secs = r
                    cpu = {"value": round(nrec_c / secs, 2), "unit": UNIT, "cores": os.cpu_count(),
                           "kind": "reference",
                           "fft": cpu_fft_proxy(job.sett.nfftf, os.cpu_count() or 1, nrec_c, secs),
                           "sample": "%d templates (1 sky point x %d spindowns) of the same workload, reference "
                                     "search sources PREC=FLOAT built with the project FFTW-API shim "
                                     "(textbook radix-2 FFT; FFTW absent), %.1f s" % (nrec_c, wl.nspd, secs)}
            per_step = int(round(nsum / args.steps))
            out = {
                "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 3), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                "dtype": "f32+f64 (split)" if args.form == "split" else "f64",
                "data": "synthetic (seeded Gaussian noise + injected CW signals, synthetic ephemeris)",
                "config": dict(wl.config, form=args.form, tuning=tuned,
                               step=("one %d-point slice of the %d-point patch per step, slices in turn"
                                     % (len(slices[0][0]), len(pm)) if len(slices) > 1
                                     else "the whole patch per step"),
                               templates_searched_per_step=per_step,
                               l2="flush: 256 MiB write between timed steps; per-step working set > L2"),
                "e2e": {"value": round(e2e, 1), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                        "d2h_bytes_per_step": int(d2h // args.steps)},
                "gpu_launches": int(launches),
                "triggers_per_step": int(ntrig // args.steps),
                "fp64": fp64,
                "roofline": roof, "cpu_baseline": cpu, "clocks": clk,
            }
        return out
    finally:
        shutil.rmtree(root, ignore_errors=True)


def run_sweep(args, rank, world, local_rank):
    """cfg5 scale sweep on one GPU: sky patches of 2^10 .. 2^18 points x 801
    spindowns of the same segment (N = 258492, sigma 1.0 / 1.3, 10% gaps).
    Each size is one device-only search over the patch's first
    min(size, --sweep-cap) points, timed with CUDA events after one untimed
    warm-up search of 64 points; every template counted is searched.  Prints
    one JSON line per size."""
    import torch
    from tdfstat_b200.engine import Engine

    if world > 1 or rank != 0:
        return None
    torch.cuda.set_device(local_rank)
    root = tempfile.mkdtemp(prefix="tdfsweep_")
    try:
        wl = Workload("cfg5", root)
        job = wl.job
        seg, opts = job.segment(), job.search_opts()
        eng = Engine(seg, opts, form=args.form, device=local_rank, max_sky_batch=args.sky_batch)
        stream = torch.cuda.ExternalStream(eng.stream(), device=local_rank)
        flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
        if not args.no_autotune:
            eng.autotune(wl.pm[:16], wl.mm[:16], wl.nn[:16])
        tuned = eng.tuning()
        peak, peak_kind = measured_peaks()
        bt = len(job.dets) * job.sett.N * (24 if args.form == "split" else 40)
        for k in range(10, 19):
            npts = 1 << k
            pm, mm, nn = wl.patch(npts)
            timed = min(npts, args.sweep_cap)
            sl = [(pm[:timed], mm[:timed], nn[:timed])]
            eng.search_device(pm[:64], mm[:64], nn[:64])
            torch.cuda.synchronize()
            ms, nsearched, ntrig, launches, clk = _timed_steps(eng, stream, flush, sl, 0, 1, lambda: None,
                                                               local_rank)
            value = nsearched / (ms / 1e3)
            ach = value * bt / 1e9
            print(json.dumps({
                "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": 1, "steps": 1, "warmup": 1,
                "ms_per_step": round(ms, 3), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32+f64 (split)" if args.form == "split" else "f64",
                "data": "synthetic (seeded Gaussian noise, sigma 1.0 / 1.3, 10% gaps, injected CW signal)",
                "config": dict(wl.config, sky_points=npts, templates_per_step=npts * wl.nspd,
                               timed_sky_points=timed, templates_searched=int(nsearched),
                               form=args.form, tuning=tuned,
                               patch="%d x %d points over 3.2 x 3.2 grid cells" % (1 << (k // 2), 1 << (k - k // 2)),
                               timed=("the whole patch" if timed == npts else
                                      "the patch's first %d points (every template counted is searched)" % timed)),
                "hbm": {"achieved": round(ach, 1), "peak": peak, "unit": "GB/s", "frac": round(ach / peak, 4),
                        "algorithmic_bytes_per_template": bt, "peak_kind": peak_kind},
                "gpu_launches": int(launches), "triggers": int(ntrig), "clocks": clk}), flush=True)
        eng.close()
        return None
    finally:
        shutil.rmtree(root, ignore_errors=True)


def run_tdf_segments(args, rank, world, local_rank):
    """cfg4: 64 segments of four sizes (N = 86164, 129246, 172328, 258492),
    each with its own inputs and a 16 x 16 patch x 401 spindowns.  A step
    brings every segment's inputs in from host memory and searches all of
    them.  Three ways to run the same step are timed, each with its own
    engines (one per segment size):
      plan        every segment of a size resident in its own slot of one
                  engine (tdf_engine_add_segment / upload_segment) and the
                  size's whole search one call (tdf_search_segments_device):
                  one captured graph per segment size spanning all its
                  segments
      batch       one segment at a time in slot 0 (tdf_engine_upload), one
                  captured graph per 8-point sky batch (the engine's default
                  path and the line's value)
      plain       as batch with every kernel launched from the host
                  (TDF_GRAPHS=0): one launch set per segment
    `value` includes the uploads (the data of 64 segments is brought in
    every step); `e2e` (batch form) also brings the records back
    (tdf_search_points)."""
    import torch
    import torch.distributed as dist
    from tdfstat_b200.engine import Engine

    torch.cuda.set_device(local_rank)
    root = tempfile.mkdtemp(prefix="tdfbench4_")
    try:
        if args.segments_by_cost:
            # whole segments to ranks by estimated cost; the total work is fixed
            from tdfstat_b200 import shard as _shard
            mw = MultiWorkload(root, world=1)
            costs = [_shard.segment_cost(w.templates, w.job.sett.nfftf, w.job.sett.nifo, w.job.sett.N)
                     for w in mw.segments]
            mine = set(_shard.assign_segments(costs, world)[rank])
            shards = [(w,) + tuple(w.shard(0, 1)) for k, w in enumerate(mw.segments) if k in mine]
        else:
            mw = MultiWorkload(root, world=world)
            shards = [(w,) + tuple(w.shard(rank, world)) for w in mw.segments]
        sizes = sorted({w.job.sett.N for w, _, _, _ in shards})
        # above the default priority, so that the engines' low-priority sky
        # stream fills this stream's kernel tails instead of competing
        stream = torch.cuda.Stream(device=local_rank, priority=-1)
        flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

        def barrier():
            if world > 1:
                dist.barrier()

        def make_engines(plain):
            if plain:
                os.environ["TDF_GRAPHS"] = "0"
            try:
                engines, tuned = {}, {}
                for w, pm, mm, nn in shards:
                    N = w.job.sett.N
                    if N not in engines:
                        e = Engine(w.job.segment(), w.job.search_opts(), form=args.form, device=local_rank,
                                   max_sky_batch=args.sky_batch)
                        e.set_stream(stream.cuda_stream)
                        if not args.no_autotune:
                            e.autotune(pm[:16], mm[:16], nn[:16])
                        tuned[N] = e.tuning()
                        engines[N] = e
                return engines, tuned
            finally:
                os.environ.pop("TDF_GRAPHS", None)

        def timed(step, steps):
            clocks = ClockSampler(local_rank)
            clocks.start()
            barrier()
            torch.cuda.synchronize()
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ev0.record(stream)
            n = 0
            for _ in range(steps):
                with torch.cuda.stream(stream):
                    flush.zero_()
                n += step()
            ev1.record(stream)
            torch.cuda.synchronize()
            barrier()
            return ev0.elapsed_time(ev1), n, clocks.stop()

        res = {}
        # ---- plan: all segments of a size resident, one call (one graph) per size
        engines, tuned = make_engines(False)
        slot_of, groups = {}, {N: [] for N in sizes}
        for w, pm, mm, nn in shards:
            e = engines[w.job.sett.N]
            if not groups[w.job.sett.N]:
                slot_of[id(w)] = 0
            else:
                slot_of[id(w)] = e.add_segment(w.job.segment())
            groups[w.job.sett.N].append((w, pm, mm, nn))
        calls = {}
        for N, g in groups.items():
            calls[N] = ([slot_of[id(w)] for w, _, _, _ in g], [len(pm) for _, pm, _, _ in g],
                        np.concatenate([pm for _, pm, _, _ in g]), np.concatenate([mm for _, _, mm, _ in g]),
                        np.concatenate([nn for _, _, _, nn in g]))

        def step_plan():
            n = 0
            for N, g in groups.items():
                e = engines[N]
                for w, _, _, _ in g:
                    e.upload_segment(slot_of[id(w)], w.job.segment())
                n += e.search_segments_device(*calls[N])[0]
            return n

        for _ in range(max(args.warmup, 2)):   # the second call captures each size's graph
            step_plan()
        l0 = sum(e.launch_count() for e in engines.values())
        ms, nsearched, clk = timed(step_plan, args.steps)
        launches = sum(e.launch_count() for e in engines.values()) - l0
        res["plan"] = (ms, nsearched)
        tuned_plan = tuned
        for e in engines.values():
            e.close()

        # ---- batch (graph per 8-point batch) and plain (no graphs): one segment at a time
        def per_segment(engines, records=False):
            def step():
                n = 0
                for w, pm, mm, nn in shards:
                    e = engines[w.job.sett.N]
                    e.upload(w.job.segment())
                    n += len(e.search(pm, mm, nn)) if records else e.search_device(pm, mm, nn)[0]
                return n
            return step

        e2e = None
        for mode in ("batch", "plain"):
            if mode == "plain" and args.no_cfg4_compare:
                continue
            engines, _ = make_engines(mode == "plain")
            st = per_segment(engines)
            for _ in range(args.warmup):
                st()
            l0m = sum(e.launch_count() for e in engines.values())
            ms_m, n_m, clk_m = timed(st, args.steps)
            res[mode] = (ms_m, n_m)
            if mode == "batch":
                launches, clk = sum(e.launch_count() for e in engines.values()) - l0m, clk_m
                ms_e, n_e, _ = timed(per_segment(engines, records=True), args.steps)
                e2e = (ms_e, n_e)
            for e in engines.values():
                e.close()

        keys = ["batch"] + [k for k in res if k != "batch"]
        t = torch.tensor([res[k][0] for k in keys] + [e2e[0]], dtype=torch.float64, device="cuda")
        n = torch.tensor([res[k][1] for k in keys] + [e2e[1]], dtype=torch.float64, device="cuda")
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            dist.all_reduce(n, op=dist.ReduceOp.SUM)
        vals = {k: float(n[i]) / (float(t[i]) / 1e3) for i, k in enumerate(keys)}
        ms = float(t[0])
        h2d = sum(sum(d.xdat.nbytes + d.detssb.nbytes for d in w.job.dets) + w.job.cosmodf.nbytes +
                  w.job.sinmodf.nbytes for w, _, _, _ in shards)
        if rank != 0:
            return None
        return {
            "metric": METRIC, "value": round(vals["batch"], 1), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 3),
            "higher_is_better": True, "scaling": "strong" if args.segments_by_cost else "weak",
            "vs_baseline": None,
            "dtype": "f32+f64 (split)" if args.form == "split" else "f64",
            "data": "synthetic (seeded Gaussian noise + injected CW signal per segment, synthetic ephemeris)",
            "config": dict(mw.config, form=args.form, tuning={str(k): v for k, v in tuned_plan.items()},
                           distribution=("whole segments to ranks by estimated cost" if args.segments_by_cost
                                         else "every segment's sky patch split over the ranks"),
                           templates_searched_per_step=int(round(float(n[0]) / args.steps)),
                           engines="one per segment size; value: one segment at a time, one captured graph per "
                                   "8-point sky batch; inputs of all 64 segments uploaded from host memory in "
                                   "every step (all three forms in 'compare')",
                           l2="flush: 256 MiB write between timed steps; per-step working set > L2"),
            "compare": {"one_graph_per_segment_size": round(vals["plan"], 1),
                        "graph_per_8_point_batch": round(vals["batch"], 1),
                        "plain_launches_per_segment": round(vals["plain"], 1) if "plain" in vals else None},
            "e2e": {"value": round(float(n[-1]) / (float(t[-1]) / 1e3), 1), "unit": UNIT,
                    "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": None,
                    "form": "graph per 8-point batch, records brought back (tdf_search_points)"},
            "gpu_launches": int(launches),
            "roofline": None, "cpu_baseline": None, "clocks": clk,
        }
    finally:
        shutil.rmtree(root, ignore_errors=True)


def run_reference(args, rank, world):
    if rank != 0:
        return None
    root = tempfile.mkdtemp(prefix="tdfref_")
    try:
        # cfg4: the sample comes from its largest segment kind (nod 6, the 4th)
        wl = Workload("cfg4:4" if args.workload == "cfg4" else args.workload, root)
        threads = os.cpu_count() or 1
        sroot = tempfile.mkdtemp(prefix="tdfrefs_")
        for _ in range(args.warmup):
            r = cpu_reference_sample(wl, sroot, 1, threads)
            if r is None:
                return {"impl": "reference", "unavailable": "oracle/_ref/gwsearch-ref-f32 not built"}
        tot_n, tot_s = 0, 0.0
        for _ in range(args.steps):
            n, s = cpu_reference_sample(wl, sroot, 1, threads)
            tot_n += n
            tot_s += s
        v = tot_n / tot_s
        fftp = cpu_fft_proxy(wl.job.sett.nfftf, threads, tot_n, tot_s)
        sample = ("%d templates per step (1 sky point x %d spindowns) of the %s workload; reference search "
                  "sources (PREC=FLOAT, SIMD=NONE) compiled unmodified against the project FFTW-API shim "
                  "(textbook radix-2 FFT, FFTW absent)" % (tot_n // args.steps, wl.nspd, wl.name))
        config = dict(wl.config, sky_points=1, templates_per_step=tot_n // args.steps,
                      step="one sky point of the workload's segment x its spindowns (a bounded sample of the "
                           "GPU arm's workload; same segment, grid, F range and threshold)")
        return {"impl": "reference", "metric": METRIC, "value": round(v, 2), "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * tot_s / args.steps, 3),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic", "config": config,
                "cpu_baseline": {"value": round(v, 2), "unit": UNIT, "cores": threads, "kind": "reference",
                                 "sample": sample, "fft": fftp},
                "e2e": {"value": round(v, 2), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    finally:
        shutil.rmtree(root, ignore_errors=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="tdf", choices=["tdf", "reference"])
    ap.add_argument("--form", default="split", choices=["split", "fp64"])
    ap.add_argument("--workload", default="cfg3", choices=["cfg1", "cfg2", "cfg3", "cfg4", "cfg5"])
    ap.add_argument("--slice-points", type=int, default=None,
                    help="sky points per step (default: 1024 for cfg3, the whole patch otherwise)")
    ap.add_argument("--no-fp64", action="store_true", help="skip the plain FP64 form's line entry")
    ap.add_argument("--fp64-steps", type=int, default=3, help="timed steps of the FP64 form (at most --steps)")
    ap.add_argument("--sky-batch", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--segments-by-cost", action="store_true",
                    help="cfg4 on several GPUs: whole segments to ranks by estimated cost (strong scaling)")
    ap.add_argument("--sky-points", type=int, default=0, help="use only the first K sky points (profiling runs)")
    ap.add_argument("--sweep", action="store_true", help="cfg5: one line per sky-patch size 2^10 .. 2^18")
    ap.add_argument("--no-cfg4-compare", action="store_true", help="cfg4: skip the plain-launch comparison")
    ap.add_argument("--sweep-cap", type=int, default=4096, help="sky points timed per sweep size at most")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1 and args.impl == "tdf":
        import torch
        import torch.distributed as dist
        import datetime
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    if args.impl == "reference":
        out = run_reference(args, rank, world)
    elif args.sweep:
        if args.workload != "cfg5":
            ap.error("--sweep is the cfg5 scale sweep (--workload cfg5)")
        out = run_sweep(args, rank, world, local_rank)
    elif args.workload == "cfg4":
        out = run_tdf_segments(args, rank, world, local_rank)
    else:
        out = run_tdf(args, rank, world, local_rank)
    if world > 1 and args.impl == "tdf":
        import torch.distributed as dist
        dist.destroy_process_group()
    if rank == 0 and out is not None:
        print(json.dumps(out))


if __name__ == "__main__":
    main()
