"""Benchmark of the coherent-search hot path (job_core chain) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl tdf|reference]
                    [--form split|fp64] [--workload cfg2|cfg1|cfg3]

Workload (default cfg2): H1+L1, 2-sidereal-day segment at dt = 2 s
(N = 86164, nfft = nfftf = 2^17, Ninterp = 2^18), seeded Gaussian noise
(sigma 1, 5% gaps) plus an injected CW signal (network SNR 12, f = 100.1234 Hz,
fdot = -3e-10 Hz/s), a 32 x 32 sky patch around the injection x 401
spindowns = 410,624 templates per step, F over bins [1024, 64512], thr 14.5.
A step is one pass of the hot path over the whole patch.  Inputs are synthetic
(no public data set is used).

  value : templates/s with the segment resident in HBM (device-only pass:
          sky stage + spindown stage + trigger compaction), CUDA events on
          the engine's stream, barrier + synchronize around the K steps,
          max over ranks.
  e2e   : the same through the C ABI with host buffers: upload of the
          segment's inputs (xdat, DetSSB, aux arrays) and download of the
          records inside every step.
  --impl reference: the reference's own C search (its unmodified sources,
          PREC=FLOAT, built by oracle/Makefile) on the host cores, each step
          a bounded sample (2 sky points x 401 spindowns) of the workload.
Under torchrun (N > 1) every rank searches its own 32 x 32 patch (the same
region, shifted by a fraction of a grid step per rank) as a contiguous shard
of one point list: weak scaling, no collective on the data path; the
whole-job value counts all ranks' templates; rank 0 prints the JSON line.
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


def profile_traffic(workload: str, form: str):
    """DRAM bytes per template of the column pass, from the committed ncu
    summary profiles/traffic_<workload>_<form>.md (its k_colpass table row),
    or None when there is no summary for this workload and form."""
    p = os.path.join(REPO, "profiles", "traffic_%s_%s.md" % (workload, form))
    if not os.path.exists(p):
        return None
    with open(p) as f:
        for line in f:
            cells = [c.strip() for c in line.strip().strip("|").split("|")]
            if cells and cells[0] == "k_colpass" and len(cells) >= 6:
                return float(cells[5].split()[0])
    return None


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
    second of warm-up, ~1 s timed) and with scipy.fft (pocketfft; one
    transform does not use several workers, so this is a single-thread
    time).  The per-sky-point interpolation transforms (FP64, 4 per
    detector per point) are left in.  When the isolated shim time exceeds
    the sample's own time the share is reported as measured and no
    substituted rate is derived."""
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
    x = (_np.random.default_rng(0).standard_normal(nfftf) + 1j * _np.random.default_rng(1).standard_normal(nfftf))
    x = x.astype(_np.complex64)
    t0 = _t.perf_counter()
    while _t.perf_counter() - t0 < 0.3:
        sfft.fft(x)
    t0 = _t.perf_counter()
    for _ in range(100):
        sfft.fft(x)
    t_sp = (_t.perf_counter() - t0) / 100
    fft_s = 2 * ntmpl * t_shim
    rest = secs - fft_s
    out = {"fft_share": round(fft_s / secs, 3), "shim_ms_per_fft": round(1e3 * t_shim, 3),
           "scipy_ms_per_fft_1thread": round(1e3 * t_sp, 3)}
    if rest > 0:
        out["value_with_scipy_fft"] = round(ntmpl / (rest + 2 * ntmpl * t_sp), 2)
    else:
        out["value_with_scipy_fft"] = None
        out["note"] = "isolated shim FFT slower than inside the sample; no substituted rate"
    return out


# ------------------------------------------------------------------ arms

def run_tdf(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from tdfstat_b200.engine import Engine, load_library
    import ctypes as C

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
        seg, opts = job.segment(), job.search_opts()
        eng = Engine(seg, opts, form=args.form, device=local_rank, max_sky_batch=args.sky_batch)
        lib = load_library()
        stream = torch.cuda.ExternalStream(eng.stream(), device=local_rank)
        flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

        def barrier():
            if world > 1:
                dist.barrier()

        # chunk size by the engine's autotuner on a 16-point sample (untimed)
        tuned = eng.autotune(pm[:16], mm[:16], nn[:16]) if not args.no_autotune else None
        # warm-up steps are the timed step exactly (the flush included: its
        # first launch loads torch's fill kernel)
        for _ in range(args.warmup):
            with torch.cuda.stream(stream):
                flush.zero_()
            eng.search_device(pm, mm, nn)
        torch.cuda.synchronize()
        # templates a step searches = records it writes (one per spindown of
        # every point inside the grid ellipse)
        ntmpl, _ = eng.search_device(pm, mm, nn)
        if ntmpl != len(pm) * wl.nspd:
            print("bench: %d of %d patch templates lie inside the sky grid" % (ntmpl, len(pm) * wl.nspd),
                  file=sys.stderr)
        # ---- value: device-resident inputs, K steps
        launches0 = eng.launch_count()
        clocks = ClockSampler(local_rank)
        clocks.start()
        barrier()
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ntrig = 0
        nsearched = 0
        ev0.record(stream)
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()   # 256 MiB (> L2) written between steps, on the engine's stream
            nrec, nt = eng.search_device(pm, mm, nn)
            ntrig += nt
            nsearched += nrec
        ev1.record(stream)
        torch.cuda.synchronize()
        barrier()
        clk = clocks.stop()
        ms = ev0.elapsed_time(ev1)
        launches = eng.launch_count() - launches0
        # ---- per-kernel durations: the same K steps again with CUDA events
        # recorded on the engine's stream around every launch.  Timing runs
        # the kernels one after another (one lane); each launch gets at
        # least 32 templates (1024 column-pass CTAs, 3.5 waves at 2 per SM)
        # so that a launch has the GPU to itself rather than under-filling it
        tc_run = eng.templates_per_chunk
        tc_timed = max(tc_run, 32)
        eng.templates_per_chunk = tc_timed
        eng.enable_kernel_timing(True)
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
            eng.search_device(pm, mm, nn)
        torch.cuda.synchronize()
        ktimes = eng.kernel_times()
        eng.enable_kernel_timing(False)
        eng.templates_per_chunk = tc_run
        # ---- e2e: host buffers through the C ABI
        for _ in range(1):
            eng.upload(seg)
            eng.search(pm, mm, nn)
        torch.cuda.synchronize()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        nsearched_e2e = 0
        for _ in range(args.steps):
            eng.upload(seg)
            res = eng.search(pm, mm, nn)
            nsearched_e2e += len(res)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        ms_e2e = e0.elapsed_time(e1)
        h2d = sum(d.xdat.nbytes + d.detssb.nbytes for d in job.dets) + job.cosmodf.nbytes + job.sinmodf.nbytes \
            + pm.nbytes + mm.nbytes + nn.nbytes
        d2h = len(res) * 40 + res.pairs_flat.nbytes
        # times: max over ranks; templates searched: sum over ranks
        t = torch.tensor([ms, ms_e2e], dtype=torch.float64, device="cuda")
        n = torch.tensor([nsearched, nsearched_e2e], dtype=torch.float64, device="cuda")
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            dist.all_reduce(n, op=dist.ReduceOp.SUM)
        ms, ms_e2e = float(t[0]), float(t[1])
        value = float(n[0]) / (ms / 1e3)
        e2e = float(n[1]) / (ms_e2e / 1e3)
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
                tr = profile_traffic(args.workload, args.form)
                traffic = round(tr * col_t / col_n) if tr is not None else None
                roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                        "frac": round(achieved / peak, 4), "traffic": traffic,
                        "kernel": "k_colpass (demodulation + first FFT pass)",
                        "peak_kind": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind,
                        "algorithmic_bytes_per_template": bt,
                        "kernel_ms_share": {k: round(v, 3) for k, v in ktimes.items() if k.endswith("_ms")},
                        "avg_launch_ms": round(col_ms / col_n, 4), "templates_per_launch": col_t / col_n,
                        "timed": "CUDA events on the engine stream around each launch, one lane, %d templates "
                                 "per launch (the run itself: %d per chunk over concurrent lanes)" % (tc_timed, tc_run)}
            cpu = None
            if not args.no_cpu_baseline and world == 1:   # the CPU baseline is an N = 1 figure
                r = cpu_reference_sample(wl, tempfile.mkdtemp(prefix="tdfcpu_"), 3, os.cpu_count() or 1)
                if r:
                    nrec_c, secs = r
                    cpu = {"value": round(nrec_c / secs, 2), "unit": UNIT, "cores": os.cpu_count(),
                           "kind": "reference",
                           "fft": cpu_fft_proxy(job.sett.nfftf, os.cpu_count() or 1, nrec_c, secs),
                           "sample": "%d templates (3 sky points x %d spindowns) of the same workload, reference "
                                     "search sources PREC=FLOAT built with the project FFTW-API shim "
                                     "(textbook radix-2 FFT; FFTW absent), %.1f s" % (nrec_c, wl.nspd, secs)}
            out = {
                "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 3), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                "dtype": "f32+f64 (split)" if args.form == "split" else "f64",
                "data": "synthetic (seeded Gaussian noise + injected CW signal, synthetic ephemeris)",
                "config": dict(wl.config, form=args.form, templates_per_chunk=tuned,
                               templates_searched_per_step_per_gpu=int(ntmpl),
                               templates_searched_per_step=int(round(float(n[0]) / args.steps)),
                               l2="flush: 256 MiB write between timed steps; per-step working set > L2"),
                "e2e": {"value": round(e2e, 1), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                        "d2h_bytes_per_step": int(d2h)},
                "gpu_launches": int(launches),
                "triggers_per_step": int(ntrig // args.steps),
                "roofline": roof, "cpu_baseline": cpu, "clocks": clk,
            }
        eng.close()
        return out
    finally:
        shutil.rmtree(root, ignore_errors=True)


def run_tdf_segments(args, rank, world, local_rank):
    """cfg4: 64 segments of four sizes.  One engine per size, all on one
    stream; a step streams every segment in (tdf_engine_upload: its inputs
    from host memory) and searches its patch.  `value` includes the uploads
    (the data of 64 segments is not resident at once); `e2e` also brings the
    records back (tdf_search_points)."""
    import torch
    import torch.distributed as dist
    from tdfstat_b200.engine import Engine

    torch.cuda.set_device(local_rank)
    root = tempfile.mkdtemp(prefix="tdfbench4_")
    engines = {}
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
        # above the default priority, so that the engines' low-priority sky
        # stream fills this stream's kernel tails instead of competing
        stream = torch.cuda.Stream(device=local_rank, priority=-1)
        tuned = {}
        for w, pm, mm, nn in shards:
            N = w.job.sett.N
            if N not in engines:
                e = Engine(w.job.segment(), w.job.search_opts(), form=args.form, device=local_rank,
                           max_sky_batch=args.sky_batch)
                e.set_stream(stream.cuda_stream)
                tuned[N] = e.autotune(pm[:16], mm[:16], nn[:16]) if not args.no_autotune else None
                engines[N] = e
        flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

        def step(records=False):
            n = 0
            for w, pm, mm, nn in shards:
                e = engines[w.job.sett.N]
                e.upload(w.job.segment())
                n += len(e.search(pm, mm, nn)) if records else e.search_device(pm, mm, nn)[0]
            return n

        def barrier():
            if world > 1:
                dist.barrier()

        for _ in range(args.warmup):
            with torch.cuda.stream(stream):
                flush.zero_()
            step()
        torch.cuda.synchronize()
        launches0 = sum(e.launch_count() for e in engines.values())
        clocks = ClockSampler(local_rank)
        clocks.start()
        barrier()
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        nsearched = 0
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
            nsearched += step()
        ev1.record(stream)
        torch.cuda.synchronize()
        barrier()
        clk = clocks.stop()
        ms = ev0.elapsed_time(ev1)
        launches = sum(e.launch_count() for e in engines.values()) - launches0
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        nsearched_e2e = 0
        for _ in range(args.steps):
            nsearched_e2e += step(records=True)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        ms_e2e = e0.elapsed_time(e1)
        t = torch.tensor([ms, ms_e2e], dtype=torch.float64, device="cuda")
        n = torch.tensor([nsearched, nsearched_e2e], dtype=torch.float64, device="cuda")
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            dist.all_reduce(n, op=dist.ReduceOp.SUM)
        ms, ms_e2e = float(t[0]), float(t[1])
        h2d = sum(sum(d.xdat.nbytes + d.detssb.nbytes for d in w.job.dets) + w.job.cosmodf.nbytes +
                  w.job.sinmodf.nbytes for w, _, _, _ in shards)
        if rank != 0:
            return None
        return {
            "metric": METRIC, "value": round(float(n[0]) / (ms / 1e3), 1), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 3),
            "higher_is_better": True, "scaling": "strong" if args.segments_by_cost else "weak",
            "vs_baseline": None,
            "dtype": "f32+f64 (split)" if args.form == "split" else "f64",
            "data": "synthetic (seeded Gaussian noise + injected CW signal per segment, synthetic ephemeris)",
            "config": dict(mw.config, form=args.form, templates_per_chunk={str(k): v for k, v in tuned.items()},
                           distribution=("whole segments to ranks by estimated cost" if args.segments_by_cost
                                         else "every segment's sky patch split over the ranks"),
                           templates_searched_per_step=int(round(float(n[0]) / args.steps)),
                           engines="one per segment size, segments streamed in by tdf_engine_upload each step",
                           l2="flush: 256 MiB write between timed steps; per-step working set > L2"),
            "e2e": {"value": round(float(n[1]) / (ms_e2e / 1e3), 1), "unit": UNIT,
                    "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": None},
            "gpu_launches": int(launches),
            "roofline": None, "cpu_baseline": None, "clocks": clk,
        }
    finally:
        for e in engines.values():
            e.close()
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
        return {"impl": "reference", "metric": METRIC, "value": round(v, 2), "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * tot_s / args.steps, 3),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic", "config": dict(wl.config),
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
    ap.add_argument("--workload", default="cfg2", choices=["cfg1", "cfg2", "cfg3", "cfg4", "cfg5"])
    ap.add_argument("--sky-batch", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--segments-by-cost", action="store_true",
                    help="cfg4 on several GPUs: whole segments to ranks by estimated cost (strong scaling)")
    ap.add_argument("--sky-points", type=int, default=0, help="use only the first K sky points (profiling runs)")
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
