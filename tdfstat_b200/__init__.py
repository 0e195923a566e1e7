"""tdfstat_b200: B200 (sm_100a) engine for TDFstat's coherent F-statistic
search hot path (the per-sky-point job_core() chain of search/network).

The compute runs in libtdfcuda (hand-written CUDA kernels behind the C ABI of
include/tdfcuda.h); this package holds the host-side mirror of the
reference's set-up (:mod:`tdfstat_b200.host`), the ctypes binding
(:mod:`tdfstat_b200.engine`) and seeded input generators
(:mod:`tdfstat_b200.synth`).
"""
__all__ = ["host", "synth", "engine"]
