"""tdfstat_b200: B200 (sm_100a) engine for TDFstat's coherent F-statistic
search hot path (the per-sky-point job_core() chain of search/network).

The compute runs in libtdfcuda (hand-written CUDA kernels behind the C ABI of
include/tdfcuda.h); this package holds the Python side:

* :mod:`tdfstat_b200.engine` — ctypes binding of the engine (search,
  spectra, injection, tuning);
* :mod:`tdfstat_b200.host` — mirror of the reference's set-up from its INI
  (settings, grid, data, ranges, the [gpu] section);
* :mod:`tdfstat_b200.vlines` — the band's veto lines (extraction and the
  veto file);
* :mod:`tdfstat_b200.coinc` — coincidences between segments;
* :mod:`tdfstat_b200.shard` — sharding over GPUs;
* :mod:`tdfstat_b200.synth`, :mod:`tdfstat_b200.workloads` — seeded input
  generators and the benchmark workloads;
* :mod:`tdfstat_b200.build` — builds libtdfcuda for sm_100a in-tree.
"""
__all__ = ["engine", "host", "vlines", "coinc", "shard", "synth", "workloads", "build"]
