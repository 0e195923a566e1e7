"""The batch pipeline variants give identical records: kernels launched one by
one on a single stream (TDF_GRAPHS=0, TDF_LANES=1) against the default
engine, which spreads resolve groups over several lanes and, from the second
time a batch configuration is seen, replays it as a captured CUDA graph.
Repeated calls on one engine go through the first-sighting, capture and
replay paths in turn.  Records are also the same for every chunk size."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _records(res):
    return res.hdr.copy(), [p.copy() for p in res.pairs], res.per_point.copy()


def _same(a, b):
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[2], b[2])
    assert len(a[1]) == len(b[1])
    for x, y in zip(a[1], b[1]):
        np.testing.assert_array_equal(x, y)


@pytest.mark.parametrize("name", ["g2_h1l1_inj", "g3_allsky_blocks"])
def test_graph_replay_matches_plain_launches(golden, monkeypatch, name):
    from tdfstat_b200.engine import Engine
    g = golden(name)
    pm, mm, nn = g.job32.sky_points()
    monkeypatch.setenv("TDF_GRAPHS", "0")
    monkeypatch.setenv("TDF_LANES", "1")
    plain = Engine.from_job(g.job32, form="split")
    ref = _records(plain.search(pm, mm, nn))
    plain.close()
    monkeypatch.delenv("TDF_GRAPHS")
    monkeypatch.delenv("TDF_LANES")
    eng = Engine.from_job(g.job32, form="split")
    launches = []
    for _ in range(3):   # plain launches, capture, replay
        n0 = eng.launch_count()
        _same(_records(eng.search(pm, mm, nn)), ref)
        launches.append(eng.launch_count() - n0)
    # a replayed graph counts the kernels it holds
    assert launches[0] == launches[1] == launches[2] > 0
    eng.close()


@pytest.mark.parametrize("name", ["g2_h1l1_inj", "g6_h1l1v1"])
def test_sky_stage_overlap_matches_in_line(golden, monkeypatch, name):
    """The default runs the next batch's sky stage on its own low-priority
    stream; TDF_SKY_OVERLAP=0 runs it in line on the engine stream.  Small
    sky batches give several batches per search, so the overlap is used."""
    from tdfstat_b200.engine import Engine
    g = golden(name)
    pm, mm, nn = g.job32.sky_points()
    ref = None
    for ov in ("0", None):
        if ov is None:
            monkeypatch.delenv("TDF_SKY_OVERLAP")
        else:
            monkeypatch.setenv("TDF_SKY_OVERLAP", ov)
        eng = Engine(g.job32.segment(), g.job32.search_opts(), form="split", device=0, max_sky_batch=2)
        got = _records(eng.search(pm, mm, nn))
        eng.close()
        if ref is None:
            ref = got
        else:
            _same(got, ref)
    # on a caller's stream: default priority (sky stage in line) and a
    # higher one (sky stage overlapped)
    import torch
    for prio in (0, -1):
        s = torch.cuda.Stream(device=0, priority=prio)
        eng = Engine(g.job32.segment(), g.job32.search_opts(), form="split", device=0, max_sky_batch=2)
        eng.set_stream(s.cuda_stream)
        _same(_records(eng.search(pm, mm, nn)), ref)
        eng.close()


def test_records_do_not_depend_on_chunk_size(golden):
    from tdfstat_b200.engine import Engine, TdfError
    g = golden("g2_h1l1_inj")
    pm, mm, nn = g.job32.sky_points()
    eng = Engine.from_job(g.job32, form="split")
    ref = _records(eng.search(pm, mm, nn))
    for tc in (1, 3, 17, 48, 96):
        eng.templates_per_chunk = tc
        assert eng.templates_per_chunk == tc
        _same(_records(eng.search(pm, mm, nn)), ref)
    for bad in (0, 97):
        with pytest.raises(TdfError):
            eng.templates_per_chunk = bad
    eng.close()


@pytest.mark.parametrize("name", ["g2_h1l1_inj", "g1_h1_directed"])
def test_tma_staged_operands_match(golden, monkeypatch, name):
    """TDF_STAGED_OPERANDS=1 (column-pass operands brought in by TMA boxes)
    computes the same arithmetic as the default per-thread loads."""
    from tdfstat_b200.engine import Engine
    g = golden(name)
    pm, mm, nn = g.job32.sky_points()
    eng = Engine.from_job(g.job32, form="split")
    ref = _records(eng.search(pm, mm, nn))
    eng.close()
    monkeypatch.setenv("TDF_STAGED_OPERANDS", "1")
    eng = Engine.from_job(g.job32, form="split")
    _same(_records(eng.search(pm, mm, nn)), ref)
    eng.close()


def test_engine_takes_the_ini_gpu_section(golden):
    """Engine.from_job without arguments uses the job's [gpu] options."""
    import dataclasses
    from tdfstat_b200 import host
    from tdfstat_b200.engine import Engine
    g = golden("g2_h1l1_inj")
    job = g.job32
    keep = job.gpu
    try:
        job.gpu = dataclasses.replace(host.GpuOptions(), form="fp64", templates_per_chunk=3)
        eng = Engine.from_job(job)
        assert eng.form == "fp64" and eng.templates_per_chunk == 3
        eng.close()
        job.gpu = host.GpuOptions()
        eng = Engine.from_job(job)
        assert eng.form == "split"
        eng.close()
    finally:
        job.gpu = keep


@pytest.mark.parametrize("name", ["g2_h1l1_inj", "g7_fftpad2"])
def test_row_pass_without_bulk_copies_matches(golden, monkeypatch, name):
    """TDF_ROW_BULK=0 (row-pass inputs by per-thread loads) gives the same
    records as the default bulk copies into shared memory."""
    from tdfstat_b200.engine import Engine
    g = golden(name)
    pm, mm, nn = g.job32.sky_points()
    eng = Engine.from_job(g.job32, form="split")
    ref = _records(eng.search(pm, mm, nn))
    eng.close()
    monkeypatch.setenv("TDF_ROW_BULK", "0")
    eng = Engine.from_job(g.job32, form="split")
    _same(_records(eng.search(pm, mm, nn)), ref)
    eng.close()


@pytest.mark.parametrize("name", ["g2_h1l1_inj", "g5_vlines", "g6_h1l1v1", "g7_fftpad2"])
def test_sparse_f_store_matches_full_store(golden, monkeypatch, name):
    """The split form's default F store (the row pass keeps F on the chip:
    candidate records and the edge bins of its runs only) gives the same
    records, bit for bit, as TDF_FULL_F=1 (every F spectrum written to the
    F ring and scanned by the trigger selection)."""
    from tdfstat_b200.engine import Engine
    g = golden(name)
    pm, mm, nn = g.job32.sky_points()
    eng = Engine.from_job(g.job32, form="split")
    ref = _records(eng.search(pm, mm, nn))
    eng.close()
    monkeypatch.setenv("TDF_FULL_F", "1")
    eng = Engine.from_job(g.job32, form="split")
    _same(_records(eng.search(pm, mm, nn)), ref)
    eng.close()
