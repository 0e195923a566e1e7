"""Several segments resident on one engine (tdf_engine_add_segment) and the
whole-call search over them (tdf_search_segments_device, one enqueue
sequence captured into one CUDA graph from its second call on).

Three segments of the same sizes (the golden case g2_h1l1_inj with other
seeds and segment numbers: other noise, gaps, grid matrix and injection
phase) searched in one call must give the record and trigger counts of
separate single-segment engines with the same options, in every order of
the slots, on the first (plain launches), second (capture) and third
(replay) call, in both forms; the template parameters the call forms on
the device must equal the host's bit for bit.
"""
import dataclasses
import shutil
import tempfile

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def three_jobs():
    from golden.cases import CASES
    from tdfstat_b200 import host, synth
    base = CASES["g2_h1l1_inj"]
    roots, jobs = [], {}
    for k in range(3):
        root = tempfile.mkdtemp(prefix="tdf_segs_")
        roots.append(root)
        ini = synth.write_case(root, dataclasses.replace(base, seed=base.seed + 17 * k, seg=1 + k))
        jobs.setdefault("split", []).append(host.Job(ini, float_build=True))
        jobs.setdefault("fp64", []).append(host.Job(ini, float_build=False))
    yield jobs
    for r in roots:
        shutil.rmtree(r, ignore_errors=True)


@pytest.mark.parametrize("form", ["split", "fp64"])
def test_segments_in_one_call_match_separate_engines(three_jobs, monkeypatch, form):
    """TDF_CHECK_PLAN=1 also compares the template parameters the device forms
    for the call with the host's (bit for bit) on every call."""
    from tdfstat_b200.engine import Engine
    monkeypatch.setenv("TDF_CHECK_PLAN", "1")
    jobs = three_jobs[form]
    opts = jobs[0].search_opts()
    pts = [j.sky_points() for j in jobs]
    want = []
    for j, (pm, mm, nn) in zip(jobs, pts):
        e1 = Engine(j.segment(), opts, form=form)
        want.append(e1.search_device(pm, mm, nn))
        e1.close()
    assert all(n > 0 for n, _ in want) and sum(t for _, t in want) > 0
    eng = Engine(jobs[0].segment(), opts, form=form)
    slots = [0] + [eng.add_segment(j.segment()) for j in jobs[1:]]
    assert slots == [0, 1, 2]
    for order in ([0, 1, 2], [2, 0, 1]):
        pm = np.concatenate([np.asarray(pts[k][0]) for k in order])
        mm = np.concatenate([np.asarray(pts[k][1]) for k in order])
        nn = np.concatenate([np.asarray(pts[k][2]) for k in order])
        npts = [len(pts[k][0]) for k in order]
        expect = (sum(want[k][0] for k in order), sum(want[k][1] for k in order))
        for rep in range(3):   # plain launches, capture, replay
            got = eng.search_segments_device(order, npts, pm, mm, nn)
            print(form, order, rep, got, expect)
            assert got == expect
    # a segment with no points, and slot 0's own search afterwards
    got = eng.search_segments_device([1, 0], [0, len(pts[0][0])], *pts[0])
    assert got == want[0]
    assert eng.search_device(*pts[0]) == want[0]
    eng.close()


def test_segment_slot_upload_replaces_data(three_jobs):
    """tdf_engine_upload_segment: slot 1 re-uploaded with segment 3's inputs
    searches as segment 3."""
    from tdfstat_b200.engine import Engine
    jobs = three_jobs["split"]
    opts = jobs[0].search_opts()
    pm, mm, nn = jobs[2].sky_points()
    e1 = Engine(jobs[2].segment(), opts, form="split")
    want = e1.search_device(pm, mm, nn)
    e1.close()
    eng = Engine(jobs[0].segment(), opts, form="split")
    s1 = eng.add_segment(jobs[1].segment())
    eng.upload_segment(s1, jobs[2].segment())
    assert eng.search_segments_device([s1], [len(pm)], pm, mm, nn) == want
    eng.close()
