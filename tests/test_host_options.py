"""Search options the golden cases leave at their defaults, checked against
the reference's own FP64 build run here: one hemisphere of an all-sky grid
(search:hemi = 1 or 2), a band overlap (search:overlap), an output label (search:label, which also names the
veto file), and search:usedet selecting one detector of a two-detector data
tree.  The host mirror's set-up feeds the oracle restatement, whose records
must be the reference's bit for bit."""
import dataclasses
import os

import numpy as np
import pytest

import refkit
from golden.cases import CASES
from tdfstat_b200 import host, synth

pytestmark = pytest.mark.skipif(not os.path.exists(refkit.REF_BIN["f64"]), reason="reference build not present")


def _case(variant):
    if variant == "hemi1":
        return dataclasses.replace(CASES["g3_allsky_blocks"], hemi=1), None
    if variant == "hemi2":
        return dataclasses.replace(CASES["g3_allsky_blocks"], hemi=2), None
    if variant == "overlap":
        # band overlap 0.25: fpo = 10 + 0.75 band/(2 dt) = 77.5 Hz, default
        # narrowdown (1 - overlap)/2 (common.c:14-18, init.c:134-139)
        return dataclasses.replace(CASES["g1_h1_directed"], overlap=0.25,
                                   gcenter=(77.5152, -2e-10, 1.2, 0.3)), None
    if variant == "label":
        return dataclasses.replace(CASES["g2_h1l1_inj"], label="run7"), None
    return CASES["g2_h1l1_inj"], "H1"     # usedet = H1 on an H1L1 tree


@pytest.mark.parametrize("variant", ["hemi1", "hemi2", "label", "usedet_H1", "overlap"])
def test_options_match_reference(tmp_path, oracle, variant):
    case, usedet = _case(variant)
    ini = synth.write_case(str(tmp_path), case)
    if usedet:
        with open(ini) as f:
            text = f.read()
        with open(ini, "w") as f:
            f.write(text.replace("usedet = %s" % "".join(case.dets), "usedet = %s" % usedet))
    ref, _, _ = refkit.run_reference(ini, "f64", threads=1)
    job = host.Job(ini, float_build=False)
    if usedet:
        assert [d.name for d in job.dets] == [usedet]
    pm, mm, nn = job.sky_points()
    if variant in ("hemi1", "hemi2"):
        assert set(np.unique(pm)) == {int(variant[-1])}
        assert set(np.unique(ref.pm)) == {int(variant[-1])}
    os_ = refkit.OracleSegment(job, oracle)
    st, rec, _ = refkit.search_points(oracle.orc_search_points, os_.seg, job.search_opts(), pm, mm, nn)
    assert st == 0
    assert len(rec) == len(ref) > 0
    np.testing.assert_array_equal(rec.hdr, ref.hdr)
    assert rec.ntrig == ref.ntrig
    for a, b in zip(rec.pairs, ref.pairs):
        np.testing.assert_array_equal(a, b)
