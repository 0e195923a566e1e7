"""mods=write_signal (init.c:475-497): the injected signal h0*s_n[i] of
every detector, one "%e" line per sample, in
<outdir>/injections/signal_<seg>_<band>_<det><label>.  The oracle's signal
(orc_add_signal_out) written by host.write_signal_files must be the text the
reference's own FP64 build writes for golden case g4_addsig."""
import dataclasses
import os

import pytest

import refkit
from golden.cases import CASES
from tdfstat_b200 import host, synth


@pytest.mark.skipif(not os.path.exists(refkit.REF_BIN["f64"]), reason="reference build not present")
def test_oracle_signal_file_is_the_references(tmp_path, oracle):
    case = dataclasses.replace(CASES["g4_addsig"], mods_extra="write_signal")
    ref = refkit.reference_signal_files(synth.write_case(str(tmp_path / "ref"), case))
    assert sorted(ref) == ["signal_001_1440_H1", "signal_001_1440_L1"]
    job = host.Job(synth.write_case(str(tmp_path / "mine"), case), float_build=False)
    assert job.write_signal
    os_ = refkit.OracleSegment(job, oracle)
    paths = host.write_signal_files(job, list(os_.signal))
    for p in paths:
        with open(p) as f:
            assert f.read() == ref[os.path.basename(p)]
