"""The INI's [gpu] section (host.GpuOptions): parsed by the host mirror,
defaults when absent, invalid values refused."""
import pytest

from golden.cases import CASES
from tdfstat_b200 import host, synth


def _ini_with(tmp_path, text):
    ini = synth.write_case(str(tmp_path), CASES["g1_h1_directed"])
    with open(ini, "a") as f:
        f.write(text)
    return ini


def test_gpu_section_defaults(tmp_path):
    job = host.Job(synth.write_case(str(tmp_path), CASES["g1_h1_directed"]))
    assert job.gpu == host.GpuOptions()


def test_gpu_section_values(tmp_path):
    job = host.Job(_ini_with(tmp_path, "\n[gpu]\nform = FP64\ndevice = 1\nsky_batch = 4\n"
                                       "templates_per_chunk = 12   ; comment\n"))
    assert job.gpu == host.GpuOptions(form="fp64", device=1, sky_batch=4, templates_per_chunk=12)


@pytest.mark.parametrize("bad", ["form = half", "templates_per_chunk = 49", "device = -1"])
def test_gpu_section_invalid(tmp_path, bad):
    with pytest.raises(ValueError):
        host.Job(_ini_with(tmp_path, "\n[gpu]\n%s\n" % bad))
