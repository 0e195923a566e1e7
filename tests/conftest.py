import os
import shutil
import sys
import tempfile

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
for p in (REPO, HERE):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the libtdfcuda kernels")


@pytest.fixture(scope="session")
def oracle():
    import refkit
    refkit.build_oracle()
    return refkit.load_oracle()


class GoldenCase:
    """A golden case written to a temp dir, with its reference records."""

    def __init__(self, name):
        from tdfstat_b200 import host, synth
        import refkit
        from golden.cases import CASES, GOLDEN_DIR, input_checksum
        self.name = name
        self.case = CASES[name]
        self.root = tempfile.mkdtemp(prefix="tdf_" + name + "_")
        self.ini = synth.write_case(self.root, self.case)
        self.checksum = input_checksum(self.root)
        g = np.load(os.path.join(GOLDEN_DIR, name + ".npz"))
        self.expected_checksum = str(g["checksum"])
        self.ref = {}
        for which in ("f64", "f32"):
            lens = g[which + "_lens"]
            flat = g[which + "_pairs"]
            pairs = np.split(flat, np.cumsum(lens)[:-1]) if len(lens) else []
            self.ref[which] = refkit.Records(g[which + "_hdr"], pairs, g[which + "_pm"])
        self.job = host.Job(self.ini, float_build=False)
        self.job32 = host.Job(self.ini, float_build=True)

    def close(self):
        shutil.rmtree(self.root, ignore_errors=True)


_CACHE = {}


@pytest.fixture(scope="session")
def golden():
    def get(name):
        if name not in _CACHE:
            _CACHE[name] = GoldenCase(name)
        return _CACHE[name]
    yield get
    for c in _CACHE.values():
        c.close()
