"""Failure detection of the bounded waits, without a GPU fault: a warp waits
on a barrier whose copy never arrives (nothing is issued), then one thread on
a block count that nothing raises (the fused passes' row-block wait); each
wait gives up after a short limit, the kernel reports TDF_WAIT_TIMEOUT_BIT
and TDF_ORDER_TIMEOUT_BIT, the host reads them, and the device stays
usable."""
import ctypes as C
import time

import pytest

from tdfstat_b200 import _abi

pytestmark = pytest.mark.gpu

TDF_WAIT_TIMEOUT_BIT = 2
TDF_ORDER_TIMEOUT_BIT = 8


def test_wait_gives_up_and_reports(golden):
    from tdfstat_b200.engine import Engine, load_library
    lib = load_library()
    st = C.c_uint32(0)
    t0 = time.monotonic()
    assert lib.tdf_check_bounded_wait(0, 1000, C.byref(st)) == _abi.TDF_OK
    assert time.monotonic() - t0 < 5.0
    assert st.value & TDF_WAIT_TIMEOUT_BIT
    assert st.value & TDF_ORDER_TIMEOUT_BIT
    # the context is intact: a search right after gives its records
    g = golden("g2_h1l1_inj")
    eng = Engine.from_job(g.job32, form="split")
    res = eng.search(*g.job32.sky_points())
    assert len(res) > 0
    eng.close()
