"""The pass order of the fused spindown launch (TDF_FUSED_PASSES=1), checked
on the CPU against the library's own mapping (tdf_spin_order_item runs the
function the kernel runs):

  * tickets 0 .. 2*nt*blocks-1 name every column and row block exactly once;
  * every column block of a template comes before all of its row blocks;
  * persistent CTAs that each hold a current and a prefetched ticket,
    publish a finished column block before they wait, and wait only for
    their template's column blocks always finish -- the deadlock-freedom
    argument of the kernel, simulated for random sizes, lags, CTA counts
    and item durations, down to a single CTA.
"""
import ctypes as C
import random

import pytest

from tdfstat_b200 import _abi


@pytest.fixture(scope="module")
def lib():
    from tdfstat_b200 import build
    build.build()
    return _abi.bind(C.CDLL(_abi.LIB_PATH))


def _order(lib, nt, blocks, lag):
    """[(row, template, block)] for tickets 0 .. 2*nt*blocks-1."""
    b, k, r = C.c_int32(), C.c_int32(), C.c_int32()
    out = []
    for t in range(2 * nt * blocks):
        assert lib.tdf_spin_order_item(nt, blocks, lag, t, C.byref(b), C.byref(k), C.byref(r)) == _abi.TDF_OK
        out.append((bool(r.value), b.value, k.value))
    return out


@pytest.mark.parametrize("blocks", [1, 3, 32, 64])
def test_order_is_a_bijection_with_columns_first(lib, blocks):
    for nt in (1, 2, 3, 5, 8, 13, 48, 96):
        for lag in (1, 2, 3, 8, 200):
            if nt * blocks > 2048 and lag not in (1, 3):
                continue
            items = _order(lib, nt, blocks, lag)
            seen = {it: t for t, it in enumerate(items)}
            assert len(seen) == len(items) == 2 * nt * blocks
            for row, b, k in items:
                assert 0 <= b < nt and 0 <= k < blocks
            for b in range(nt):
                last_col = max(seen[(False, b, k)] for k in range(blocks))
                first_row = min(seen[(True, b, k)] for k in range(blocks))
                assert last_col < first_row, (nt, blocks, lag, b)


def test_rows_trail_columns_by_the_lag(lib):
    """With lag D (< nt), the row blocks of template b start after the
    column blocks of template b + D have been handed out."""
    nt, blocks, lag = 20, 8, 3
    items = _order(lib, nt, blocks, lag)
    seen = {it: t for t, it in enumerate(items)}
    for b in range(nt - lag):
        assert min(seen[(True, b, k)] for k in range(blocks)) > max(seen[(False, b + lag, k)] for k in range(blocks))


def test_invalid_arguments(lib):
    b, k, r = C.c_int32(), C.c_int32(), C.c_int32()
    f = lib.tdf_spin_order_item
    assert f(4, 8, 3, 0, None, C.byref(k), C.byref(r)) == _abi.TDF_ERR_INVALID
    assert f(0, 8, 3, 0, C.byref(b), C.byref(k), C.byref(r)) == _abi.TDF_ERR_INVALID
    assert f(4, 0, 3, 0, C.byref(b), C.byref(k), C.byref(r)) == _abi.TDF_ERR_INVALID
    assert f(4, 8, 0, 0, C.byref(b), C.byref(k), C.byref(r)) == _abi.TDF_ERR_INVALID
    assert f(4, 8, 3, 64, C.byref(b), C.byref(k), C.byref(r)) == _abi.TDF_ERR_INVALID
    assert f(4, 8, 3, 63, C.byref(b), C.byref(k), C.byref(r)) == _abi.TDF_OK


def _simulate(items, nt, blocks, nctas, rnd):
    """Persistent CTAs as k_spinpass runs them; True when every CTA finishes."""
    total = len(items)
    nxt = 0
    done_cols = [0] * nt
    ctas = []
    for _ in range(nctas):
        ctas.append({"cur": nxt, "pend": -1, "item": None, "left": 0, "fin": False})
        nxt += 1
    while True:
        progress = False
        for c in ctas:
            if c["fin"]:
                continue
            if c["item"] is None:
                # item start: publish the previous column block, take the next ticket
                if c["pend"] >= 0:
                    done_cols[c["pend"]] += 1
                    c["pend"] = -1
                if c["cur"] >= total:
                    c["fin"] = True
                    progress = True
                    continue
                c["nxt"] = nxt
                nxt += 1
                c["item"] = items[c["cur"]]
                c["left"] = rnd.randint(1, 6)
                progress = True
            row, b, _ = c["item"]
            if row and done_cols[b] < blocks:
                continue   # the row block waits for its template's column blocks
            c["left"] -= 1
            progress = True
            if c["left"] == 0:
                if not row:
                    c["pend"] = b
                c["item"] = None
                c["cur"] = c["nxt"]
        if all(c["fin"] for c in ctas):
            return True
        if not progress:
            return False


def test_persistent_ctas_always_finish(lib):
    rnd = random.Random(1234)
    cache = {}
    for _ in range(120):
        nt = rnd.randint(1, 24)
        blocks = rnd.choice([1, 2, 4, 8])
        lag = rnd.randint(1, 10)
        nctas = rnd.randint(1, 40)
        key = (nt, blocks, lag)
        if key not in cache:
            cache[key] = _order(lib, nt, blocks, lag)
        assert _simulate(cache[key], nt, blocks, nctas, rnd), (nt, blocks, lag, nctas)
