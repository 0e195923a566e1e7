"""CPU tests of the C-ABI boundary: libtdfcuda loads without a GPU, exports
every function include/*.h declares, its structs have the layout a C
compiler gives them, and the no-device path fails with a status (never a
CPU fallback)."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

from tdfstat_b200 import _abi

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(REPO, "include", h) for h in ("tdfcuda.h", "tdfcuda_refabi.h")]


@pytest.fixture(scope="module")
def lib():
    from tdfstat_b200 import build
    build.build()
    return _abi.bind(C.CDLL(_abi.LIB_PATH))


def declared_functions():
    names = []
    for h in HEADERS:
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b([a-z_][a-z0-9_]*)\s*\(", src, flags=re.M):
            name = m.group(1)
            if name not in ("if", "sizeof", "defined"):
                names.append(name)
    return sorted(set(names))


def test_every_declared_function_is_exported(lib):
    names = declared_functions()
    assert "tdf_search_points" in names and "job_core" in names
    nm = subprocess.run(["nm", "-D", "--defined-only", _abi.LIB_PATH], capture_output=True, text=True).stdout
    exported = {l.split()[-1] for l in nm.splitlines() if " T " in l}
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    bound = {n for n, _, _ in _abi.ABI_FUNCTIONS + _abi.REFABI_FUNCTIONS}
    assert set(names) == bound, set(names) ^ bound


def _c_sizeof(header, types):
    src = "#include <stdio.h>\n#include <stddef.h>\n#include \"%s\"\nint main(void){\n" % header
    for t in types:
        src += 'printf("%%zu\\n", sizeof(%s));\n' % t
    src += "return 0;}\n"
    d = tempfile.mkdtemp()
    c = os.path.join(d, "s.c")
    open(c, "w").write(src)
    exe = os.path.join(d, "s")
    subprocess.run(["gcc", "-I" + os.path.join(REPO, "include"), "-o", exe, c], check=True)
    return [int(x) for x in subprocess.run([exe], capture_output=True, text=True).stdout.split()]


def test_struct_layouts_match_c():
    types = ["tdf_detector", "tdf_segment", "tdf_search_opts", "tdf_record", "tdf_kernel_times", "tdf_signal",
             "tdf_coinc_opts", "tdf_coinc_segment", "tdf_coincidence"]
    sizes = _c_sizeof("tdfcuda.h", types)
    py = [C.sizeof(t) for t in (_abi.TdfDetector, _abi.TdfSegment, _abi.TdfSearchOpts, _abi.TdfRecord,
                                _abi.TdfKernelTimes, _abi.TdfSignal, _abi.TdfCoincOpts, _abi.TdfCoincSegment,
                                _abi.TdfCoincidence)]
    assert sizes == py


def test_refabi_struct_sizes(lib):
    """The restated reference structs have the library's view of their size;
    LP64 sizes of the reference's struct.h (Command_line_opts, Signals,
    Search_range, Aux_arrays, Search_settings, Detector_settings, Trigger)."""
    c = _c_sizeof("tdfcuda_refabi.h", ["tdf_ref_Command_line_opts", "tdf_ref_Signals", "tdf_ref_Search_range",
                                        "tdf_ref_Aux_arrays", "tdf_ref_Search_settings", "tdf_ref_Detector_settings",
                                        "tdf_ref_Trigger"])
    assert [lib.tdf_ref_struct_size(i) for i in range(7)] == c
    assert c[6] == 40     # 6 floats + hvl_t {size_t, void*}


def test_no_device_is_an_error_not_a_fallback(lib):
    n = C.c_int32(-1)
    st = lib.tdf_device_count(C.byref(n))
    if st == 0 and n.value > 0:
        pytest.skip("a CUDA device is present")
    seg = _abi.TdfSegment()
    opts = _abi.TdfSearchOpts()
    h = C.c_void_p()
    st = lib.tdf_engine_create(C.byref(seg), C.byref(opts), 0, 0, 0, C.byref(h))
    assert st != 0 and not h.value
    assert lib.tdf_status_string(st)


def test_invalid_arguments(lib):
    h = C.c_void_p()
    assert lib.tdf_engine_create(None, None, 0, 0, 0, C.byref(h)) == _abi.TDF_ERR_INVALID
    assert b"null" in lib.tdf_last_error()
    seg = _abi.TdfSegment()
    seg.nifo = 1
    seg.N = 100
    seg.nfft = 100        # not a power of two
    opts = _abi.TdfSearchOpts()
    assert lib.tdf_engine_create(C.byref(seg), C.byref(opts), 0, 0, 0, C.byref(h)) == _abi.TDF_ERR_INVALID
    assert lib.tdf_status_string(_abi.TDF_ERR_TRIGGER_OVERFLOW) == b"too many triggers in one spindown"
    st = C.c_uint32(0)
    assert lib.tdf_check_bounded_wait(0, 0, C.byref(st)) == _abi.TDF_ERR_INVALID
    assert lib.tdf_check_bounded_wait(0, 1000, None) == _abi.TDF_ERR_INVALID
    assert lib.tdf_check_bounded_wait(0, 1000, C.byref(st)) == _abi.TDF_ERR_NO_DEVICE
    # the segment-slot and tuning entries check their arguments before any device work
    slot = C.c_int32(0)
    assert lib.tdf_engine_add_segment(None, C.byref(seg), C.byref(slot)) == _abi.TDF_ERR_INVALID
    assert lib.tdf_engine_upload_segment(None, 0, C.byref(seg)) == _abi.TDF_ERR_INVALID
    n = C.c_int64(0)
    assert lib.tdf_search_segments_device(None, 0, None, None, None, None, None, C.byref(n),
                                          C.byref(n)) == _abi.TDF_ERR_INVALID
    assert lib.tdf_engine_get_tuning(None, None, None, None) == _abi.TDF_ERR_INVALID
    assert lib.tdf_engine_segment_count(None, None) == _abi.TDF_ERR_INVALID


def test_frequency_range_below_bin_zero_is_refused(lib, tmp_path):
    """A directed range whose frequency band starts below bin 0 makes the
    reference write F before its array (jobcore.c:481-484 with fr[0] < 0,
    heap corruption, seen here as an abort of the reference build); the
    library refuses such a range before it touches a device."""
    import dataclasses
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from golden.cases import CASES
    from tdfstat_b200 import host, synth
    case = dataclasses.replace(CASES["g6_h1l1v1"], gcenter=(100.027, -2e-10, 0.7, 0.9))
    job = host.Job(synth.write_case(str(tmp_path), case))
    assert job.range.fr[0] < 0
    seg, opts = job.segment(), job.search_opts()
    h = C.c_void_p()
    assert lib.tdf_engine_create(C.byref(seg), C.byref(opts), 0, 0, 0, C.byref(h)) == _abi.TDF_ERR_INVALID
    assert b"fr range" in lib.tdf_last_error()


def test_engine_module_refuses_missing_library(tmp_path):
    from tdfstat_b200 import engine
    with pytest.raises(RuntimeError):
        engine.load_library(str(tmp_path / "nope.so"))
