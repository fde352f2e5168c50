"""C-ABI checks that need no GPU: the library loads, exports every entry point
include/ymflow.h declares, and fails cleanly (status + message, no abort)
where no B200 is present."""
import ctypes
import re

import pytest

from conftest import ROOT

HEADER = ROOT / "include" / "ymflow.h"


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"YMFLOW_API[^;(]*?\b(ymflow_\w+)\s*\(", text)))


def header_defines():
    return {m.group(1): int(m.group(2)) for m in
            re.finditer(r"#define\s+(YMFLOW_\w+)\s+\(?(-?\d+)\)?", HEADER.read_text())}


def test_library_exports_every_declared_symbol():
    from latticeyangmills_b200 import _native as N

    lib = N.load()
    names = declared_symbols()
    assert len(names) >= 19
    for name in names:
        assert hasattr(lib, name), name
    assert sorted(N.EXPORTS) == names


def test_status_and_enum_values_match_header():
    from latticeyangmills_b200 import _native as N

    d = header_defines()
    assert d["YMFLOW_OK"] == N.OK
    assert d["YMFLOW_ERR_ARG"] == N.ERR_ARG and d["YMFLOW_ERR_CUDA"] == N.ERR_CUDA
    assert d["YMFLOW_ERR_NONFINITE"] == N.ERR_NONFINITE and d["YMFLOW_ERR_CAPACITY"] == N.ERR_CAPACITY
    assert d["YMFLOW_ERR_STATE"] == N.ERR_STATE and d["YMFLOW_ERR_NODEVICE"] == N.ERR_NODEVICE
    assert d["YMFLOW_ERR_UNITARITY"] == N.ERR_UNITARITY and d["YMFLOW_ERR_OOM"] == N.ERR_OOM
    assert (d["YMFLOW_FP64"], d["YMFLOW_FP32_18"], d["YMFLOW_FP32_12"]) == (N.FP64, N.FP32_18, N.FP32_12)
    assert (d["YMFLOW_FIELD_COLD"], d["YMFLOW_FIELD_EXPIAH"], d["YMFLOW_FIELD_HOT"], d["YMFLOW_FIELD_CURRENT"]) == (
        N.FIELD_COLD, N.FIELD_EXPIAH, N.FIELD_HOT, N.FIELD_CURRENT)
    assert (d["YMFLOW_OPT_BLOCK"], d["YMFLOW_OPT_GRAPH"], d["YMFLOW_OPT_OBS_BLOCK"], d["YMFLOW_OPT_STAGE_FORM"]) == (
        N.OPT_BLOCK, N.OPT_GRAPH, N.OPT_OBS_BLOCK, N.OPT_STAGE_FORM)


def test_obs_struct_layout():
    from latticeyangmills_b200 import _native as N

    # int32 step, int32 pad, 5 doubles
    assert ctypes.sizeof(N.Obs) == 48
    assert N.Obs.t.offset == 8 and N.Obs.t2E.offset == 40


def test_argument_errors_without_device():
    from latticeyangmills_b200 import _native as N

    lib = N.load()
    assert lib.ymflow_version().startswith(b"ymflow")
    st = ctypes.c_int(99)
    assert not lib.ymflow_create(None, 0, 0, ctypes.byref(st))
    assert st.value == N.ERR_ARG
    bad = N._I4(4, 0, 4, 4)
    assert not lib.ymflow_create(bad, 0, 0, ctypes.byref(st)) and st.value == N.ERR_ARG
    assert not lib.ymflow_create(N._I4(4, 4, 4, 4), 7, 0, ctypes.byref(st)) and st.value == N.ERR_ARG
    assert lib.ymflow_last_error(None)
    assert lib.ymflow_flow(None, 0.01, 1, 1, 0, None, 0, None) == N.ERR_ARG
    assert lib.ymflow_upload(None, None) == N.ERR_ARG
    assert lib.ymflow_su3_exp(None, None, 1, 0) == N.ERR_ARG
    lib.ymflow_destroy(None)


@pytest.mark.skipif(__import__("torch").cuda.is_available(), reason="checks the no-device path")
def test_no_device_is_reported_not_aborted():
    from latticeyangmills_b200 import GluonField, YmflowError
    from latticeyangmills_b200 import _native as N

    n = ctypes.c_int(-1)
    assert N.load().ymflow_device_count(ctypes.byref(n)) == N.OK and n.value == 0
    with pytest.raises(YmflowError) as e:
        GluonField((4, 4, 4, 4))
    assert e.value.status == N.ERR_NODEVICE
