"""Error paths of the C ABI on the GPU: every failure is a status code and a
message, none aborts or leaves the context unusable."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_flow_before_upload_is_a_state_error():
    from latticeyangmills_b200 import GluonField, YmflowError
    from latticeyangmills_b200 import _native as N

    with GluonField((4, 4, 4, 4)) as f:
        with pytest.raises(YmflowError) as e:
            f.flow(0.01, 1, 1)
        assert e.value.status == N.ERR_STATE


def test_output_capacity_checked_before_work():
    from latticeyangmills_b200 import GluonField
    from latticeyangmills_b200 import _native as N

    with GluonField((4, 4, 4, 4)) as f:
        f.init_links("expiah", 0.3, 1)
        out = (N.Obs * 2)()
        n = ctypes.c_int(-1)
        st = N.load().ymflow_flow(f.ctx, 0.01, 5, 1, 0, out, 2, ctypes.byref(n))
        assert st == N.ERR_CAPACITY and n.value == 0
        assert b"rows" in N.load().ymflow_last_error(f.ctx)
        assert f.observables().step == 0  # nothing flowed


def test_nan_link_is_reported_and_context_recovers():
    from latticeyangmills_b200 import GluonField, YmflowError
    from latticeyangmills_b200 import _native as N

    n = (4, 4, 4, 4)
    with GluonField(n) as f:
        f.init_links("expiah", 0.3, 1)
        U = f.download()
        bad = U.copy()
        bad[1, 2, 3, 0, 2, 5] = np.nan
        f.upload(bad)
        with pytest.raises(YmflowError) as e:
            f.flow(0.01, 2, 1)
        assert e.value.status == N.ERR_NONFINITE
        f.upload(U)  # the same context keeps working
        rows = f.flow(0.01, 2, 1)
        assert np.isfinite(rows).all()


def test_bad_options_rejected():
    from latticeyangmills_b200 import GluonField, YmflowError
    from latticeyangmills_b200 import _native as N

    with GluonField((4, 4, 4, 4)) as f:
        for key, val in [(N.OPT_BLOCK, 64), (N.OPT_BLOCK, 256), (N.OPT_OBS_BLOCK, 48), (99, 1)]:
            with pytest.raises(YmflowError):
                f.set_option(key, val)


def test_wrong_size_upload_rejected_on_host():
    from latticeyangmills_b200 import GluonField

    with GluonField((4, 4, 4, 4)) as f:
        with pytest.raises(ValueError):
            f.upload(np.zeros(10))


def test_fma_peak_is_measured():
    import ctypes

    from latticeyangmills_b200 import _native as N

    tf = {}
    for p in (N.FP32_18, N.FP64):
        v = ctypes.c_double(0.0)
        assert N.load().ymflow_fma_peak(0, p, ctypes.byref(v)) == N.OK
        tf[p] = v.value
    print("FMA peak TFLOP/s: fp32", tf[N.FP32_18], "fp64", tf[N.FP64])
    assert 20.0 < tf[N.FP32_18] < 200.0
    assert 5.0 < tf[N.FP64] < tf[N.FP32_18]
    assert N.load().ymflow_fma_peak(0, 7, ctypes.byref(ctypes.c_double())) == N.ERR_ARG


def test_pinned_host_buffers_feed_uploads():
    """ymflow_host_alloc / ymflow_host_free: page-locked staging for uploads."""
    import ctypes

    import numpy as np

    from latticeyangmills_b200 import GluonField
    from latticeyangmills_b200 import _native as N

    lib = N.load()
    p = ctypes.c_void_p()
    assert lib.ymflow_host_alloc(0, ctypes.byref(p)) == N.ERR_ARG
    assert lib.ymflow_host_alloc(-5, ctypes.byref(p)) == N.ERR_ARG
    n = (4, 4, 4, 4)
    count = 4 * 256 * 18
    assert lib.ymflow_host_alloc(count * 8, ctypes.byref(p)) == N.OK and p.value
    buf = np.ctypeslib.as_array(ctypes.cast(p, ctypes.POINTER(ctypes.c_double)), shape=(count,))
    with GluonField(n, "fp64") as f:
        f.init_links("expiah", 0.3, 4)
        U = f.download()
        buf[:] = U.reshape(-1)
        f.init_links("cold")
        assert lib.ymflow_upload(f.ctx, p) == N.OK
        assert np.array_equal(f.download(), U)
    assert lib.ymflow_host_free(p) == N.OK


@pytest.mark.parametrize("precision", ["fp64", "fp32_18"])
def test_checkpoint_resume_continues_the_flow(precision):
    """Download mid-flow, upload into a fresh context, set (step, t): the
    remaining rows and links equal those of an unbroken flow."""
    import numpy as np

    from latticeyangmills_b200 import GluonField

    n = (8, 8, 8, 8)
    kw = dict(reunit_every=5) if precision != "fp64" else {}
    with GluonField(n, precision) as f:
        f.init_links("expiah", 0.35, 8)
        whole = f.flow(0.02, 20, 5, **kw)
        end = f.download()
    with GluonField(n, precision) as f:
        f.init_links("expiah", 0.35, 8)
        first = f.flow(0.02, 10, 5, **kw)
        ckpt = f.download()
    with GluonField(n, precision) as g:
        g.upload(ckpt)
        g.set_time(int(first[-1, 0]), first[-1, 1])
        rest = g.flow(0.02, 10, 5, **kw)
        resumed = g.download()
    assert np.array_equal(rest[:, :2], whole[2:, :2])  # steps and t continue exactly
    if precision == "fp64":
        assert np.array_equal(resumed, end)
        np.testing.assert_array_equal(rest[:, 2:], whole[2:, 2:])
    else:  # the checkpoint passes through the FP64 .bin layout: equal to FP32 rounding of that round trip
        assert np.abs(resumed - end).max() < 1e-5
        np.testing.assert_allclose(rest[:, 2:], whole[2:, 2:], rtol=1e-5)
