"""The C ABI's argument checks, which run before any device work: every bad
call returns its status code (and a message) on a machine without a GPU."""
import ctypes

import pytest

from latticeyangmills_b200 import _native as N


def create(dims, precision=0, device=0):
    st = ctypes.c_int(0)
    d = None if dims is None else (ctypes.c_int * 4)(*dims)
    ctx = N.load().ymflow_create(d, precision, device, ctypes.byref(st))
    return ctx, st.value, N.load().ymflow_last_error(None).decode()


def create_slab(dims, t0, nt, precision=0, device=0):
    st = ctypes.c_int(0)
    ctx = N.load().ymflow_create_slab((ctypes.c_int * 4)(*dims), t0, nt, precision, device, ctypes.byref(st))
    return ctx, st.value, N.load().ymflow_last_error(None).decode()


@pytest.mark.parametrize("dims,prec,msg", [
    (None, 0, "dims is NULL"),
    ((0, 4, 4, 4), 0, "extents"),
    ((4, 4, 4, 5000), 0, "extents"),
    ((4, 4, 4, 4), 7, "unknown precision"),
    ((4096, 4096, 256, 1), 0, "too large"),
])
def test_create_rejects_bad_arguments(dims, prec, msg):
    ctx, st, err = create(dims, prec)
    assert not ctx and st == N.ERR_ARG and msg in err


@pytest.mark.parametrize("dims,t0,nt,msg", [
    ((8, 4, 4, 8), 6, 4, "outside"),
    ((8, 4, 4, 8), -1, 2, "outside"),
    ((8, 4, 4, 8), 0, 0, "outside"),
    ((3, 3, 3, 8), 0, 4, "divisible by 32"),
])
def test_create_slab_rejects_bad_arguments(dims, t0, nt, msg):
    ctx, st, err = create_slab(dims, t0, nt)
    assert not ctx and st == N.ERR_ARG and msg in err


def test_calls_without_a_context_or_buffer():
    lib = N.load()
    q = (ctypes.c_double * 18)()
    assert lib.ymflow_su3_exp(q, q, -1, 0) == N.ERR_ARG
    assert lib.ymflow_su3_exp(None, q, 1, 0) == N.ERR_ARG
    assert lib.ymflow_su3_exp(q, q, 0, 0) == N.OK  # nothing to do
    assert lib.ymflow_fma_peak(0, 9, ctypes.byref(ctypes.c_double())) == N.ERR_ARG
    assert lib.ymflow_fma_peak(0, 0, None) == N.ERR_ARG
    assert lib.ymflow_host_alloc(0, ctypes.byref(ctypes.c_void_p())) == N.ERR_ARG
    assert lib.ymflow_device_count(None) == N.ERR_ARG
    assert lib.ymflow_nccl_unique_id(None) == N.ERR_ARG
    for fn in ("ymflow_reset_time", "ymflow_observables", "ymflow_upload", "ymflow_download"):
        args = [None] * len(getattr(lib, fn).argtypes)
        assert getattr(lib, fn)(*args) == N.ERR_ARG, fn
    assert lib.ymflow_set_time(None, 0, 0.0) == N.ERR_ARG
    assert lib.ymflow_set_option(None, N.OPT_STAGE_FORM, 1) == N.ERR_ARG
    ms = ctypes.c_float()
    assert lib.ymflow_time_steps(None, 0.01, 1, ctypes.byref(ms), None) == N.ERR_ARG
    assert lib.ymflow_time_kernels(None, 0.01, 1, ctypes.byref(ms), None, None) == N.ERR_ARG
    assert lib.ymflow_load_file(None, b"x", 0, 0) == N.ERR_ARG
    assert lib.ymflow_slab_group_flow(None, 0, 0.01, 1, 0, 0, None, 0, None) == N.ERR_ARG


def test_allocation_free_entry_point_checks_before_the_device():
    lib = N.load()
    out = ctypes.c_void_p(1)
    big = (ctypes.c_int * 4)(256, 256, 256, 1)  # 16.7 M sites > YMFLOW_NOALLOC_MAX_SITES
    assert lib.ymflow_observables_noalloc(None, big, out, None) == N.ERR_ARG
    assert lib.ymflow_observables_noalloc(ctypes.c_void_p(1), big, out, None) == N.ERR_CAPACITY
    bad = (ctypes.c_int * 4)(4, 0, 4, 4)
    assert lib.ymflow_observables_noalloc(ctypes.c_void_p(1), bad, out, None) == N.ERR_ARG
    # a caller's pool offset that is not 16-byte aligned (links) or 8-byte aligned
    # (output) is refused before anything touches a device
    small = (ctypes.c_int * 4)(4, 4, 4, 4)
    aligned = ctypes.c_void_p(4096)
    assert lib.ymflow_observables_noalloc(ctypes.c_void_p(4096 + 8), small, aligned, None) == N.ERR_ARG
    assert lib.ymflow_observables_noalloc(aligned, small, ctypes.c_void_p(4096 + 4), None) == N.ERR_ARG


def test_valid_create_without_a_b200_says_so():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    ctx, st, err = create((4, 4, 4, 4))
    assert not ctx and st == N.ERR_NODEVICE and err
    ctx, st, err = create_slab((8, 4, 4, 8), 0, 4)
    assert not ctx and st == N.ERR_NODEVICE
    count = ctypes.c_int(-1)
    assert N.load().ymflow_device_count(ctypes.byref(count)) == N.OK and count.value == 0
