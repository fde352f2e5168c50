"""The allocation-free observables entry point (ymflow_observables_noalloc).

It exists for callers that cannot call cudaMalloc where they measure: a host
application that has reserved the device for its own memory pool, or a
latency-critical loop that cannot take an allocation's implicit
synchronisation.  Its scratch is a fixed array inside the library, so it is
checked here against the ordinary entry point (ymflow_observables, which owns
its scratch), on two calls in a row, through the C ABI.

This file sorts last so that a run stopping at the first failure has run
every other test before it; it also passes when run alone in a fresh process."""
import ctypes

import numpy as np
import pytest

from conftest import case_field, load_case

pytestmark = pytest.mark.gpu

RTOL = 1e-12  # the FP64 parity tolerance of the other GPU tests


def test_noalloc_observables_match_ymflow_observables_twice():
    import torch

    from latticeyangmills_b200 import GluonField
    from latticeyangmills_b200 import _native as N

    lib = N.load()
    cases = [load_case("g8_metropolis"), load_case("g3456_expiah")]
    side = torch.cuda.Stream()
    # two calls in a row, different lattices: the first on the default stream,
    # the second (a smaller lattice, after the first's partials stay in the
    # shared array) on a non-default stream
    for call, case in enumerate(cases):
        n = tuple(case["dims"])
        U = case_field(case)
        with GluonField(n, "fp64") as f:
            f.upload(U)
            want = f.observables()
        # the caller owns the device buffers (allocated here by the test, not by the entry point)
        links = torch.from_numpy(np.ascontiguousarray(U).reshape(-1)).to("cuda")
        out = torch.full((4,), float("nan"), dtype=torch.float64, device="cuda")
        dims = (ctypes.c_int * 4)(*n)
        torch.cuda.synchronize()
        stream = None if call == 0 else ctypes.c_void_p(side.cuda_stream)
        st = lib.ymflow_observables_noalloc(ctypes.c_void_p(links.data_ptr()), dims,
                                            ctypes.c_void_p(out.data_ptr()), stream)
        assert st == N.OK, (call, st)
        if call == 0:
            torch.cuda.synchronize()
        else:
            side.synchronize()
        plaq, topc, energy, flag = out.cpu().numpy().tolist()
        assert flag == 0.0
        np.testing.assert_allclose(plaq, want.plaq, rtol=RTOL, atol=0)
        np.testing.assert_allclose(energy, want.energy, rtol=RTOL, atol=0)
        assert abs(topc - want.topc) <= RTOL * abs(want.energy) / (512 * np.pi ** 2) + 1e-300
        # and against the reference's own numbers for the configuration as read
        ref = case["rows"][0]
        np.testing.assert_allclose([plaq, energy], [ref[2], ref[4]], rtol=RTOL, atol=0)


def test_noalloc_rejects_lattices_beyond_its_scratch():
    import torch

    from latticeyangmills_b200 import _native as N

    lib = N.load()
    small = torch.zeros(72, dtype=torch.float64, device="cuda")
    out = torch.zeros(4, dtype=torch.float64, device="cuda")
    too_big = (ctypes.c_int * 4)(64, 64, 64, 64)  # 16.8M sites > YMFLOW_NOALLOC_MAX_SITES
    assert 64 ** 4 > N.NOALLOC_MAX_SITES
    st = lib.ymflow_observables_noalloc(ctypes.c_void_p(small.data_ptr()), too_big,
                                        ctypes.c_void_p(out.data_ptr()), None)
    assert st == N.ERR_CAPACITY
    bad = (ctypes.c_int * 4)(4, 0, 4, 4)
    assert lib.ymflow_observables_noalloc(ctypes.c_void_p(small.data_ptr()), bad,
                                          ctypes.c_void_p(out.data_ptr()), None) == N.ERR_ARG
    assert lib.ymflow_observables_noalloc(None, bad, None, None) == N.ERR_ARG
