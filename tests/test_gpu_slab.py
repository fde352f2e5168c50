"""One configuration split along t into slab contexts (ymflow_create_slab)
against the whole-lattice context: the same seeded links, the same flow.
Links must agree bit for bit (every link's arithmetic is the same); the
observables differ only in the order of the final sums."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N8 = (8, 4, 4, 10)  # spatial volume 128 (whole warp groups), 10 time slices


def whole(precision, n=N8, seed=11, steps=6, every=2):
    # slabs and the whole lattice run the same stage form (the default for
    # their sizes: the fused kernel for these small FP32 lattices, the
    # two-kernel stage in FP64)
    from latticeyangmills_b200 import GluonField

    with GluonField(n, precision) as f:
        f.init_links("expiah", 0.4, seed)
        U0 = f.download()
        rows = f.flow(0.02, steps, every, reunit_every=3 if precision != "fp64" else 0)
        return U0, rows, f.download()


def close_rows(got, want, precision):
    """plaquette, energy and t^2 E relative; the charge absolute (it crosses zero)."""
    rtol, qtol = (1e-12, 1e-12) if precision == "fp64" else (1e-6, 1e-6)
    np.testing.assert_allclose(got[:, [2, 4, 5]], want[:, [2, 4, 5]], rtol=rtol, atol=1e-15)
    assert np.abs(got[:, 3] - want[:, 3]).max() < qtol


def split(n, parts):
    t0 = 0
    for nt in parts:
        yield t0, nt
        t0 += nt


@pytest.mark.parametrize("precision", ["fp64", "fp32_18", "fp32_12"])
@pytest.mark.parametrize("parts", [(10,), (5, 5), (4, 3, 3), (1, 2, 7)])
def test_group_flow_matches_whole_lattice(precision, parts):
    from latticeyangmills_b200 import GluonField, slab_group_flow

    U0, rows, U1 = whole(precision)
    slabs = [GluonField.slab(N8, t0, nt, precision) for t0, nt in split(N8, parts)]
    try:
        for s in slabs:
            s.init_links("expiah", 0.4, 11)
        # the seeded slab holds exactly its slices of the whole-lattice field
        assert np.array_equal(np.concatenate([s.download() for s in slabs]), U0)
        got = slab_group_flow(slabs, 0.02, 6, 2, reunit_every=3 if precision != "fp64" else 0)
        after = np.concatenate([s.download() for s in slabs])
    finally:
        for s in slabs:
            s.close()
    # The slabs' stage kernel stores its boundary links into its neighbours'
    # halos as well; it is a separate kernel, whose FP32 multiply-adds the
    # compiler may fuse differently: FP64 is bit-identical, FP32 equal to its
    # rounding.
    diff = np.abs(after - U1).max()
    print(precision, parts, "max |dU|", diff, "max |d obs|", np.abs(got[:, 2:] - rows[:, 2:]).max())
    assert diff == 0.0 if precision == "fp64" else diff < 1e-5
    assert got.shape == rows.shape
    assert np.array_equal(got[:, :2], rows[:, :2])
    close_rows(got, rows, precision)


@pytest.mark.parametrize("precision", ["fp64", "fp32_18"])
def test_copy_exchange_matches_fused_exchange(precision, monkeypatch):
    """The halo exchange as copies after each stage (the fallback for GPUs
    that cannot reach each other's memory) gives the same links as the
    exchange fused into the stage kernel."""
    from latticeyangmills_b200 import GluonField, slab_group_flow

    out = {}
    for mode in ("fused", "copy"):
        if mode == "copy":
            monkeypatch.setenv("YMFLOW_SLAB_COPY_EXCHANGE", "1")
        slabs = [GluonField.slab(N8, t0, nt, precision) for t0, nt in split(N8, (4, 3, 3))]
        try:
            for sl in slabs:
                sl.init_links("expiah", 0.4, 11)
            rows = slab_group_flow(slabs, 0.02, 6, 3)
            out[mode] = (rows, np.concatenate([sl.download() for sl in slabs]))
        finally:
            for sl in slabs:
                sl.close()
    diff = np.abs(out["fused"][1] - out["copy"][1]).max()
    print(precision, "fused vs copy max |dU|", diff)
    assert diff == 0.0 if precision == "fp64" else diff < 1e-5
    close_rows(out["fused"][0], out["copy"][0], precision)


def test_uploaded_slabs_match_whole_lattice():
    from latticeyangmills_b200 import GluonField, slab_group_flow

    U0, rows, U1 = whole("fp64", seed=5)
    flat = U0.reshape(N8[3], -1)
    slabs = [GluonField.slab(N8, t0, nt, "fp64") for t0, nt in split(N8, (6, 4))]
    try:
        for s in slabs:
            s.upload(flat[s.t0:s.t0 + s.nt])
        got = slab_group_flow(slabs, 0.02, 6, 2)
        after = np.concatenate([s.download() for s in slabs])
    finally:
        for s in slabs:
            s.close()
    assert np.array_equal(after, U1)
    np.testing.assert_allclose(got[:, 2:], rows[:, 2:], rtol=1e-12, atol=1e-15)


@pytest.mark.parametrize("precision", ["fp64", "fp32_18"])
def test_nccl_single_rank_slab_matches_whole_lattice(precision):
    """One rank whose slab is the whole time extent exchanges its halos with
    itself through NCCL: the path a multi-GPU run takes, on one GPU."""
    from latticeyangmills_b200 import GluonField, nccl_unique_id

    U0, rows, U1 = whole(precision)
    with GluonField.slab(N8, 0, N8[3], precision) as s:
        s.init_links("expiah", 0.4, 11)
        s.connect(nccl_unique_id(), 0, 1, 0, 0)
        o = s.observables()
        got = s.flow(0.02, 6, 2, reunit_every=3 if precision != "fp64" else 0)
        after = s.download()
    assert np.array_equal(after, U1)
    close_rows(got, rows, precision)
    assert abs(o.plaq - rows[0, 2]) < 1e-14


def test_slab_errors():
    from latticeyangmills_b200 import GluonField, YmflowError, slab_group_flow

    with pytest.raises(YmflowError):
        GluonField.slab((3, 3, 3, 8), 0, 4)  # spatial volume not a multiple of 32
    with pytest.raises(YmflowError):
        GluonField.slab(N8, 8, 4)  # slices beyond the time extent
    a = GluonField.slab(N8, 0, 5, "fp64")
    b = GluonField.slab(N8, 6, 4, "fp64")
    try:
        a.init_links("cold")
        b.init_links("cold")
        with pytest.raises(YmflowError):
            a.flow(0.01, 1)  # neither connected nor flowed with its group
        with pytest.raises(YmflowError):
            slab_group_flow([a, b], 0.01, 1)  # slice 5 missing
        with pytest.raises(YmflowError):
            a.generate_metropolis(6.0, sweeps=1)
        with pytest.raises(YmflowError):
            a.derivative(0)
    finally:
        a.close()
        b.close()


def test_nccl_then_torch_in_one_process():
    """The slab path loads NCCL at run time; torch imported afterwards in the
    same process must still import (one NCCL, the one torch was built for)."""
    import subprocess
    import sys

    code = ("from latticeyangmills_b200 import GluonField, nccl_unique_id\n"
            "f = GluonField.slab((8, 4, 4, 4), 0, 4, 'fp64'); f.init_links('cold')\n"
            "f.connect(nccl_unique_id(), 0, 1, 0, 0); f.flow(0.01, 1)\n"
            "import torch; print('torch', torch.__version__)\n")
    res = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stderr[-2000:]
    assert "torch" in res.stdout
