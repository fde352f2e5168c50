"""One configuration split along t into slab contexts (ymflow_create_slab)
against the whole-lattice context: the same seeded links, the same flow.
Links must agree bit for bit (every link's arithmetic is the same); the
observables differ only in the order of the final sums."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N8 = (8, 4, 4, 10)  # spatial volume 128 (whole warp groups), 10 time slices


def whole(precision, n=N8, seed=11, steps=6, every=2):
    from latticeyangmills_b200 import GluonField

    with GluonField(n, precision) as f:
        f.init_links("expiah", 0.4, seed)
        U0 = f.download()
        rows = f.flow(0.02, steps, every, reunit_every=3 if precision != "fp64" else 0)
        return U0, rows, f.download()


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
    assert np.array_equal(after, U1)
    assert got.shape == rows.shape
    assert np.array_equal(got[:, :2], rows[:, :2])
    np.testing.assert_allclose(got[:, 2:], rows[:, 2:], rtol=1e-12, atol=1e-15)


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
    np.testing.assert_allclose(got[:, 2:], rows[:, 2:], rtol=1e-12, atol=1e-15)
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
