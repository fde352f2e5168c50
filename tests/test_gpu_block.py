"""One configuration decomposed in several directions into blocks
(ymflow_create_block + ymflow_block_group_flow): the reference's Cartesian
domain decomposition (src/ParallelTools/parallel.cpp:57-100) with the
second-neighbour halo of the clover (:117-140).  On one GPU the blocks flow
together; links equal the whole-lattice flow bit for bit (the same kernels on
the same neighbour data), observables to the parity tolerance."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def own_part(U, origin, extent):
    """The block's own sites of a whole field (t, z, y, x, 4, 18), .bin order."""
    x0, y0, z0, t0 = origin
    ex, ey, ez, et = extent
    return np.ascontiguousarray(U[t0:t0 + et, z0:z0 + ez, y0:y0 + ey, x0:x0 + ex])


def flow_both(n, layout, prec, steps=4, every=2, reunit=0, form=None):
    from latticeyangmills_b200 import GluonField, _native as N, block_group_flow

    grid, blocks = layout
    with GluonField(n, prec) as f:
        if form is not None:
            f.set_option(N.OPT_STAGE_FORM, form)
        f.init_links("expiah", 0.4, 5)
        U0 = f.download()
        want = f.flow(0.02, steps, every, reunit_every=reunit)
        want_links = f.download()
    ctxs = [GluonField.block(n, o, e, prec) for o, e in blocks]
    try:
        for b, (o, e) in zip(ctxs, blocks):
            if form is not None:
                b.set_option(N.OPT_STAGE_FORM, form)
            b.upload(own_part(U0, o, e))
        got = block_group_flow(ctxs, grid, 0.02, steps, every, reunit_every=reunit)
        links = np.empty_like(want_links)
        for b, (o, e) in zip(ctxs, blocks):
            x0, y0, z0, t0 = o
            ex, ey, ez, et = e
            links[t0:t0 + et, z0:z0 + ez, y0:y0 + ey, x0:x0 + ex] = b.download()
    finally:
        for b in ctxs:
            b.close()
    return want, want_links, got, links


@pytest.mark.parametrize("n,sub,prec", [
    ((8, 4, 6, 10), (8, 4, 3, 5), "fp64"),      # z and t
    ((8, 4, 6, 10), (8, 4, 3, 5), "fp32_12"),
    ((8, 8, 8, 8), (4, 4, 4, 4), "fp64"),       # every direction: 16 blocks
    ((8, 4, 4, 6), (4, 4, 4, 3), "fp32_18"),    # x and t
    ((6, 6, 4, 4), (3, 2, 4, 4), "fp64"),       # x and y, a 2 x 3 grid
])
def test_blocks_equal_the_whole_lattice(n, sub, prec):
    from latticeyangmills_b200 import block_layout

    reunit = 2 if prec != "fp64" else 0
    want, want_links, got, links = flow_both(n, block_layout(n, sub), prec, reunit=reunit)
    np.testing.assert_array_equal(links, want_links)
    np.testing.assert_array_equal(got[:, :2], want[:, :2])
    np.testing.assert_allclose(got[:, [2, 4, 5]], want[:, [2, 4, 5]], rtol=1e-12)
    assert np.abs(got[:, 3] - want[:, 3]).max() < 1e-12


def test_uneven_blocks_and_the_fused_form():
    # t split 4 + 6, z split 2 + 4, by hand; the FP32 fused stage form
    n = (8, 4, 6, 10)
    blocks = [((0, 0, 0, 0), (8, 4, 2, 4)), ((0, 0, 2, 0), (8, 4, 4, 4)),
              ((0, 0, 0, 4), (8, 4, 2, 6)), ((0, 0, 2, 4), (8, 4, 4, 6))]
    want, want_links, got, links = flow_both(n, ([1, 1, 2, 2], blocks), "fp32_12", form=0, reunit=3)
    np.testing.assert_array_equal(links, want_links)
    np.testing.assert_allclose(got[:, [2, 4, 5]], want[:, [2, 4, 5]], rtol=1e-12)


def test_block_refusals():
    from latticeyangmills_b200 import GluonField, YmflowError, block_group_flow, block_layout

    n = (8, 4, 6, 10)
    with pytest.raises(YmflowError):
        GluonField.block(n, (0, 0, 4, 0), (8, 4, 3, 5))  # past the z extent
    grid, blocks = block_layout(n, (8, 4, 3, 5))
    ctxs = [GluonField.block(n, o, e, "fp64") for o, e in blocks]
    try:
        with pytest.raises(YmflowError):
            ctxs[0].init_links("expiah", 0.4, 1)  # blocks take uploads
        for b in ctxs:
            b.upload(np.zeros((b.sites, 4, 18)) + np.eye(3, dtype=complex).view(float).reshape(18))
        with pytest.raises(YmflowError):
            ctxs[0].flow(0.01, 1, 1)  # a single block has no neighbours to refresh its halos
        with pytest.raises(YmflowError):
            block_group_flow(ctxs, [1, 1, 4, 1], 0.01, 1, 1)  # grid does not match the halos
        with pytest.raises(YmflowError):
            block_group_flow(ctxs[::-1], grid, 0.01, 1, 1)  # not in grid order
        rows = block_group_flow(ctxs, grid, 0.01, 1, 1)  # cold field: plaquette 1
        assert abs(rows[0, 2] - 1.0) < 1e-14
    finally:
        for b in ctxs:
            b.close()
