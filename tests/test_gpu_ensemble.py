"""Batched ensemble (one persistent launch per stage for many configurations of
uneven sizes) against flowing each configuration on its own."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SIZES = [(4, 4, 4, 4), (3, 4, 5, 6), (2, 3, 2, 4), (6, 6, 6, 8), (8, 8, 8, 8)]


def single(n, prec, seed, steps, every):
    # the single contexts run the ensemble's stage form (fused in FP64, the
    # two-kernel stage in FP32)
    from latticeyangmills_b200 import GluonField, _native as N

    with GluonField(n, prec) as f:
        f.set_option(N.OPT_STAGE_FORM, 0 if prec == "fp64" else 1)
        f.init_links("expiah", 0.3 + 0.02 * seed, seed)
        rows = f.flow(0.01, steps, every)
        return rows, f.download()


# the ensemble kernel is a separate compilation of the same link code, so the
# compiler may contract a few multiply-adds differently: equal to rounding
LINK_TOL = {"fp64": 1e-13, "fp32_18": 1e-5, "fp32_12": 1e-5}
OBS_RTOL = {"fp64": 1e-12, "fp32_18": 1e-6, "fp32_12": 1e-6}


@pytest.mark.parametrize("prec", ["fp64", "fp32_18", "fp32_12"])
def test_ensemble_equals_one_by_one(prec):
    from latticeyangmills_b200 import Ensemble

    steps, every = 6, 3
    with Ensemble(SIZES, prec) as ens:
        for c, n in enumerate(SIZES):
            ens.init_links(c, "expiah", 0.3 + 0.02 * c, c)
        rows = ens.flow(0.01, steps, every)
        for c, n in enumerate(SIZES):
            want_rows, want_links = single(n, prec, c, steps, every)
            assert np.abs(ens.download(c) - want_links).max() < LINK_TOL[prec]
            np.testing.assert_array_equal(rows[:, c, :2], want_rows[:, :2])
            np.testing.assert_allclose(rows[:, c, [2, 4]], want_rows[:, [2, 4]], rtol=OBS_RTOL[prec])


def test_autotune_keeps_state_and_results(oracle):
    from latticeyangmills_b200 import Ensemble

    with Ensemble(SIZES, "fp32_18") as a, Ensemble(SIZES, "fp32_18") as b:
        for c in range(len(SIZES)):
            a.init_links(c, "expiah", 0.35, 10 + c)
            b.init_links(c, "expiah", 0.35, 10 + c)
        block, grid = a.autotune()
        assert block in (128, 256, 384, 512) and grid >= 0
        assert b.autotune() == (block, grid)  # the cached choice
        assert a.tuning() == b.tuning()
        ra = a.flow(0.01, 4, 2)
        rb = b.flow(0.01, 4, 2)
        np.testing.assert_array_equal(ra, rb)
        for c in range(len(SIZES)):
            np.testing.assert_array_equal(a.download(c), b.download(c))


def test_ensemble_matches_reference_golden():
    import json

    from conftest import GOLDEN, case_field, load_case
    from latticeyangmills_b200 import Ensemble

    names = ["g4_expiah", "g3456_expiah", "g2324_expiah"]
    cases = [load_case(n) for n in names]
    with Ensemble([tuple(c["dims"]) for c in cases], "fp64") as ens:
        for i, c in enumerate(cases):
            ens.upload(i, case_field(c))
        rows = ens.flow(0.01, 5, 1)
    for i, c in enumerate(cases):
        if c["eps"] != 0.01:
            continue
        ref = np.array(c["rows"])[:6]
        np.testing.assert_allclose(rows[:, i, 2], ref[:, 2], rtol=1e-12)
        np.testing.assert_allclose(rows[:, i, 4], ref[:, 4], rtol=1e-12)


# lattices the tile kernel covers, 12^4 with x-y runs that straddle warps
TILE_SIZES = [(8, 8, 8, 8), (16, 4, 4, 6), (32, 4, 6, 5), (12, 12, 12, 12)]


@pytest.mark.parametrize("prec,threads", [("fp64", 128), ("fp64", 256), ("fp32_12", 256), ("fp32_18", 512)])
def test_tile_ensemble_equals_one_by_one(prec, threads):
    """The one-kernel stage with tiles in shared memory over every
    configuration in one launch (block runs crossing configurations) against
    each configuration on its own: FP64 link by link to 1e-13."""
    from latticeyangmills_b200 import Ensemble

    steps, every = 5, 5
    with Ensemble(TILE_SIZES, prec) as ens:
        ens.set_tuning(2, threads)
        assert ens.tuning()[:2] == (2, threads)
        for c, n in enumerate(TILE_SIZES):
            ens.init_links(c, "expiah", 0.3 + 0.02 * c, c)
        rows = ens.flow(0.01, steps, every, reunit_every=0)
        for c, n in enumerate(TILE_SIZES):
            want_rows, want_links = single(n, prec, c, steps, every)
            assert np.abs(ens.download(c) - want_links).max() < LINK_TOL[prec]
            np.testing.assert_allclose(rows[:, c, [2, 4]], want_rows[:, [2, 4]], rtol=OBS_RTOL[prec])


def test_set_tuning_refusals():
    from latticeyangmills_b200 import Ensemble, YmflowError

    with Ensemble([(2, 3, 2, 4), (8, 8, 8, 8)], "fp32_12") as ens:  # 2x3x2: fewer than 32 sites a slice
        with pytest.raises(YmflowError):
            ens.set_tuning(2, 256)
        with pytest.raises(YmflowError):
            ens.set_tuning(1, 256)
        ens.set_tuning(1)
        assert ens.tuning()[0] == 1
    with Ensemble([(8, 8, 8, 8)], "fp64") as ens:
        with pytest.raises(YmflowError):
            ens.set_tuning(4)  # no such form
        with pytest.raises(YmflowError):
            ens.set_tuning(3, 256)  # the two-kernel stage runs 128 threads


# runs of equal extents: two of 8^4, one of 3x4x5x6, three of 6^3x8, one of 8^4
RUN_SIZES = [(8, 8, 8, 8)] * 2 + [(3, 4, 5, 6)] + [(6, 6, 6, 8)] * 3 + [(8, 8, 8, 8)]


@pytest.mark.parametrize("prec", ["fp32_18", "fp32_12"])
def test_per_run_two_kernel_stage_equals_work_list_form(prec):
    """Stage form 3 (the two-kernel stage launched per run of equal extents,
    the runs as concurrent branches of the step graph) runs the same link code
    as form 1 over the work list: rows and links bit for bit, with the
    reunitarisation between steps."""
    from latticeyangmills_b200 import Ensemble

    out = {}
    for form in (1, 3):
        with Ensemble(RUN_SIZES, prec) as ens:
            ens.set_tuning(form)
            assert ens.tuning() == (form, 128, 0)
            for c in range(len(RUN_SIZES)):
                ens.init_links(c, "expiah", 0.3 + 0.02 * c, 20 + c)
            rows = ens.flow(0.02, 6, 3, reunit_every=2)
            out[form] = (rows, [ens.download(c) for c in range(len(RUN_SIZES))])
    np.testing.assert_array_equal(out[3][0], out[1][0])
    for a, b in zip(out[3][1], out[1][1]):
        np.testing.assert_array_equal(a, b)


def test_fp64_per_run_two_kernel_stage_equals_the_fused_form():
    """FP64 ensembles flow with the fused kernel by default; the per-run
    two-kernel form (stage form 3) gives the same flow to FP64 rounding, and
    the reference's golden rows to 1e-12."""
    from latticeyangmills_b200 import Ensemble

    out = {}
    for form in (0, 3):
        with Ensemble(RUN_SIZES, "fp64") as ens:
            assert ens.tuning()[0] == 0
            ens.set_tuning(form)
            assert ens.tuning()[0] == form
            for c in range(len(RUN_SIZES)):
                ens.init_links(c, "expiah", 0.3 + 0.02 * c, 20 + c)
            rows = ens.flow(0.02, 6, 3)
            out[form] = (rows, [ens.download(c) for c in range(len(RUN_SIZES))])
    np.testing.assert_array_equal(out[3][0][:, :, :2], out[0][0][:, :, :2])
    np.testing.assert_allclose(out[3][0][:, :, [2, 4]], out[0][0][:, :, [2, 4]], rtol=1e-12)
    for a, b in zip(out[3][1], out[0][1]):
        assert np.abs(a - b).max() < 1e-13
