"""The one-kernel RK3 stage with a tile's plaquette field in shared memory
(YMFLOW_OPT_STAGE_FORM 2, csrc/flow_tile.cu).  In FP64 it is the reference's
flow to 1e-12 against the golden tables; at every tiling (faces recomputed or
wrapped inside the tile, runs of units streaming along t across columns) it
equals the other forms to rounding; in FP32 it meets the accuracy target
against the FP64 flow."""
import numpy as np
import pytest

from conftest import case_field, load_case

pytestmark = pytest.mark.gpu


def flow_with(n, precision, form=None, tile=None, steps=6, every=2, eps=0.02, seed=7, reunit=0, a=0.4):
    from latticeyangmills_b200 import GluonField, _native as N

    with GluonField(n, precision) as f:
        if tile is not None:
            f.set_tile(*tile)
        if form is not None:
            f.set_option(N.OPT_STAGE_FORM, form)
        f.init_links("expiah", a, seed)
        rows = f.flow(eps, steps, every, reunit_every=reunit)
        return rows, f.download()


@pytest.mark.parametrize("name,tile", [("g8_haar", (4, 2)), ("g8_haar", (8, 4)), ("g8_haar", (4, 8)),
                                       ("g16x32_expiah", (2, 2)), ("g16x32_expiah", (4, 4)),
                                       ("g16x32_expiah", (16, 1)), ("g16x32_full", (4, 2))])
def test_fp64_tile_stage_matches_reference(name, tile):
    """The reference's own flow tables (puregauge.cpp:36-79 through
    wilsonflow.cpp:141-172) to the parity tolerance, with the tile kernel."""
    from test_gpu_parity import assert_rows_match

    from latticeyangmills_b200 import GluonField

    case = load_case(name)
    with GluonField(tuple(case["dims"]), "fp64") as f:
        f.set_tile(*tile)
        f.upload(case_field(case))
        rows = f.flow(case["eps"], case["nsteps"], case["every"])
    assert_rows_match(case, rows)


# (lattice, tile): faces in y and z, a face in one direction only, tiles that
# span y or z (periodic neighbour inside the tile), extents 1 and 3, and
# lattices with more units than resident blocks (runs cross tile columns).
SHAPES = [
    ((32, 4, 6, 5), (2, 3)), ((32, 4, 6, 5), (4, 1)), ((32, 4, 6, 5), (1, 6)), ((32, 4, 6, 5), (4, 2)),
    ((32, 1, 3, 4), (1, 3)), ((32, 2, 2, 1), (2, 2)), ((16, 4, 4, 6), (2, 4)), ((8, 8, 4, 3), (4, 2)),
    ((64, 4, 4, 3), (2, 2)), ((32, 16, 16, 12), (2, 4)), ((32, 16, 16, 12), (2, 2)),
    # one or two links per thread, the 64-register kernel
    ((32, 4, 6, 5), (2, 3, 1, 1)), ((32, 4, 6, 5), (2, 3, 2, 1)), ((32, 16, 16, 12), (2, 2, 2, 1)),
    ((32, 16, 16, 12), (4, 2, 2, 0)), ((16, 4, 4, 6), (2, 4, 1, 1)), ((32, 16, 16, 12), (2, 2, 4, 1)),
]


@pytest.mark.parametrize("n,tile", SHAPES)
def test_fp64_tile_equals_fused_link_by_link(n, tile):
    rows0, u0 = flow_with(n, "fp64", form=0)
    rows2, u2 = flow_with(n, "fp64", form=2, tile=tile)
    assert np.abs(u2 - u0).max() < 1e-13
    np.testing.assert_array_equal(rows2[:, :2], rows0[:, :2])
    np.testing.assert_allclose(rows2[:, [2, 4, 5]], rows0[:, [2, 4, 5]], rtol=1e-12)
    assert np.abs(rows2[:, 3] - rows0[:, 3]).max() < 1e-12


@pytest.mark.parametrize("precision", ["fp32_18", "fp32_12"])
@pytest.mark.parametrize("n,tile", [((32, 4, 6, 5), (2, 3)), ((32, 16, 16, 12), (4, 4)), ((16, 4, 4, 6), (2, 4)),
                                    ((32, 16, 16, 12), (4, 4, 2, 1)), ((32, 16, 16, 12), (4, 2, 1, 1))])
def test_fp32_tile_equals_two_kernel_form(precision, n, tile):
    """Same plaquette generators, same conjugations, same accumulation order as
    the two-kernel form: equal to FP32 rounding."""
    rows1, u1 = flow_with(n, precision, form=1, reunit=3)
    rows2, u2 = flow_with(n, precision, form=2, tile=tile, reunit=3)
    assert np.abs(u2 - u1).max() < 2e-6
    np.testing.assert_allclose(rows2[:, [2, 4, 5]], rows1[:, [2, 4, 5]], rtol=2e-6)


@pytest.mark.parametrize("precision", ["fp32_18", "fp32_12"])
def test_fp32_tile_meets_the_accuracy_target_at_t4(precision):
    """32^4, U = e^{iaH} (a = 0.35), eps 0.01 to t = 4, reunitarisation every 10
    steps, with the tile kernel: |d(t^2 E)| / t^2 E < 1e-6 and
    |dQ| < 1e-4 against the FP64 flow at t = 4; earlier rows within 1e-5."""
    from latticeyangmills_b200 import GluonField, _native as N

    n = (32, 32, 32, 32)
    r64, _ = flow_with(n, "fp64", steps=400, every=100, eps=0.01, seed=1, a=0.35)
    r32, _ = flow_with(n, precision, tile=(4, 4, 2, 1), steps=400, every=100, eps=0.01, seed=1, a=0.35,
                       reunit=10)
    rel = np.abs(r32[1:, 5] - r64[1:, 5]) / np.abs(r64[1:, 5])
    dq = np.abs(r32[:, 3] - r64[:, 3]).max()
    print(precision, "t", r32[1:, 1], "rel err t2E", rel, "|dQ|", dq)
    assert abs(r32[-1, 1] - 4.0) < 1e-9
    assert rel[-1] < 1e-6
    assert rel.max() < 1e-5
    assert dq < 1e-4


def test_tile_defaults_and_refusals():
    from latticeyangmills_b200 import GluonField, YmflowError, _native as N, tile_option

    with GluonField((32, 32, 32, 32), "fp32_12") as f:
        assert f.get_option(N.OPT_STAGE_FORM) == 1
        assert f.get_option(N.OPT_TILE) == tile_option(4, 4, 2, 1)  # the prepared default tiling
        f.set_option(N.OPT_STAGE_FORM, 2)
    with GluonField((32, 32, 32, 32), "fp64") as f:
        assert f.get_option(N.OPT_STAGE_FORM) == 1
        f.set_tile(2, 2)
        assert f.get_option(N.OPT_STAGE_FORM) == 2
        assert f.get_option(N.OPT_TILE) == tile_option(2, 2)
    with GluonField((16, 16, 16, 32), "fp32_18") as f:
        # 3 does not divide 16; Lx ty < 32; zero; 4096 sites; 3 links a thread; 1024 threads on the 128-register kernel
        for bad in ((3, 2), (1, 4), (0, 1), (16, 16), (4, 4, 3, 0), (8, 4, 1, 0)):
            with pytest.raises(YmflowError):
                f.set_option(N.OPT_TILE, tile_option(*bad))
    with GluonField((12, 12, 12, 12), "fp32_12") as f:  # 12-site x lines fill no whole warp
        assert f.get_option(N.OPT_STAGE_FORM) == 1
        with pytest.raises(YmflowError):
            f.set_option(N.OPT_STAGE_FORM, 2)
    with GluonField.slab((32, 8, 8, 10), 0, 5, "fp32_12") as s:
        assert s.get_option(N.OPT_STAGE_FORM) == 1
        with pytest.raises(YmflowError):
            s.set_option(N.OPT_STAGE_FORM, 2)


def test_autotune_picks_a_form_and_keeps_the_field():
    from latticeyangmills_b200 import GluonField, _native as N

    n = (32, 16, 16, 16)
    with GluonField(n, "fp32_12") as f:
        f.init_links("expiah", 0.35, 4)
        before = f.download()
        form, ty, tz = f.autotune(0.01)
        assert form in (0, 1, 2)
        assert f.get_option(N.OPT_STAGE_FORM) == form
        if form == 2:
            assert (f.get_option(N.OPT_TILE) & 0xFFFFFFFF) == (ty << 16) | tz
        np.testing.assert_array_equal(f.download(), before)
        rows = f.flow(0.01, 4, 2, reunit_every=2)
    want, _ = flow_with(n, "fp32_12", form=1, steps=4, every=2, eps=0.01, seed=4, a=0.35, reunit=2)
    np.testing.assert_allclose(rows[:, [2, 4, 5]], want[:, [2, 4, 5]], rtol=1e-5)
    with GluonField(n, "fp32_12") as g:  # cached per extents and precision
        g.init_links("expiah", 0.35, 4)
        assert g.autotune(0.01) == (form, ty, tz)


def test_timed_steps_carry_the_reunitarisation():
    from latticeyangmills_b200 import GluonField, _native as N

    with GluonField((32, 16, 16, 16), "fp32_12") as f:
        f.init_links("expiah", 0.35, 1)
        f.time_steps(0.01, 3)
        plain, _ = f.time_steps(0.01, 20)
        f.set_option(N.OPT_TIMED_REUNIT, 10)
        assert f.get_option(N.OPT_TIMED_REUNIT) == 10
        with_reunit, _ = f.time_steps(0.01, 20)
        el, field, stage = f.time_kernels(0.01, 20)
    assert with_reunit > 0 and plain > 0 and el > 0 and stage > 0
    # the instrumented pass: the stage kernels inside the step time, which also holds two reunitarisations
    assert field + stage < el
