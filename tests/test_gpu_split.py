"""The two-kernel RK3 stage (YMFLOW_OPT_STAGE_FORM 1): a stored plaquette field,
then each link's force as its upper plaquettes plus its conjugated lower ones.
In FP64 it is the reference's flow to 1e-12 against the golden tables; in FP32
(the mixed forms' default) it meets the accuracy target against the FP64 flow."""
import numpy as np
import pytest

from conftest import case_field, load_case

pytestmark = pytest.mark.gpu


def flow_form(n, precision, form, steps=6, every=2, eps=0.02, seed=7, reunit=0, a=0.4):
    from latticeyangmills_b200 import GluonField, _native as N

    with GluonField(n, precision) as f:
        f.set_option(N.OPT_STAGE_FORM, form)
        f.init_links("expiah", a, seed)
        rows = f.flow(eps, steps, every, reunit_every=reunit)
        return rows, f.download()


@pytest.mark.parametrize("name", ["g4_expiah", "g3456_expiah", "g2324_expiah", "g8_haar", "g16x32_expiah"])
def test_fp64_split_stage_matches_reference(name):
    """The plaquette-field form of the force against the reference's own
    numbers (staples, puregauge.cpp:36-79) to the parity tolerance."""
    from test_gpu_parity import assert_rows_match

    from latticeyangmills_b200 import GluonField, _native as N

    case = load_case(name)
    with GluonField(tuple(case["dims"]), "fp64") as f:
        f.set_option(N.OPT_STAGE_FORM, 1)
        f.upload(case_field(case))
        rows = f.flow(case["eps"], case["nsteps"], case["every"])
    assert_rows_match(case, rows)


@pytest.mark.parametrize("n", [(4, 4, 4, 4), (3, 4, 5, 6), (2, 3, 2, 4), (8, 8, 8, 8)])
def test_fp64_split_equals_fused_to_rounding(n):
    rows0, u0 = flow_form(n, "fp64", 0)
    rows1, u1 = flow_form(n, "fp64", 1)
    assert np.abs(u1 - u0).max() < 1e-13
    np.testing.assert_array_equal(rows1[:, :2], rows0[:, :2])
    np.testing.assert_allclose(rows1[:, [2, 4, 5]], rows0[:, [2, 4, 5]], rtol=1e-12)
    assert np.abs(rows1[:, 3] - rows0[:, 3]).max() < 1e-12


@pytest.mark.parametrize("precision", ["fp32_18", "fp32_12"])
def test_fp32_split_meets_the_accuracy_target_at_t4(precision):
    """The acceptance configuration: 32^4, U = e^{iaH} (a = 0.35), eps 0.01 to
    t = 4 with reunitarisation every 10 steps.  |d(t^2 E)| / t^2 E < 1e-6 and
    |dQ| < 1e-4 against the FP64 flow at t = 4; the earlier rows (smaller t^2 E)
    within 1e-5."""
    n = (32, 32, 32, 32)
    r64, _ = flow_form(n, "fp64", 0, steps=400, every=100, eps=0.01, seed=1, a=0.35)
    r32, _ = flow_form(n, precision, 1, steps=400, every=100, eps=0.01, seed=1, a=0.35, reunit=10)
    rel = np.abs(r32[1:, 5] - r64[1:, 5]) / np.abs(r64[1:, 5])
    dq = np.abs(r32[:, 3] - r64[:, 3]).max()
    print(precision, "t", r32[1:, 1], "rel err t2E", rel, "|dQ|", dq)
    assert abs(r32[-1, 1] - 4.0) < 1e-9
    assert rel[-1] < 1e-6
    assert rel.max() < 1e-5
    assert dq < 1e-4


def test_stage_form_defaults_and_refusals():
    from latticeyangmills_b200 import GluonField, YmflowError, _native as N

    # the two-kernel form, except FP32 lattices of at most 8192 sites (launch-bound: the fused kernel)
    for n, prec, want in (((4, 4, 4, 4), "fp64", 1), ((4, 4, 4, 4), "fp32_18", 0), ((8, 8, 8, 8), "fp32_12", 0),
                          ((8, 8, 8, 18), "fp32_12", 1), ((8, 8, 8, 16), "fp32_18", 0)):
        with GluonField(n, prec) as f:
            assert f.get_option(N.OPT_STAGE_FORM) == want
            with pytest.raises(YmflowError):
                f.set_option(N.OPT_STAGE_FORM, 2)
            f.set_option(N.OPT_STAGE_FORM, 1)  # the plaquette field is allocated on demand
            assert f.get_option(N.OPT_STAGE_FORM) == 1
    with GluonField.slab((32, 8, 8, 10), 0, 5, "fp32_18") as s:  # 32 x 8 x 8 x 7 local sites
        assert s.get_option(N.OPT_STAGE_FORM) == 1
        s.set_option(N.OPT_STAGE_FORM, 0)
        assert s.get_option(N.OPT_STAGE_FORM) == 0


def test_slab_group_needs_one_stage_form():
    from latticeyangmills_b200 import GluonField, YmflowError, _native as N, slab_group_flow

    a = GluonField.slab((8, 4, 4, 10), 0, 5, "fp32_12")
    b = GluonField.slab((8, 4, 4, 10), 5, 5, "fp32_12")
    try:
        for sl in (a, b):
            sl.init_links("expiah", 0.4, 3)
        a.set_option(N.OPT_STAGE_FORM, 1)
        b.set_option(N.OPT_STAGE_FORM, 0)
        with pytest.raises(YmflowError):
            slab_group_flow([a, b], 0.02, 2, 1)
        b.set_option(N.OPT_STAGE_FORM, 1)
        rows = slab_group_flow([a, b], 0.02, 2, 1)
        assert rows.shape[0] == 3
    finally:
        a.close()
        b.close()


@pytest.mark.parametrize("form", [0, 1])
def test_fp32_slabs_in_both_forms_match_the_whole_lattice(form):
    """Three FP32 slabs flowing together (the two-kernel stage stores its
    boundary links into the neighbours' halos as the fused one does) against
    the whole lattice in the same form: equal to FP32 rounding."""
    from latticeyangmills_b200 import GluonField, _native as N, slab_group_flow

    n = (8, 4, 4, 10)
    with GluonField(n, "fp32_12") as f:
        f.set_option(N.OPT_STAGE_FORM, form)
        f.init_links("expiah", 0.4, 5)
        want = f.flow(0.02, 6, 3, reunit_every=3)
        want_links = f.download()
    slabs = [GluonField.slab(n, t0, nt, "fp32_12") for t0, nt in ((0, 4), (4, 3), (7, 3))]
    try:
        for sl in slabs:
            sl.set_option(N.OPT_STAGE_FORM, form)
            sl.init_links("expiah", 0.4, 5)
        got = slab_group_flow(slabs, 0.02, 6, 3, reunit_every=3)
        links = np.concatenate([sl.download() for sl in slabs])
    finally:
        for sl in slabs:
            sl.close()
    assert np.abs(links - want_links).max() < 1e-5
    np.testing.assert_array_equal(got[:, :2], want[:, :2])
    np.testing.assert_allclose(got[:, [2, 4, 5]], want[:, [2, 4, 5]], rtol=1e-6)


def test_switching_forms_mid_flow_continues_the_flow():
    """Switching the stage form between calls (the captured step graphs are
    rebuilt) continues from the current links."""
    from latticeyangmills_b200 import GluonField, _native as N

    n = (6, 4, 4, 8)
    with GluonField(n, "fp64") as f:
        f.init_links("expiah", 0.4, 9)
        f.flow(0.02, 3, 0)
        f.set_option(N.OPT_STAGE_FORM, 1)
        f.flow(0.02, 3, 0)
        f.set_option(N.OPT_STAGE_FORM, 0)
        rows = f.flow(0.02, 2, 0)
        mixed = f.download()
    _, plain = flow_form(n, "fp64", 0, steps=8, every=0, seed=9, eps=0.02)
    assert rows[-1, 0] == 8
    assert np.abs(mixed - plain).max() < 1e-13


def test_kernel_timing_splits_by_kernel():
    from latticeyangmills_b200 import GluonField, _native as N

    with GluonField((8, 8, 8, 8), "fp32_12") as f:
        f.init_links("expiah", 0.35, 1)
        el, field, stage = f.time_kernels(0.01, 4)
        assert el > 0 and field > 0 and stage > 0 and field + stage <= el * 1.05
        f.set_option(N.OPT_STAGE_FORM, 0)
        el, field, stage = f.time_kernels(0.01, 4)
        # two back-to-back events (no kernel between them): a few microseconds per stage
        assert field / (3 * 4) < 0.01
        _, km = f.time_steps(0.01, 4, kernels=True)
        assert km > 0


def test_fp64_context_without_room_for_the_plaquette_field_uses_the_fused_form():
    """An FP64 context whose plaquette field (384 B per site) does not fit
    beside its links starts in the fused form instead of failing, and flows as
    a context with room does (to 1e-12)."""
    import torch

    from latticeyangmills_b200 import GluonField, YmflowError, _native as N

    n = (32, 32, 32, 32)
    sites = 32**4
    need = 2 * 4 * sites * 144 + 4 * sites * 64  # both link buffers and the generator
    field = 6 * sites * 64                        # the plaquette field

    def run(f):
        f.init_links("expiah", 0.35, 5)
        return f.flow(0.02, 2, 1)

    free, _ = torch.cuda.mem_get_info()
    filler = torch.empty(int(free - need - field // 2), dtype=torch.uint8, device="cuda")
    try:
        with GluonField(n, "fp64") as f:
            assert f.get_option(N.OPT_STAGE_FORM) == 0
            with pytest.raises(YmflowError):
                f.set_option(N.OPT_STAGE_FORM, 1)  # no room for the field either
            got = run(f)
    finally:
        del filler
        torch.cuda.empty_cache()
    with GluonField(n, "fp64") as f:
        assert f.get_option(N.OPT_STAGE_FORM) == 1
        want = run(f)
    np.testing.assert_array_equal(got[:, :2], want[:, :2])
    np.testing.assert_allclose(got[:, [2, 4]], want[:, [2, 4]], rtol=1e-12)
