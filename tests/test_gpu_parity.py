"""FP64 GPU path against the reference: parity to 1e-12 relative.

Golden tables come from the reference's own code (tests/golden); link-level
and larger checks use the CPU oracle, itself pinned bit-for-bit to those
tables (test_oracle_golden.py)."""
import numpy as np
import pytest

from conftest import GOLDEN, case_field, load_case, topc_tolerance

pytestmark = pytest.mark.gpu

REL = 1e-12  # relative tolerance on plaq, energy and t^2<E> (FP64 path)
CASES = ["g4_expiah", "g3456_expiah", "g2324_expiah", "g8_metropolis", "g8_haar", "g16x32_expiah", "g16x32_full"]


def run_case(name, precision="fp64"):
    from latticeyangmills_b200 import GluonField

    case = load_case(name)
    U = case_field(case)
    n = tuple(case["dims"])
    with GluonField(n, precision) as f:
        f.upload(U)
        rows = f.flow(case["eps"], case["nsteps"], case["every"])
    return case, rows


def assert_rows_match(case, rows, rel=REL):
    ref = np.array(case["rows"])
    assert rows.shape[0] == ref.shape[0]
    np.testing.assert_array_equal(rows[:, 0], ref[:, 0])  # steps
    np.testing.assert_array_equal(rows[:, 1], ref[:, 1])  # t, accumulated as t += eps
    np.testing.assert_allclose(rows[:, 2], ref[:, 2], rtol=rel, atol=0)  # plaq
    np.testing.assert_allclose(rows[:, 4], ref[:, 4], rtol=rel, atol=0)  # energy
    for q, qr, e in zip(rows[:, 3], ref[:, 3], ref[:, 4]):
        assert abs(q - qr) <= topc_tolerance(e, rel), (q, qr)
    V = int(np.prod(case["dims"]))
    t2e_ref = -ref[:, 1] ** 2 * ref[:, 4] / (64.0 * V)
    np.testing.assert_allclose(rows[:, 5], t2e_ref, rtol=rel, atol=0)


@pytest.mark.parametrize("name", CASES)
def test_fp64_flow_matches_reference(name):
    case, rows = run_case(name)
    assert_rows_match(case, rows)


def test_links_match_oracle_after_flow(oracle):
    from latticeyangmills_b200 import GluonField

    case = load_case("g3456_expiah")
    U = case_field(case)
    n = tuple(case["dims"])
    with GluonField(n, "fp64") as f:
        f.upload(U)
        np.testing.assert_array_equal(f.download(), U)  # upload/download round trip is exact
        f.flow(case["eps"], 5, 0)
        got = f.download()
    want = U.copy()
    oracle.flow(want, n, case["eps"], 5, 0)
    assert np.abs(got - want).max() < 1e-13


def test_derivative_matches_reference():
    from latticeyangmills_b200 import GluonField

    case = load_case("g4_expiah")
    U = case_field(case)
    Z = np.load(GOLDEN / "g4_expiah_deriv.npy")
    with GluonField(tuple(case["dims"]), "fp64") as f:
        f.upload(U)
        for mu in range(4):
            z = f.derivative(mu)
            want = Z[..., mu, :].reshape(-1, 18)
            assert np.abs(z - want).max() <= 1e-13 * np.abs(want).max()


def test_exp_matches_reference_and_fixes_its_nans():
    from latticeyangmills_b200 import su3_exp

    d = np.load(GOLDEN / "exp_cases.npz")
    q, ref = d["q"], d["r"]
    r = su3_exp(q)
    ok = ~np.isnan(ref).any(axis=1)
    np.testing.assert_allclose(r[ok], ref[ok], rtol=0, atol=1e-13)
    # where the reference returns NaN (Q = 0, degenerate spectra) the GPU returns e^{iQ}
    assert np.isfinite(r).all()
    h = q.reshape(-1, 3, 3, 2)
    h = h[..., 0] + 1j * h[..., 1]
    w, v = np.linalg.eigh(h[~ok])
    want = np.einsum("nij,nj,nkj->nik", v, np.exp(1j * w), np.conj(v))
    got = r[~ok].reshape(-1, 3, 3, 2)
    np.testing.assert_allclose(got[..., 0] + 1j * got[..., 1], want, atol=1e-12)


def test_cold_field_stays_cold():
    # The reference returns NaN here (tests/golden/g4_cold.json); e^{i0} = 1 exactly on the GPU.
    from latticeyangmills_b200 import GluonField

    with GluonField((4, 4, 4, 4), "fp64") as f:
        f.init_links("cold")
        rows = f.flow(0.01, 3, 1)
    assert (rows[:, 2] == 1.0).all() and (rows[:, 3] == 0.0).all() and (rows[:, 4] == 0.0).all()


def test_graph_and_block_size_do_not_change_results():
    from latticeyangmills_b200 import GluonField
    from latticeyangmills_b200 import _native as N

    case = load_case("g3456_expiah")
    U = case_field(case)
    outs = []
    for graph, block, obs_block in [(1, 128, 192), (0, 128, 192)]:
        with GluonField(tuple(case["dims"]), "fp64") as f:
            f.set_option(N.OPT_GRAPH, graph)
            f.set_option(N.OPT_BLOCK, block)
            f.set_option(N.OPT_OBS_BLOCK, obs_block)
            assert f.get_option(N.OPT_OBS_BLOCK) == 192
            f.upload(U)
            rows = f.flow(case["eps"], 4, 0)
            outs.append((f.download(), rows))
    for links, rows in outs[1:]:
        np.testing.assert_array_equal(links, outs[0][0])
        # observables fold block partials in a different grouping: equal to rounding
        np.testing.assert_allclose(rows[:, 2:], outs[0][1][:, 2:], rtol=1e-13)


def test_device_generator_matches_fixture_generator(oracle):
    from latticeyangmills_b200 import GluonField

    n = (4, 4, 6, 8)
    want = oracle.gen_expiah(n, 0.35, 77, 3)
    oracle.gen_haar_mix(want, n, 0.05, 77, 3)
    with GluonField(n, "fp64") as f:
        f.init_links("expiah", 0.35, 77, 3, haar_frac=0.05)
        got = f.download()
    assert np.abs(got - want).max() < 1e-13


def random_gauge(oracle, n, seed):
    g = oracle.gen_cold((n[0], n[1], n[2], n[3]))
    oracle.gen_haar_mix(g, n, 1.0, seed)
    m = g[..., 0, :].reshape(n[3], n[2], n[1], n[0], 3, 3, 2)
    return m[..., 0] + 1j * m[..., 1]


def test_observables_gauge_invariant(oracle):
    from latticeyangmills_b200 import GluonField

    case = load_case("g3456_expiah")
    U = case_field(case)
    n = tuple(case["dims"])
    om = random_gauge(oracle, n, 5)
    u = U.reshape(n[3], n[2], n[1], n[0], 4, 3, 3, 2)
    uc = u[..., 0] + 1j * u[..., 1]
    ut = np.empty_like(uc)
    for mu in range(4):
        ax = 3 - mu  # array axis of direction mu (t, z, y, x order)
        om_fwd = np.roll(om, -1, axis=ax)  # Omega(x + mu)
        ut[..., mu, :, :] = om @ uc[..., mu, :, :] @ np.conj(np.swapaxes(om_fwd, -1, -2))
    Ut = np.stack([ut.real, ut.imag], -1).reshape(U.shape)
    with GluonField(n, "fp64") as f:
        f.upload(U)
        a = f.flow(case["eps"], 3, 1)
        f.upload(Ut)
        b = f.flow(case["eps"], 3, 1)
    np.testing.assert_allclose(b[:, 2], a[:, 2], rtol=1e-12)
    np.testing.assert_allclose(b[:, 4], a[:, 4], rtol=1e-12)
    for q, qr, e in zip(b[:, 3], a[:, 3], a[:, 4]):
        assert abs(q - qr) <= topc_tolerance(e, 1e-12) * 10


def test_wilsonflow_app_mirror_writes_reference_rows(tmp_path):
    from latticeyangmills_b200 import WilsonFlow, read_conf, write_conf

    case = load_case("g4_expiah")
    U = case_field(case)
    indir = tmp_path / "in"
    indir.mkdir()
    write_conf(indir / "conf0000.bin", U)
    app = WilsonFlow(tauFinal=0.05, epsilon=0.01)  # int(0.05/0.01) = 5 rows, 4 steps
    app.createLattice(tuple(case["dims"]))
    (path,) = app.flowConfigurations(indir, tmp_path / "out")
    lines = path.read_text().splitlines()
    assert lines[0] == "Flow Time\tPlaq.\tTopc.\tEnerg.\t"
    assert len(lines) == 1 + 5
    ref = np.array(case["rows"])[:5]
    for line, r in zip(lines[1:], ref):
        assert line == "".join("%f\t" % v for v in (r[1], r[2], r[3], r[4]))
    app.field.close()


@pytest.mark.parametrize("n", [(1, 2, 3, 4), (2, 2, 2, 2), (1, 1, 1, 6), (5, 1, 2, 3)])
def test_degenerate_extents_match_oracle(oracle, n):
    """Extents of 1 (a link is its own neighbour) and 2 (both neighbours are
    one site): the periodic indexing against the oracle's."""
    from latticeyangmills_b200 import GluonField

    U = oracle.gen_expiah(n, 0.35, 7, 0)
    with GluonField(n, "fp64") as f:
        f.upload(U)
        rows = f.flow(0.02, 4, 2)
        got = f.download()
    want = U.copy()
    ref = oracle.flow(want, n, 0.02, 4, 2)
    assert np.abs(got - want).max() < 1e-13
    np.testing.assert_allclose(rows[:, 2], ref[:, 2], rtol=REL, atol=1e-15)  # plaq
    np.testing.assert_allclose(rows[:, 4], ref[:, 4], rtol=REL, atol=1e-12)  # energy
    assert np.abs(rows[:, 3] - ref[:, 3]).max() < 1e-12  # topc


def test_full_size_steps_match_oracle(oracle):
    """The headline workload itself: 32^4, two RK3 steps, every link and the
    observables of both rows against the oracle (about 7 s of oracle time)."""
    from latticeyangmills_b200 import GluonField

    n = (32, 32, 32, 32)
    U = oracle.gen_expiah(n, 0.35, 20260, 0)
    want = U.copy()
    ref = oracle.flow(want, n, 0.01, 2, 2)
    with GluonField(n, "fp64") as f:
        f.upload(U)
        rows = f.flow(0.01, 2, 2)
        got = f.download()
    assert np.abs(got - want).max() < 1e-13
    np.testing.assert_allclose(rows[:, 2], ref[:, 2], rtol=REL, atol=0)
    np.testing.assert_allclose(rows[:, 4], ref[:, 4], rtol=REL, atol=0)
    assert np.abs(rows[:, 3] - ref[:, 3]).max() <= topc_tolerance(ref[:, 4].min(), REL)
    with GluonField(n, "fp32_18") as f:
        f.upload(U)
        rows32 = f.flow(0.01, 2, 2)
        got32 = f.download()
    assert np.abs(got32 - want).max() < 5e-6
    np.testing.assert_allclose(rows32[:, 2], ref[:, 2], rtol=1e-6)
    np.testing.assert_allclose(rows32[:, 4], ref[:, 4], rtol=1e-6)
