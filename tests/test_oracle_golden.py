"""Pins the CPU oracle (oracle/ymoracle.c) to the reference's own numbers.

The golden tables were printed by the reference's code itself
(oracle/_ref/ref_flow, regenerate with tests/golden/make_golden.py); the
oracle must reproduce them bit for bit, which is what lets it check the GPU
path at sizes and schedules the goldens do not cover."""
import json

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, case_field, load_case

BITWISE_CASES = ["g4_expiah", "g3456_expiah", "g2324_expiah", "g8_metropolis", "g8_haar"]


@pytest.mark.parametrize("name", BITWISE_CASES)
def test_oracle_flow_matches_reference_bitwise(oracle, name):
    case = load_case(name)
    U = case_field(case)
    rows = oracle.flow(U, tuple(case["dims"]), case["eps"], case["nsteps"], case["every"])
    ref = np.array(case["rows"])
    assert rows.shape == ref.shape
    np.testing.assert_array_equal(rows, ref)


def test_oracle_large_case_matches_reference(oracle):
    case = load_case("g16x32_expiah")
    U = case_field(case)
    rows = oracle.flow(U, tuple(case["dims"]), case["eps"], case["nsteps"], case["every"])
    np.testing.assert_array_equal(rows, np.array(case["rows"]))


def test_reference_cold_field_is_nan_after_one_step():
    # exp(0) divides 0 by 0 in the reference (src/Math/su3.cpp:111-112): a cold
    # configuration flows to NaN.  The GPU path returns the identity instead.
    case = load_case("g4_cold")
    rows = np.array(case["rows"])
    assert rows[0, 2] == 1.0 and rows[0, 3] == 0.0 and rows[0, 4] == 0.0
    assert np.isnan(rows[1:, 2:]).all()


def test_oracle_exp_matches_reference(oracle):
    d = np.load(GOLDEN / "exp_cases.npz")
    r = oracle.su3_exp(d["q"])
    ref = d["r"]
    nan = np.isnan(ref).any(axis=1)
    assert nan.sum() >= 1  # Q = 0 (and exactly degenerate spectra) give NaN in the reference
    np.testing.assert_array_equal(r[~nan], ref[~nan])
    assert np.isnan(r[nan]).any(axis=1).all()


def test_oracle_derivative_matches_reference(oracle):
    case = load_case("g4_expiah")
    U = case_field(case)
    Z = np.load(GOLDEN / "g4_expiah_deriv.npy")
    n = tuple(case["dims"])
    for mu in range(4):
        z = oracle.derivative(U, n, mu)
        np.testing.assert_array_equal(z, Z[..., mu, :].reshape(-1, 18))


def test_exp_is_unitary_and_matches_eigendecomposition(oracle):
    rng = np.random.default_rng(5)
    m = rng.normal(size=(64, 3, 3)) + 1j * rng.normal(size=(64, 3, 3))
    h = (m + np.conj(np.swapaxes(m, 1, 2))) / 2
    h -= np.trace(h, axis1=1, axis2=2)[:, None, None] / 3 * np.eye(3)
    h *= 0.3
    q = np.stack([h.real, h.imag], -1).reshape(64, 18)
    r = oracle.su3_exp(q).reshape(64, 3, 3, 2)
    e = r[..., 0] + 1j * r[..., 1]
    w, v = np.linalg.eigh(h)
    want = np.einsum("nij,nj,nkj->nik", v, np.exp(1j * w), np.conj(v))
    np.testing.assert_allclose(e, want, atol=1e-13)
    np.testing.assert_allclose(np.linalg.det(e), 1.0, atol=1e-13)


def test_philox_known_answers(oracle):
    # Known-answer vectors of Philox4x32-10 (Salmon et al., Random123 kat_vectors)
    assert oracle.philox([0, 0, 0, 0], [0, 0]) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    f = 0xFFFFFFFF
    assert oracle.philox([f, f, f, f], [f, f]) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert oracle.philox([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0]) == [
        0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


def test_generated_fields_are_su3(oracle):
    n = (4, 4, 4, 2)
    U = oracle.gen_expiah(n, 0.35, 9)
    assert max(oracle.unitarity(U)) < 1e-13
    oracle.gen_haar_mix(U, n, 0.5, 9)
    assert max(oracle.unitarity(U)) < 1e-13
    cold = oracle.gen_cold(n)
    assert oracle.superobs(cold, n) == (1.0, 0.0, 0.0)


def test_metropolis_fixture_is_thermalised():
    case = load_case("g8_metropolis")
    g = case["generator"]
    assert g["sweeps"] == 200 and g["beta"] == 6.0
    # plaquette of the committed beta = 6.0 configuration near its equilibrium value
    assert 0.55 < case["rows"][0][2] < 0.62


def test_goldens_record_reference_schedule():
    for name in BITWISE_CASES + ["g16x32_expiah", "g4_cold"]:
        case = load_case(name)
        rows = np.array(case["rows"])
        steps = rows[:, 0].astype(int)
        assert steps[0] == 0 and steps[-1] == case["nsteps"]
        # t accumulated by repeated addition of eps (src/Apps/wilsonflow.cpp:126)
        t = 0.0
        ts = [0.0]
        for s in range(1, case["nsteps"] + 1):
            t += case["eps"]
            if s % case["every"] == 0 or s == case["nsteps"]:
                ts.append(t)
        np.testing.assert_array_equal(rows[:, 1], np.array(ts))


def test_checkerboard_chain_properties(oracle):
    """The device generator's chain on the CPU: beta = 0 accepts everything,
    numbered sweeps continue a chain, and beta = 6 moves a cold field towards
    the equilibrium plaquette while the links stay unitary."""
    n = (4, 4, 4, 4)
    V = oracle.volume(n)
    U = oracle.gen_cold(n)
    assert oracle.gen_metropolis_cb(U, n, 0.0, 0.24, 1, 3, 5) == 3 * 4 * V
    a = oracle.gen_cold(n)
    oracle.gen_metropolis_cb(a, n, 6.0, 0.24, 3, 4, 9)
    b = oracle.gen_cold(n)
    oracle.gen_metropolis_cb(b, n, 6.0, 0.24, 1, 4, 9)
    oracle.gen_metropolis_cb(b, n, 6.0, 0.24, 2, 4, 9, sweep0=1)
    assert np.array_equal(a, b)
    c = oracle.gen_cold(n)
    acc = oracle.gen_metropolis_cb(c, n, 6.0, 0.24, 40, 10, 3)
    plaq = oracle.superobs(c, n)[0]
    assert 0.08 < acc / (40 * 10 * 4 * V) < 0.2
    assert 0.55 < plaq < 0.7
    assert max(oracle.unitarity(c)) < 1e-12


def test_oracle_clean_under_sanitizers():
    """Every oracle entry point on odd and degenerate lattices under
    AddressSanitizer and UndefinedBehaviorSanitizer (oracle/sanitize_driver.c)."""
    import shutil
    import subprocess

    if shutil.which("gcc") is None:
        pytest.skip("no gcc")
    res = subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "sanitize"], capture_output=True, text=True,
                         timeout=600)
    if res.returncode != 0 and "cannot find" in res.stderr and "asan" in res.stderr:
        pytest.skip("no sanitizer runtime")
    assert res.returncode == 0, res.stdout[-2000:] + res.stderr[-2000:]
    assert "sanitize ok" in res.stdout
