"""Device Metropolis generator (ymflow_generate_metropolis) against the
oracle's checkerboard chain with the same counter-based random numbers, and
its equilibrium against the Wilson action's known plaquette."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BETA, EPS = 6.0, 0.24


def generate(n, precision, start, sweeps, hits, seed, beta=BETA):
    from latticeyangmills_b200 import GluonField

    with GluonField(n, precision) as f:
        acc = f.generate_metropolis(beta, EPS, sweeps, hits, seed, start)
        return f.download(), acc


@pytest.mark.parametrize("start", ["cold", "hot"])
def test_fp64_chain_matches_oracle(oracle, start):
    n = (4, 4, 6, 4)
    sweeps, hits, seed = 2, 5, 77
    U = oracle.gen_cold(n)
    if start == "hot":
        oracle.gen_haar_mix(U, n, 1.0, seed, 0)
    acc = oracle.gen_metropolis_cb(U, n, BETA, EPS, sweeps, hits, seed)
    got, frac = generate(n, "fp64", start, sweeps, hits, seed)
    tries = sweeps * hits * 4 * oracle.volume(n)
    print(start, "max |dU|", np.abs(got - U).max(), "acceptance", frac, acc / tries)
    assert round(frac * tries) == acc
    assert np.abs(got - U).max() < 1e-12


def test_current_start_continues_the_chain(oracle):
    n = (4, 4, 4, 4)
    from latticeyangmills_b200 import GluonField

    with GluonField(n, "fp64") as f:
        f.generate_metropolis(BETA, EPS, 2, 4, 9, "cold")
        f.generate_metropolis(BETA, EPS, 3, 4, 9, "current")
        two = f.download()
        f.generate_metropolis(BETA, EPS, 5, 4, 9, "cold")
        one = f.download()
    assert np.array_equal(one, two)
    U = oracle.gen_cold(n)
    oracle.gen_metropolis_cb(U, n, BETA, EPS, 2, 4, 9)
    oracle.gen_metropolis_cb(U, n, BETA, EPS, 3, 4, 9, sweep0=2)
    assert np.abs(one - U).max() < 1e-12


def test_beta_zero_accepts_every_proposal():
    _, frac = generate((4, 4, 4, 4), "fp64", "cold", 1, 3, 5, beta=0.0)
    assert frac == 1.0


@pytest.mark.parametrize("precision", ["fp64", "fp32_18", "fp32_12"])
def test_equilibrium_plaquette(oracle, precision):
    """beta = 6 Wilson action: <Re tr U_p>/3 = 0.5937.  The reference's proposal
    (random-sign SU(2) factors) accepts about 11% at su3eps = 0.24, so a cold
    start is thermalised after 200 sweeps of 10 hits and a hot start is still
    approaching from below after 300."""
    from latticeyangmills_b200 import GluonField

    n = (8, 8, 8, 8)
    res = {}
    for start in ("cold", "hot"):
        with GluonField(n, precision) as f:
            acc = f.generate_metropolis(BETA, EPS, 200, 10, 31, start)
            vals = []
            for _ in range(10):
                f.generate_metropolis(BETA, EPS, 10, 10, 31, "current")
                vals.append(f.observables().plaq)
            res[start] = (float(np.mean(vals)), vals[-1])
            U = f.download()
        print(precision, start, "acceptance", acc, "plaquette", res[start])
        assert 0.08 < acc < 0.2
        assert max(oracle.unitarity(U)) < (1e-12 if precision == "fp64" else 1e-5)
    assert abs(res["cold"][0] - 0.5937) < 0.005
    assert 0.56 < res["hot"][1] < res["cold"][0] + 0.005


def test_generate_rejects_bad_arguments():
    from latticeyangmills_b200 import GluonField, YmflowError

    with GluonField((4, 4, 4, 4), "fp64") as f:
        for args in [(BETA, 0.0, 1, 1, 1, "cold"), (BETA, 1.5, 1, 1, 1, "cold"), (BETA, EPS, 1, 0, 1, "cold"),
                     (float("nan"), EPS, 1, 1, 1, "cold"), (BETA, EPS, -1, 1, 1, "cold")]:
            with pytest.raises(YmflowError):
                f.generate_metropolis(*args)
        with pytest.raises(YmflowError):
            f.generate_metropolis(BETA, EPS, 1, 1, 1, "current")
    with GluonField((4, 4, 4, 5), "fp64") as f:
        with pytest.raises(YmflowError):
            f.generate_metropolis(BETA, EPS, 1, 1, 1, "cold")
