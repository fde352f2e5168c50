"""Mixed paths (FP32 link storage and site arithmetic, FP64 reductions) against
the FP64 GPU path: each result's error against FP64."""
import numpy as np
import pytest

from conftest import case_field, load_case

pytestmark = pytest.mark.gpu


def flow(precision, U, n, eps, nsteps, every, reunit=10):
    from latticeyangmills_b200 import GluonField

    with GluonField(n, precision) as f:
        f.upload(U)
        return f.flow(eps, nsteps, every, reunit_every=reunit)


@pytest.mark.parametrize("precision", ["fp32_18", "fp32_12"])
def test_mixed_matches_fp64_metropolis(precision):
    case = load_case("g8_metropolis")
    U = case_field(case)
    n = tuple(case["dims"])
    ref = flow("fp64", U, n, case["eps"], case["nsteps"], 10)
    got = flow(precision, U, n, case["eps"], case["nsteps"], 10)
    rel_e = np.abs(got[:, 5] - ref[:, 5])[1:] / np.abs(ref[:, 5])[1:]
    dq = np.abs(got[:, 3] - ref[:, 3])
    print(precision, "max rel t2E", rel_e.max(), "max |dQ|", dq.max(), "plaq", np.abs(got[:, 2] - ref[:, 2]).max())
    assert rel_e.max() < 1e-5
    assert dq.max() < 1e-4
    assert np.abs(got[:, 2] - ref[:, 2]).max() < 1e-5


@pytest.mark.parametrize("precision", ["fp32_18", "fp32_12"])
def test_mixed_matches_fp64_rough_field(precision):
    case = load_case("g16x32_expiah")
    U = case_field(case)
    n = tuple(case["dims"])
    ref = flow("fp64", U, n, 0.01, 100, 25)
    got = flow(precision, U, n, 0.01, 100, 25)
    rel_e = np.abs(got[:, 5] - ref[:, 5])[1:] / np.abs(ref[:, 5])[1:]
    print(precision, "max rel t2E", rel_e.max(), "max |dQ|", np.abs(got[:, 3] - ref[:, 3]).max())
    assert rel_e.max() < 1e-5
    assert np.abs(got[:, 3] - ref[:, 3]).max() < 1e-4


def test_fp32_links_stay_unitary_with_reunitarisation(oracle):
    from latticeyangmills_b200 import GluonField

    n = (8, 8, 8, 8)
    with GluonField(n, "fp32_18") as f:
        f.init_links("expiah", 0.35, 3)
        f.flow(0.02, 60, 0, reunit_every=10)
        U = f.download()
    assert max(oracle.unitarity(U)) < 1e-5
