"""Known answers from mathematics on the device path: e^{iQ} against a general
matrix exponential, RK3 order, the monotone plaquette, and the two-row
(12-real) storage round trip."""
import numpy as np
import pytest
from scipy.linalg import expm

from test_known_answers import random_hermitian_traceless, to_complex, to_real

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("scale", [0.0, 1e-6, 1e-3, 0.1, 1.0, 4.0])
def test_device_exponential_against_expm(scale):
    from latticeyangmills_b200 import su3_exp

    rng = np.random.default_rng(int(scale * 1000) + 7)
    q = random_hermitian_traceless(256, scale, rng)
    got = to_complex(su3_exp(to_real(q)))
    want = np.array([expm(1j * m) for m in q])
    assert np.abs(got - want).max() < 1e-13 * max(1.0, scale ** 2)


def test_device_rk3_is_third_order():
    from latticeyangmills_b200 import GluonField

    n = (8, 8, 8, 8)
    with GluonField(n, "fp64") as f:
        f.init_links("expiah", 0.3, 11)
        U0 = f.download()

        def plaq_at(eps, t=0.16):
            f.upload(U0)
            rows = f.flow(eps, int(round(t / eps)), 0)
            assert abs(rows[-1, 1] - t) < 1e-9
            return rows[-1, 2]

        fine = plaq_at(0.00125)
        errs = [abs(plaq_at(e) - fine) for e in (0.04, 0.02, 0.01)]
    ratios = [errs[0] / errs[1], errs[1] / errs[2]]
    print("errors", errs, "ratios", ratios)
    assert all(6.0 < r < 10.0 for r in ratios)


@pytest.mark.parametrize("precision", ["fp64", "fp32_18", "fp32_12"])
def test_device_flow_raises_the_plaquette(precision):
    from latticeyangmills_b200 import GluonField

    with GluonField((16, 16, 16, 16), precision) as f:
        f.init_links("expiah", 0.35, 3)
        rows = f.flow(0.02, 100, 1, reunit_every=10 if precision != "fp64" else 0)
    # the flow descends the Wilson (plaquette) action; the clover energy is a
    # different discretisation and need not be monotone at the first steps
    assert np.all(np.diff(rows[:, 2]) > 0)


def test_two_row_storage_round_trip():
    """12-real storage keeps rows 0 and 1 in FP32 and rebuilds row 2."""
    from latticeyangmills_b200 import GluonField

    n = (8, 8, 8, 8)
    with GluonField(n, "fp64") as f:
        f.init_links("expiah", 0.5, 21)
        U = f.download()
    with GluonField(n, "fp32_12") as f:
        f.upload(U)
        back = f.download()
    assert np.abs(back - U).max() < 1e-6
