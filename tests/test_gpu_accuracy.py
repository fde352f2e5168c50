"""Accuracy of the mixed forms against the FP64 flow on the benchmark's other
configurations (the 32^4 one is in test_gpu_tile.py / test_gpu_split.py):

* 64^4, U = e^{iaH} (a = 0.35) with 5 % of the links replaced by Haar-random
  SU(3), eps 0.02 to t = 6, t^2 E and Q every 5 steps, reunitarisation every
  10 steps: both FP32 forms against the FP64 flow of the same seeded field.
* 64 configurations of mixed sizes (16 each of 8^4, 12^4, 16^4, 16^3 x 32),
  a drawn in [0.25, 0.45] per configuration, flowed together as one FP32
  ensemble to t = 2 (eps 0.01): every configuration against its own FP64 flow.

Bounds: |d(t^2 E)| / t^2 E < 1e-6 and |dQ| < 1e-4 at the final t; every
earlier row of t^2 E within 1e-5 (t^2 E is small at small t)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _errors(r32, r64):
    rel = np.abs(r32[1:, 5] - r64[1:, 5]) / np.abs(r64[1:, 5])
    dq = np.abs(r32[:, 3] - r64[:, 3])
    return rel, dq


@pytest.mark.parametrize("precision", ["fp32_12", "fp32_18"])
def test_64_haar_mixed_meets_the_target_at_t6(precision):
    from latticeyangmills_b200 import GluonField

    n, a, haar, eps, steps, every, seed = (64, 64, 64, 64), 0.35, 0.05, 0.02, 300, 5, 20260
    with GluonField(n, "fp64") as f:
        f.init_links("expiah", a, seed, 0, haar)
        r64 = f.flow(eps, steps, every)
    with GluonField(n, precision) as f:
        f.init_links("expiah", a, seed, 0, haar)
        r32 = f.flow(eps, steps, every, reunit_every=10)
    rel, dq = _errors(r32, r64)
    print(precision, "final rel t2E %.3g max %.3g; |dQ| final %.3g max %.3g" % (rel[-1], rel.max(), dq[-1], dq.max()))
    assert abs(r32[-1, 1] - 6.0) < 1e-9 and r32.shape[0] == steps // every + 1
    assert rel[-1] < 1e-6
    assert rel.max() < 1e-5
    assert dq.max() < 1e-4


def test_fp32_ensemble_matches_fp64_per_configuration_at_t2():
    from latticeyangmills_b200 import Ensemble, GluonField

    sizes = [(8,) * 4] * 16 + [(12,) * 4] * 16 + [(16,) * 4] * 16 + [(16, 16, 16, 32)] * 16
    a_list = np.random.default_rng(4).uniform(0.25, 0.45, size=len(sizes))
    seed, eps, steps = 20260, 0.01, 200
    with Ensemble(sizes, "fp32_12") as ens:
        for c in range(len(sizes)):
            ens.init_links(c, "expiah", float(a_list[c]), seed + c, c)
        rows = ens.flow(eps, steps, 50, reunit_every=10)  # rows x conf x (step, t, plaq, topc, energy, t2E)
    worst_rel = worst_dq = 0.0
    for c, n in enumerate(sizes):
        with GluonField(n, "fp64") as f:
            f.init_links("expiah", float(a_list[c]), seed + c, c)
            r64 = f.flow(eps, steps, 50)
        rel, dq = _errors(rows[:, c, :], r64)
        assert abs(rows[-1, c, 1] - 2.0) < 1e-9
        assert rel[-1] < 1e-6, (c, n, rel)
        assert rel.max() < 1e-5, (c, n, rel)
        assert dq.max() < 1e-4, (c, n, dq)
        worst_rel, worst_dq = max(worst_rel, rel[-1]), max(worst_dq, dq.max())
    print("ensemble worst final rel t2E %.3g, worst |dQ| %.3g" % (worst_rel, worst_dq))
