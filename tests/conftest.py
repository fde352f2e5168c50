"""Shared fixtures.  `-m gpu` tests need a B200; everything else runs on CPU.

The oracle (oracle/ymoracle.c, oracle/_ref) is the checker here and nowhere
in the product."""
from __future__ import annotations

import hashlib
import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an NVIDIA B200 (sm_100a) and libymflow.so")


def load_case(name: str) -> dict:
    return json.loads((GOLDEN / f"{name}.json").read_text())


def sha256(U: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(U, dtype="<f8").tobytes()).hexdigest()


def case_field(case: dict) -> np.ndarray:
    """The input field of a golden case: the committed .bin, or the seeded
    generator's output (checked against the recorded sha256)."""
    from oracle import ymoracle as yo

    n = tuple(case["dims"])
    if case["bin_committed"]:
        U = yo.read_bin(GOLDEN / f"{case['name']}.bin", n).copy()
    else:
        g = case["generator"]
        if g["kind"] == "expiah":
            U = yo.gen_expiah(n, g["a"], g["seed"], g.get("config", 0))
        elif g["kind"] == "expiah_haar":
            U = yo.gen_expiah(n, g["a"], g["seed"], g.get("config", 0))
            yo.gen_haar_mix(U, n, g["haar_frac"], g["seed"], g.get("config", 0))
        elif g["kind"] == "cold":
            U = yo.gen_cold(n)
        else:
            raise ValueError(g["kind"])
    if sha256(U) != case["sha256"]:
        pytest.skip(f"{case['name']}: regenerated field differs from the recorded one (libm bits differ here)")
    return U


def topc_tolerance(energy: float, rel: float = 1e-12) -> float:
    """Absolute tolerance on topc: rel * an upper bound of sum_x |q(x)|.

    |Re tr(G_a G_b)| <= (|G_a|^2 + |G_b|^2)/2, so sum_x |q(x)| <= |energy| / (512 pi^2)."""
    return rel * abs(energy) / (512.0 * np.pi ** 2) + 1e-300


@pytest.fixture(scope="session")
def oracle():
    from oracle import ymoracle as yo

    yo.lib()
    return yo
