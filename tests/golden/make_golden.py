"""Regenerates the golden fixtures in this folder from the REFERENCE's own code.

Run from the repository root where the reference tree exists (it is read by
oracle/Makefile to build oracle/_ref/ref_flow):

    python tests/golden/make_golden.py

Each case is a seeded synthetic field written in the reference's .bin layout
(src/InputOutput/inputconf.cpp:114-155), flowed by the reference's own RK3 step
and SuperObs (oracle/_ref/ref_flow), with every printed number kept at full
precision.  Small inputs are committed as .bin files; larger ones are
regenerated by the oracle's seeded generator and checked against the recorded
sha256 before use.
"""
from __future__ import annotations

import hashlib
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from oracle import ymoracle as yo  # noqa: E402

OUT = Path(__file__).resolve().parent

CASES = [
    # name, dims, generator, flow (eps, nsteps, every), commit_bin
    ("g4_expiah", (4, 4, 4, 4), {"kind": "expiah", "a": 0.35, "seed": 1}, (0.01, 20, 1), True),
    ("g3456_expiah", (3, 4, 5, 6), {"kind": "expiah", "a": 0.5, "seed": 2}, (0.02, 10, 1), True),
    ("g2324_expiah", (2, 3, 2, 4), {"kind": "expiah", "a": 0.4, "seed": 6}, (0.01, 5, 1), True),
    ("g8_metropolis", (8, 8, 8, 8),
     {"kind": "metropolis", "beta": 6.0, "su3eps": 0.24, "sweeps": 200, "hits": 30, "seed": 3},
     (0.01, 100, 1), True),
    ("g8_haar", (8, 8, 8, 8), {"kind": "expiah_haar", "a": 0.35, "seed": 5, "haar_frac": 0.05},
     (0.02, 20, 5), False),
    ("g16x32_expiah", (16, 16, 16, 32), {"kind": "expiah", "a": 0.35, "seed": 4}, (0.01, 10, 5), False),
    # configuration 2 at full length (about 15 min of the reference on one core)
    ("g16x32_full", (16, 16, 16, 32), {"kind": "expiah", "a": 0.35, "seed": 4}, (0.01, 200, 10), False),
    ("g4_cold", (4, 4, 4, 4), {"kind": "cold"}, (0.01, 2, 1), False),
]


def generate(dims, g):
    """The seeded field of a case (oracle generators; see oracle/ymoracle.c)."""
    k = g["kind"]
    if k == "expiah":
        return yo.gen_expiah(dims, g["a"], g["seed"], g.get("config", 0))
    if k == "expiah_haar":
        U = yo.gen_expiah(dims, g["a"], g["seed"], g.get("config", 0))
        return yo.gen_haar_mix(U, dims, g["haar_frac"], g["seed"], g.get("config", 0))
    if k == "metropolis":
        U, acc = yo.gen_metropolis(dims, g["beta"], g["su3eps"], g["sweeps"], g["hits"], g["seed"])
        g["acceptance"] = acc
        return U
    if k == "cold":
        return yo.gen_cold(dims)
    raise ValueError(k)


def sha256(U: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(U, dtype="<f8").tobytes()).hexdigest()


def make_case(name, dims, gen, flow, commit_bin):
    eps, nsteps, every = flow
    gen = dict(gen)
    U = generate(dims, gen)
    binp = OUT / f"{name}.bin"
    yo.write_bin(U, binp)
    rows = yo.ref_flow(binp, dims, eps, nsteps, every)
    rec = {
        "name": name, "dims": list(dims), "generator": gen, "eps": eps, "nsteps": nsteps, "every": every,
        "sha256": sha256(U), "bin_committed": commit_bin,
        "columns": ["step", "t", "plaq", "topc", "energy"],
        "rows": rows.tolist(),
    }
    text = json.dumps({k: v for k, v in rec.items() if k != "rows"}, indent=1)[:-2]
    text += ',\n "rows": [\n' + ",\n".join("  " + json.dumps(r) for r in rec["rows"]) + "\n ]\n}\n"
    (OUT / f"{name}.json").write_text(text)
    if not commit_bin:
        binp.unlink()
    print(name, "rows", len(rows), "plaq0", rows[0, 2])


def make_exp_cases():
    """Reference exp(Q) = e^{iQ} on Hermitian traceless Q across scales, plus
    degenerate spectra and the zero matrix (where the reference returns NaN)."""
    rng = np.random.default_rng(11)
    qs = []
    for scale in (1e-4, 1e-3, 1e-2, 0.05, 0.1, 0.3, 1.0, 2.0):
        for _ in range(16):
            m = rng.normal(size=(3, 3)) + 1j * rng.normal(size=(3, 3))
            h = (m + m.conj().T) / 2
            h -= np.trace(h) / 3 * np.eye(3)
            qs.append(scale * h)
    for s in (1e-3, 0.1, 1.0):
        v = rng.normal(size=(3, 3)) + 1j * rng.normal(size=(3, 3))
        q_, _ = np.linalg.qr(v)
        qs.append(q_ @ np.diag([s, s, -2 * s]) @ q_.conj().T)   # doubly degenerate
        qs.append(q_ @ np.diag([-s, -s, 2 * s]) @ q_.conj().T)
        qs.append(np.diag([s, -s, 0.0]).astype(complex))       # c0 = 0 exactly
    qs.append(np.zeros((3, 3), dtype=complex))
    q = np.stack([np.stack([x.real, x.imag], -1).reshape(18) for x in qs])
    r = yo.ref_exp(q)
    np.savez(OUT / "exp_cases.npz", q=q, r=r)
    print("exp cases", q.shape[0], "nan rows", int(np.isnan(r).any(axis=1).sum()))


APP_JSON = {
    "App": {"type": "FLOW", "params": {"epsilon": 0.01, "tauFinal": 0.1}},
    "LatticeSize": {"x": 4, "y": 4, "z": 4, "t": 4},
    "SubLatticeSize": {"x": 4, "y": 4, "z": 4, "t": 4},
    "Action": {"type": "puregauge", "params": {"beta": 6.0}},
    "Observables": ["superobs"],
    "InputDir": "@IN@", "OutputDir": "@OUT@",
}


def app_inputs(indir: Path) -> None:
    """The FLOW app case's input directory: two 4^4 configurations."""
    import shutil
    indir.mkdir(parents=True, exist_ok=True)
    shutil.copy(OUT / "g4_expiah.bin", indir / "conf0000.bin")
    shutil.copy(OUT / "g4b_expiah.bin", indir / "conf0001.bin")


def make_app_case():
    """Runs the reference's whole FLOW application (oracle/_ref/lattice_qcd) and
    keeps its terminal output and output files."""
    import shutil
    import subprocess
    import tempfile
    yo.write_bin(yo.gen_expiah((4, 4, 4, 4), 0.3, 7), OUT / "g4b_expiah.bin")
    case = OUT / "app_flow"
    if case.exists():
        shutil.rmtree(case)
    (case / "expected" / "flow").mkdir(parents=True)
    (case / "input.json").write_text(json.dumps(APP_JSON, indent=1) + "\n")
    with tempfile.TemporaryDirectory() as d:
        d = Path(d)
        app_inputs(d / "in")
        text = (case / "input.json").read_text().replace("@IN@", str(d / "in")).replace("@OUT@", str(d / "out"))
        (d / "run.json").write_text(text)
        out = subprocess.run([str(yo.HERE / "_ref" / "lattice_qcd"), str(d / "run.json")], check=True,
                             capture_output=True, text=True).stdout
        lines = [l for l in out.splitlines(keepends=True) if not l.startswith("Total time taken")]
        (case / "expected" / "stdout.txt").write_text("".join(lines))
        for f in ["observables.dat", "flow/conf0000.dat", "flow/conf0001.dat"]:
            shutil.copy(d / "out" / f, case / "expected" / f)
    print("app case", len(lines), "terminal lines")


def make_deriv_case():
    dims = (4, 4, 4, 4)
    Z = yo.ref_derivative(OUT / "g4_expiah.bin", dims)
    np.save(OUT / "g4_expiah_deriv.npy", Z)
    print("deriv", Z.shape)


if __name__ == "__main__":
    yo.build()
    assert yo.ref_available(), "oracle/_ref/ref_flow missing: the reference tree is needed here"
    only = set(sys.argv[1:])
    for c in CASES:
        if not only or c[0] in only:
            make_case(*c)
    if not only or "exp" in only:
        make_exp_cases()
    if not only or "deriv" in only:
        make_deriv_case()
    if not only or "app" in only:
        make_app_case()
