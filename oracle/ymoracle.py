"""ctypes view of the CPU oracle (oracle/ymoracle.c) and of the reference harness
(oracle/_ref/ref_flow).

TEST INFRASTRUCTURE ONLY: tests/, the smoke check and bench.py's CPU-baseline leg
import this module as the checker.  The product (latticeyangmills_b200) never
imports it.

Fields are numpy float64 arrays shaped (Nt, Nz, Ny, Nx, 4, 18) or flat with the
same byte order: the reference's .bin layout (src/InputOutput/inputconf.cpp:114-155).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "libymoracle.so"
REF_BIN = HERE / "_ref" / "ref_flow"

_lib = None
_D = ctypes.POINTER(ctypes.c_double)
_I4 = ctypes.c_int * 4


def reference_tree():
    """The reference's source tree: $YM_REFERENCE, else a checkout named
    `reference` beside this repository; None where neither exists."""
    p = Path(os.environ["YM_REFERENCE"]) if os.environ.get("YM_REFERENCE") else HERE.parent.parent / "reference"
    return p if p.is_dir() else None


def build() -> None:
    """Compile the oracle (and the reference harness where the reference tree exists)."""
    targets = ["oracle"]
    if reference_tree() is not None:
        targets.append("ref")
    subprocess.run(["make", "-s", "-C", str(HERE)] + targets, check=True)


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        l = ctypes.CDLL(str(LIB_PATH))
        l.yo_mul.argtypes = [_D, _D, _D]
        l.yo_dag.argtypes = [_D, _D]
        l.yo_exp.argtypes = [_D, _D]
        l.yo_exp_many.argtypes = [_D, _D, ctypes.c_long]
        l.yo_derivative.argtypes = [_D, _I4, ctypes.c_int, _D]
        l.yo_flow_step.argtypes = [_D, _D, _I4, ctypes.c_double]
        l.yo_flow_stage.argtypes = [_D, _D, _I4, ctypes.c_double, ctypes.c_int]
        l.yo_superobs.argtypes = [_D, _I4, _D]
        l.yo_flow.argtypes = [_D, _I4, ctypes.c_double, ctypes.c_int, ctypes.c_int, _D]
        l.yo_flow.restype = ctypes.c_int
        l.yo_philox4x32.argtypes = [ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint32),
                                    ctypes.POINTER(ctypes.c_uint32)]
        l.yo_gen_expiah.argtypes = [_D, _I4, ctypes.c_double, ctypes.c_uint64, ctypes.c_uint32]
        l.yo_gen_haar_mix.argtypes = [_D, _I4, ctypes.c_double, ctypes.c_uint64, ctypes.c_uint32]
        l.yo_gen_cold.argtypes = [_D, _I4]
        l.yo_gen_metropolis.argtypes = [_D, _I4, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                        ctypes.c_int, ctypes.c_uint64]
        l.yo_gen_metropolis.restype = ctypes.c_double
        l.yo_gen_metropolis_cb.argtypes = [_D, _I4, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                           ctypes.c_int, ctypes.c_uint64, ctypes.c_uint32]
        l.yo_gen_metropolis_cb.restype = ctypes.c_long
        l.yo_reunitarize.argtypes = [_D, ctypes.c_long]
        l.yo_unitarity.argtypes = [_D, ctypes.c_long, _D]
        _lib = l
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_D)


def _dims(n):
    return _I4(*[int(v) for v in n])


def volume(n) -> int:
    return int(n[0]) * int(n[1]) * int(n[2]) * int(n[3])


def empty_field(n) -> np.ndarray:
    return np.zeros((n[3], n[2], n[1], n[0], 4, 18), dtype=np.float64)


def gen_expiah(n, a: float, seed: int, config: int = 0) -> np.ndarray:
    U = empty_field(n)
    lib().yo_gen_expiah(_p(U), _dims(n), a, seed, config)
    return U


def gen_haar_mix(U: np.ndarray, n, frac: float, seed: int, config: int = 0) -> np.ndarray:
    lib().yo_gen_haar_mix(_p(U), _dims(n), frac, seed, config)
    return U


def gen_cold(n) -> np.ndarray:
    U = empty_field(n)
    lib().yo_gen_cold(_p(U), _dims(n))
    return U


def gen_metropolis(n, beta: float, su3eps: float, sweeps: int, hits: int, seed: int):
    U = gen_cold(n)
    acc = lib().yo_gen_metropolis(_p(U), _dims(n), beta, su3eps, sweeps, hits, seed)
    return U, acc


def gen_metropolis_cb(U: np.ndarray, n, beta: float, su3eps: float, sweeps: int, hits: int, seed: int,
                      sweep0: int = 0) -> int:
    """The device generator's checkerboard chain, in place on U; returns the
    number of accepted proposals."""
    return int(lib().yo_gen_metropolis_cb(_p(U), _dims(n), beta, su3eps, sweeps, hits, seed, sweep0))


def su3_exp(q: np.ndarray) -> np.ndarray:
    q = np.ascontiguousarray(q, dtype=np.float64).reshape(-1, 18)
    r = np.empty_like(q)
    lib().yo_exp_many(_p(q), _p(r), q.shape[0])
    return r


def derivative(U: np.ndarray, n, mu: int) -> np.ndarray:
    Z = np.empty((volume(n), 18), dtype=np.float64)
    lib().yo_derivative(_p(U), _dims(n), mu, _p(Z))
    return Z


def superobs(U: np.ndarray, n):
    """(plaq, topc, energy) as the reference's SuperObs."""
    o = np.zeros(3)
    lib().yo_superobs(_p(U), _dims(n), _p(o))
    return float(o[0]), float(o[1]), float(o[2])


def flow_stage(U: np.ndarray, Z: np.ndarray, n, eps: float, stage: int) -> None:
    """One RK3 stage (0, 1, 2) of U in place on the periodic lattice n; Z (4 V
    x 18 doubles) carries the RK generator between the stages of a step."""
    lib().yo_flow_stage(_p(U), _p(Z), _dims(n), eps, int(stage))


def flow(U: np.ndarray, n, eps: float, nsteps: int, every: int) -> np.ndarray:
    """Flows U in place; rows (step, t, plaq, topc, energy)."""
    rows = nsteps // max(every, 1) + 2
    tab = np.zeros((rows, 5))
    k = lib().yo_flow(_p(U), _dims(n), eps, nsteps, every, _p(tab))
    return tab[:k].copy()


def reunitarize(U: np.ndarray) -> np.ndarray:
    lib().yo_reunitarize(_p(U), U.size // 18)
    return U


def unitarity(U: np.ndarray):
    o = np.zeros(2)
    lib().yo_unitarity(_p(U), U.size // 18, _p(o))
    return float(o[0]), float(o[1])


def philox(ctr, key):
    c = (ctypes.c_uint32 * 4)(*ctr)
    k = (ctypes.c_uint32 * 2)(*key)
    o = (ctypes.c_uint32 * 4)()
    lib().yo_philox4x32(c, k, o)
    return list(o)


# --- the reference itself (oracle/_ref/ref_flow) -----------------------------------------

def ref_available() -> bool:
    return REF_BIN.exists()


def write_bin(U: np.ndarray, path) -> None:
    np.ascontiguousarray(U, dtype="<f8").tofile(str(path))


def read_bin(path, n) -> np.ndarray:
    return np.fromfile(str(path), dtype="<f8").reshape(n[3], n[2], n[1], n[0], 4, 18)


def ref_flow(conf_path, n, eps: float, nsteps: int, every: int, out_bin=None) -> np.ndarray:
    """Rows (step, t, plaq, topc, energy) printed by the reference's own code."""
    args = [str(REF_BIN), "flow", str(conf_path)] + [str(int(v)) for v in n] + [repr(float(eps)), str(nsteps), str(every)]
    if out_bin is not None:
        args.append(str(out_bin))
    out = subprocess.run(args, check=True, capture_output=True, text=True).stdout
    return np.array([[float(v) for v in line.split()] for line in out.strip().splitlines()])


def ref_exp(q: np.ndarray) -> np.ndarray:
    q = np.ascontiguousarray(q, dtype=np.float64).reshape(-1, 18)
    with tempfile.TemporaryDirectory() as d:
        fi, fo = Path(d) / "q.bin", Path(d) / "r.bin"
        q.tofile(str(fi))
        subprocess.run([str(REF_BIN), "exp", str(fi), str(q.shape[0]), str(fo)], check=True)
        return np.fromfile(str(fo), dtype=np.float64).reshape(-1, 18)


def ref_derivative(conf_path, n) -> np.ndarray:
    with tempfile.TemporaryDirectory() as d:
        fo = Path(d) / "z.bin"
        subprocess.run([str(REF_BIN), "deriv", str(conf_path)] + [str(int(v)) for v in n] + [str(fo)], check=True)
        return read_bin(fo, n)


def ref_time(conf_path, n, eps: float, nsteps: int) -> dict:
    import json
    args = [str(REF_BIN), "time", str(conf_path)] + [str(int(v)) for v in n] + [repr(float(eps)), str(nsteps)]
    out = subprocess.run(args, check=True, capture_output=True, text=True).stdout
    return json.loads(out.strip().splitlines()[-1])
