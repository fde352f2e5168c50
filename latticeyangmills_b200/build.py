"""Builds the CUDA library (libymflow.so, sm_100a) and the drop-in FLOW driver in place."""
from __future__ import annotations

import os
import subprocess
from pathlib import Path

PKG = Path(__file__).resolve().parent


def build(jobs: int | None = None) -> None:
    jobs = jobs or max(1, min(8, os.cpu_count() or 1))
    subprocess.run(["make", "-s", f"-j{jobs}", "-C", str(PKG / "csrc")], check=True)


if __name__ == "__main__":
    build()
