"""Build recipe for the oracle's C code (test infrastructure): oracle/_lib/libintegrals.so."""

from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def build_oracle() -> str:
    build_et_cpu()
    out_dir = os.path.join(HERE, "_lib")
    os.makedirs(out_dir, exist_ok=True)
    out = os.path.join(out_dir, "libintegrals.so")
    src = os.path.join(HERE, "integrals.c")
    if not os.path.exists(out) or os.path.getmtime(out) < os.path.getmtime(src):
        subprocess.check_call(["gcc", "-O2", "-fPIC", "-shared", "-o", out, src, "-lm"])
    return out


def build_et_cpu() -> str:
    """oracle/_lib/libet_cpu.so: the OpenMP steps of the CPU restatement of eT's algorithm."""
    out_dir = os.path.join(HERE, "_lib")
    os.makedirs(out_dir, exist_ok=True)
    out = os.path.join(out_dir, "libet_cpu.so")
    src = os.path.join(HERE, "et_cpu.c")
    if not os.path.exists(out) or os.path.getmtime(out) < os.path.getmtime(src):
        subprocess.check_call(["gcc", "-O3", "-march=x86-64-v3", "-fopenmp", "-fPIC", "-shared", "-o", out, src])
    return out


if __name__ == "__main__":
    print(build_oracle())
    print(build_et_cpu())
