"""Time the split-BF16 tensor-core GEMM of libccsd_gpu on one shape (diagnostics CLI).

    python -m et_b200.gemm_probe --m 10240 --n 10240 --k 10240 --reps 3

Prints one JSON line: per-launch device time (CUDA events around each launch on the launching
stream), issued tensor TFLOP/s (3 bf16 products x 2mnk) and the FP64-equivalent TFLOP/s (2mnk).
The (ov)^3 shape 10240^3 is the C2/D2 product of the o=32, v=320 ground-state workload.
"""

from __future__ import annotations

import argparse
import json

import numpy as np


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--m", type=int, default=10240)
    p.add_argument("--n", type=int, default=10240)
    p.add_argument("--k", type=int, default=10240)
    p.add_argument("--reps", type=int, default=3)
    args = p.parse_args()
    from et_b200 import CCSD
    rng = np.random.default_rng(0)
    A = np.asfortranarray(rng.standard_normal((args.m, args.k)))
    B = np.asfortranarray(rng.standard_normal((args.k, args.n)))
    with CCSD(2, 3, 4) as ctx:
        ctx.selftest_gemm(A[:256, :256], B[:256, :256], mixed=True)      # warm-up
        ctx.set_profiling(True)
        for _ in range(args.reps):
            ctx.selftest_gemm(A, B, mixed=True)
        n, ms, fl = ctx.gemm_profile()
    per = ms / max(n, 1)
    print(json.dumps({"m": args.m, "n": args.n, "k": args.k, "launches": n, "ms_per_launch": round(per, 4),
                      "issued_tflops": round(fl / n / (per * 1e-3) / 1e12, 1),
                      "fp64_equivalent_tflops": round(2.0 * args.m * args.n * args.k / (per * 1e-3) / 1e12, 1)}))


if __name__ == "__main__":
    main()
