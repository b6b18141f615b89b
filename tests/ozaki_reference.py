"""CPU emulation of the int8 digit GEMM (et_b200/csrc/ozaki_gemm.cu), operation for operation.

Each row of op(A) (column of op(B)) is scaled by 2^-e, e the frexp exponent of its largest
magnitude, and cut into `digits` 7-bit digits by truncation (exact in FP64); the digit products of
one diagonal d = t + u (d <= digits - 1) are summed exactly (integers below 2^31, exact in FP64 here,
int32 on the GPU) per K chunk
of 16384; per (chunk, pass) the weighted diagonals are summed in FP64 in the kernel's order, scaled
by 2^(ea + eb) and added to C.  With alpha = 1 and beta = 0 every step is exact or the same FP64
operation in the same order as the GPU, so the results agree bit for bit.
"""

import numpy as np

K_CHUNK = 16384
MAX_DIAG_PER_PASS = 4


def exponents(X):
    """Row exponents of X (rows x K): frexp exponent of each row's max |x| (None for zero rows)."""
    m = np.abs(X).max(axis=1)
    _, e = np.frexp(m)
    return np.where(m > 0, e, 0), m > 0


def digit_planes(X, digits):
    e, nz = exponents(X)
    y = np.ldexp(X, -e[:, None]) * nz[:, None]
    out = np.empty((digits,) + X.shape)
    for t in range(digits):
        y = y * 128.0
        d = np.trunc(y)
        y = y - d
        out[t] = d
    return out, e, nz


def ozaki_gemm(A, B, digits=7):
    """C = A @ B (alpha = 1, beta = 0) as the kernel computes it; A (m x k), B (k x n)."""
    m, k = A.shape
    n = B.shape[1]
    DA, ea, nza = digit_planes(A, digits)
    DB, eb, nzb = digit_planes(B.T, digits)
    scale = np.exp2(ea.astype(np.float64))[:, None] * nza[:, None] * (np.exp2(eb.astype(np.float64)) * nzb)[None, :]
    passes = [(0, min(digits, MAX_DIAG_PER_PASS))]
    if digits > MAX_DIAG_PER_PASS:
        passes.append((MAX_DIAG_PER_PASS, digits))
    C = np.zeros((m, n))
    first = True
    for k0 in range(0, k, K_CHUNK):
        ks = slice(k0, min(k, k0 + K_CHUNK))
        for d0, d1 in passes:
            v = np.zeros((m, n))
            for d in range(d0, d1):
                # integer digit products below 2^31: exact in FP64 BLAS whatever its summation order
                acc = np.zeros((m, n))
                for t in range(max(0, d - digits + 1), min(d, digits - 1) + 1):
                    acc += DA[t][:, ks] @ DB[d - t][:, ks].T
                assert np.abs(acc).max(initial=0) < 2 ** 31
                v = v + np.exp2(-7.0 * (d + 2)) * acc
            x = scale * v
            C = x if first else x + C
            first = False
    return C
