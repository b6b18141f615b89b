"""The int8 digit GEMM's arithmetic, emulated on the CPU (tests/ozaki_reference.py): its accuracy
against FP64 for the digit counts the library offers, and the int32 range of its accumulators."""

import numpy as np
import pytest

import ozaki_reference as oz


@pytest.mark.parametrize("digits,tol", [(7, 5e-14), (6, 3e-12), (5, 3e-10), (4, 3e-8)])
def test_digit_gemm_accuracy(digits, tol):
    rng = np.random.default_rng(digits)
    A = rng.standard_normal((40, 300)) * np.exp2(rng.integers(-20, 20, size=(40, 1)))
    B = rng.standard_normal((300, 30)) * np.exp2(rng.integers(-20, 20, size=(1, 30)))
    C = oz.ozaki_gemm(A, B, digits)
    ref = A @ B
    # the error lies below the last digit of each row and column: relative to |A_r||B_c|
    rowcol = np.abs(A).max(axis=1)[:, None] * np.abs(B).max(axis=0)[None, :] * np.sqrt(A.shape[1])
    assert np.abs(C - ref).max() <= tol * rowcol.max()
    assert (np.abs(C - ref) / rowcol).max() <= tol


def test_long_k_chunks_and_zero_rows():
    """K across chunk boundaries; all-zero rows and columns give exact zeros."""
    rng = np.random.default_rng(3)
    A = rng.standard_normal((8, 40000))
    B = rng.standard_normal((40000, 6))
    A[3] = 0.0
    B[:, 2] = 0.0
    C = oz.ozaki_gemm(A, B, 7)
    ref = A @ B
    assert np.all(C[3] == 0.0) and np.all(C[:, 2] == 0.0)
    # the products beyond the last diagonal (t + u >= 7) dominate: ~1.5e-13 of the largest output
    assert np.abs(C - ref).max() <= 5e-13 * np.abs(ref).max()
