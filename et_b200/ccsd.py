"""Host-side mirror of eT's CCSD wavefunction entry points over the C ABI (include/ccsd_gpu.h).

``CCSD`` exposes the type-bound procedures of eT's ``class(ccsd)`` that the
ground-state DIIS solver and the Davidson excited-state solver call
(src/wavefunctions/ccsd/ccsd_class.F90:99-253): ``construct_omega``,
``jacobian_transformation``, ``jacobian_transpose_transformation``,
``calculate_energy``, ``construct_fock``/``construct_t1_cholesky`` (run by
``set_amplitudes``), plus the device-resident ground-state solver.

The compute runs in ``libccsd_gpu.so`` (sm_100a); there is no CPU fallback: if
the library cannot be loaded, or no sm_100 device is present, every call
raises ``CCSDGPUError``.
"""

from __future__ import annotations

import ctypes
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libccsd_gpu.so")

FP64 = 0
MIXED = 1

STATUS = {
    0: "ok", -1: "invalid argument", -2: "CUDA error", -3: "out of device memory",
    -4: "missing input", -5: "not converged", -6: "non-finite value", -7: "singular system",
    -8: "no sm_100 device", -9: "tensor-core GEMM wait timed out",
}


class CCSDGPUError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


class Options(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("precision", ctypes.c_int32), ("ladder_batch", ctypes.c_int64),
                ("mixed_min_flops", ctypes.c_int64), ("mixed_k_chunk", ctypes.c_int64),
                ("autotune", ctypes.c_int64), ("ladder_pair_budget", ctypes.c_int64), ("reserved", ctypes.c_int64 * 2)]


class DavidsonOptions(ctypes.Structure):
    _fields_ = [("max_iterations", ctypes.c_int32), ("block", ctypes.c_int32), ("max_reduced_dim", ctypes.c_int32),
                ("start_from_vectors", ctypes.c_int32), ("residual_threshold", ctypes.c_double),
                ("energy_threshold", ctypes.c_double), ("reserved", ctypes.c_int32 * 8)]


class SolverOptions(ctypes.Structure):
    _fields_ = [("max_iterations", ctypes.c_int32), ("diis_dimension", ctypes.c_int32),
                ("omega_threshold", ctypes.c_double), ("energy_threshold", ctypes.c_double),
                ("refine_threshold", ctypes.c_double), ("refine_target", ctypes.c_double),
                ("refresh_digits", ctypes.c_int32), ("reserved", ctypes.c_int32 * 5)]


class BatchSystem(ctypes.Structure):
    _fields_ = [("n_o", ctypes.c_int64), ("n_v", ctypes.c_int64), ("n_J", ctypes.c_int64),
                ("L_mo", ctypes.POINTER(ctypes.c_double)), ("h_mo", ctypes.POINTER(ctypes.c_double)),
                ("eps", ctypes.POINTER(ctypes.c_double)), ("e_hf", ctypes.c_double),
                ("t_out", ctypes.POINTER(ctypes.c_double))]


_lib = None

# name -> (restype, argtypes)
_VP = ctypes.c_void_p
_DP = ctypes.POINTER(ctypes.c_double)
_I64 = ctypes.c_int64
SIGNATURES = {
    "ccsd_gpu_create": (ctypes.c_int, [_I64, _I64, _I64, ctypes.POINTER(Options), ctypes.POINTER(_VP)]),
    "ccsd_gpu_destroy": (None, [_VP]),
    "ccsd_gpu_last_error": (ctypes.c_char_p, [_VP]),
    "ccsd_gpu_set_precision": (ctypes.c_int, [_VP, ctypes.c_int32]),
    "ccsd_gpu_set_stream": (ctypes.c_int, [_VP, _VP]),
    "ccsd_gpu_synchronize": (ctypes.c_int, [_VP]),
    "ccsd_gpu_set_cholesky_mo": (ctypes.c_int, [_VP, _DP]),
    "ccsd_gpu_set_cholesky_mo_blocks": (ctypes.c_int, [_VP, _DP, _DP, _DP, _DP]),
    "ccsd_gpu_set_cholesky_ao": (ctypes.c_int, [_VP, _I64, _DP, _DP, _DP]),
    "ccsd_gpu_set_h_mo": (ctypes.c_int, [_VP, _DP, _DP, ctypes.c_double]),
    "ccsd_gpu_set_amplitudes": (ctypes.c_int, [_VP, _DP]),
    "ccsd_gpu_get_amplitudes": (ctypes.c_int, [_VP, _DP]),
    "ccsd_gpu_mp2_guess": (ctypes.c_int, [_VP]),
    "ccsd_gpu_get_fock": (ctypes.c_int, [_VP, _DP]),
    "ccsd_gpu_energy": (ctypes.c_int, [_VP, _DP]),
    "ccsd_gpu_omega": (ctypes.c_int, [_VP, _DP]),
    "ccsd_gpu_omega_device": (ctypes.c_int, [_VP, _VP]),
    "ccsd_gpu_jacobian": (ctypes.c_int, [_VP, _I64, _DP, _DP]),
    "ccsd_gpu_jacobian_transpose": (ctypes.c_int, [_VP, _I64, _DP, _DP]),
    "ccsd_gpu_prepare_jacobian": (ctypes.c_int, [_VP, ctypes.c_int32]),
    "ccsd_gpu_jacobian_device": (ctypes.c_int, [_VP, _I64, _VP, _VP]),
    "ccsd_gpu_jacobian_transpose_device": (ctypes.c_int, [_VP, _I64, _VP, _VP]),
    "ccsd_gpu_vjp": (ctypes.c_int, [_VP, _DP, _DP, _DP, _DP]),
    "ccsd_gpu_eom_davidson": (ctypes.c_int, [_VP, ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(DavidsonOptions), _DP,
                                             _DP, ctypes.POINTER(ctypes.c_int32)]),
    "ccsd_gpu_construct_eta": (ctypes.c_int, [_VP, _DP]),
    "ccsd_gpu_solve_multipliers": (ctypes.c_int, [_VP, ctypes.POINTER(DavidsonOptions), _DP,
                                                  ctypes.POINTER(ctypes.c_int32)]),
    "ccsd_gpu_solve_gs": (ctypes.c_int, [_VP, ctypes.POINTER(SolverOptions), _DP,
                                         ctypes.POINTER(ctypes.c_int32), _DP]),
    "ccsd_gpu_stats": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int64), _DP]),
    "ccsd_gpu_set_graphs": (ctypes.c_int, [_VP, ctypes.c_int32]),
    "ccsd_gpu_set_fp64_integrals": (ctypes.c_int, [_VP, ctypes.c_int32]),
    "ccsd_gpu_set_fp64_digits": (ctypes.c_int, [_VP, ctypes.c_int32, ctypes.c_double]),
    "ccsd_gpu_digit_gemm_profile": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int64), _DP, _DP]),
    "ccsd_gpu_set_term_timing": (ctypes.c_int, [_VP, ctypes.c_int32]),
    "ccsd_gpu_term_timing_report": (ctypes.c_int, [_VP, ctypes.c_char_p, ctypes.c_int64,
                                                   ctypes.POINTER(ctypes.c_int64)]),
    "ccsd_gpu_graph_stats": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64)]),
    "ccsd_gpu_set_profiling": (ctypes.c_int, [_VP, ctypes.c_int32]),
    "ccsd_gpu_gemm_profile": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_int64), _DP, _DP]),
    "ccsd_gpu_selftest_gemm": (ctypes.c_int, [_VP, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _I64, _I64,
                                              _I64, ctypes.c_double, _DP, _I64, _DP, _I64, ctypes.c_double, _DP,
                                              _I64]),
    "ccsd_gpu_selftest_gemm_stall": (ctypes.c_int, [_VP, _I64, _I64, _I64, _I64]),
    "ccsd_gpu_mixed_gemm_noalloc": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, _I64, _I64, _I64, ctypes.c_double,
                                                   _VP, _I64, _VP, _I64, ctypes.c_double, _VP, _I64, _VP]),
    "ccsd_gpu_omega_flops": (ctypes.c_double, [_VP]),
    "ccsd_gpu_one_electron_density": (ctypes.c_int, [_VP, _DP, _DP]),
    "ccsd_gpu_solve_gs_batch": (ctypes.c_int, [ctypes.c_int32, ctypes.POINTER(BatchSystem), ctypes.POINTER(Options),
                                               ctypes.POINTER(SolverOptions), ctypes.c_int32, _DP,
                                               ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32)]),
}


def load_library(path: str = LIB_PATH):
    """Load libccsd_gpu.so (built by et_b200/build.py); raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise CCSDGPUError(-8, f"{path} not built; run `python et_b200/build.py`")
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _dp(a):
    return a.ctypes.data_as(_DP)


def _f64(a, n=None):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1, order="F") if np.ndim(a) > 1 else a,
                             dtype=np.float64)
    if n is not None and a.size != n:
        raise ValueError(f"expected {n} values, got {a.size}")
    return a


class CCSD:
    """One Cholesky-factored closed-shell CCSD system resident on one GPU."""

    def __init__(self, n_o, n_v, n_J, *, precision=FP64, device=0, ladder_batch=0, mixed_min_flops=0,
                 mixed_k_chunk=0, autotune=0, ladder_pair_budget=0):
        self.lib = load_library()
        self.n_o, self.n_v, self.n_J = int(n_o), int(n_v), int(n_J)
        self.n_mo = self.n_o + self.n_v
        self.n_t1 = self.n_o * self.n_v
        self.n_t2 = self.n_t1 * (self.n_t1 + 1) // 2
        self.n_amp = self.n_t1 + self.n_t2
        opt = Options(device=device, precision=precision, ladder_batch=ladder_batch,
                      mixed_min_flops=mixed_min_flops, mixed_k_chunk=mixed_k_chunk, autotune=autotune,
                      ladder_pair_budget=ladder_pair_budget)
        ctx = _VP()
        rc = self.lib.ccsd_gpu_create(self.n_o, self.n_v, self.n_J, ctypes.byref(opt), ctypes.byref(ctx))
        if rc != 0:
            raise CCSDGPUError(rc, self.lib.ccsd_gpu_last_error(None).decode())
        self.ctx = ctx

    # -- plumbing --
    def _check(self, rc):
        if rc != 0:
            raise CCSDGPUError(rc, self.lib.ccsd_gpu_last_error(self.ctx).decode())

    def close(self):
        if getattr(self, "ctx", None):
            self.lib.ccsd_gpu_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_precision(self, precision):
        self._check(self.lib.ccsd_gpu_set_precision(self.ctx, precision))

    def set_stream(self, stream_handle: int):
        self._check(self.lib.ccsd_gpu_set_stream(self.ctx, _VP(stream_handle)))

    def synchronize(self):
        self._check(self.lib.ccsd_gpu_synchronize(self.ctx))

    # -- inputs --
    def set_cholesky_mo(self, L):
        """L[J, p, q] (numpy, any memory order) over the full MO range."""
        L = np.asarray(L, dtype=np.float64)
        assert L.shape == (self.n_J, self.n_mo, self.n_mo)
        flat = np.ascontiguousarray(L.reshape(-1, order="F") if not L.flags.f_contiguous else L.ravel(order="K"))
        self._check(self.lib.ccsd_gpu_set_cholesky_mo(self.ctx, _dp(flat)))

    def set_cholesky_ao(self, W_ao, S, C):
        """MO Cholesky vectors built on the device (construct_cholesky_mo_vectors): W_ao[w, x, K] =
        (wx|K) over the Cholesky basis, S[K, L] = (K|L), C[w, p] the n_mo orbital coefficients."""
        W = np.asarray(W_ao, dtype=np.float64)
        n_ao = W.shape[0]
        assert W.shape == (n_ao, n_ao, self.n_J)
        Wf = np.ascontiguousarray(W.reshape(-1, order="F"))
        Sf = _f64(np.asarray(S, dtype=np.float64).reshape(-1, order="F"), self.n_J * self.n_J)
        Cf = _f64(np.asarray(C, dtype=np.float64)[:, : self.n_mo].reshape(-1, order="F"), n_ao * self.n_mo)
        self._check(self.lib.ccsd_gpu_set_cholesky_ao(self.ctx, n_ao, _dp(Wf), _dp(Sf), _dp(Cf)))

    def set_h_mo(self, h, eps, e_hf=0.0):
        h = _f64(np.asarray(h, dtype=np.float64).reshape(-1, order="F"), self.n_mo * self.n_mo)
        eps = _f64(eps, self.n_mo)
        self._check(self.lib.ccsd_gpu_set_h_mo(self.ctx, _dp(h), _dp(eps), float(e_hf)))

    def set_system(self, L, h, eps, e_hf=0.0):
        self.set_cholesky_mo(L)
        self.set_h_mo(h, eps, e_hf)

    # -- eT wavefunction entry points --
    def set_amplitudes(self, t):
        t = _f64(t, self.n_amp)
        self._check(self.lib.ccsd_gpu_set_amplitudes(self.ctx, _dp(t)))

    def get_amplitudes(self):
        out = np.empty(self.n_amp)
        self._check(self.lib.ccsd_gpu_get_amplitudes(self.ctx, _dp(out)))
        return out

    def set_initial_amplitudes_guess(self):
        self._check(self.lib.ccsd_gpu_mp2_guess(self.ctx))

    def save_amplitudes(self, path: str, energy: float | None = None):
        """Write t in eT's amplitude-file layout (save_amplitudes_ccs, file_handling_ccs.F90:147-169),
        so eT can restart from it; the energy field is the current CCSD energy unless given."""
        from . import restart
        e = self.calculate_energy() if energy is None else energy
        restart.save_amplitudes(path, self.get_amplitudes(), restart.ccsd_blocks(self.n_o, self.n_v), e)

    def read_amplitudes(self, path: str) -> int:
        """Set t from an eT amplitude file (read_amplitudes_ccs, file_handling_ccs.F90:172-195).

        Returns the number of values read; with singles only on file the doubles are zero."""
        from . import restart
        v, _, n = restart.read_amplitudes(path, restart.ccsd_blocks(self.n_o, self.n_v))
        self.set_amplitudes(v)
        return n

    def get_fock(self):
        out = np.empty(self.n_mo * self.n_mo)
        self._check(self.lib.ccsd_gpu_get_fock(self.ctx, _dp(out)))
        return out.reshape(self.n_mo, self.n_mo, order="F")

    def calculate_energy(self) -> float:
        e = ctypes.c_double()
        self._check(self.lib.ccsd_gpu_energy(self.ctx, ctypes.byref(e)))
        return e.value

    def construct_omega(self, out=None):
        """Omega at the current amplitudes into a host array: `out` (float64, contiguous, n_amp values,
        e.g. pinned memory kept across iterations as eT keeps its omega array) or a new array."""
        if out is None:
            out = np.empty(self.n_amp)
        elif not (isinstance(out, np.ndarray) and out.dtype == np.float64 and out.flags.c_contiguous
                  and out.size == self.n_amp):
            raise ValueError(f"out must be a contiguous float64 array of {self.n_amp} values")
        self._check(self.lib.ccsd_gpu_omega(self.ctx, _dp(out)))
        return out

    def construct_omega_device(self, d_ptr: int):
        self._check(self.lib.ccsd_gpu_omega_device(self.ctx, _VP(d_ptr)))

    def jacobian_transformation(self, c):
        c = np.asarray(c, dtype=np.float64)
        n_vec = 1 if c.ndim == 1 else c.shape[1]
        flat = np.ascontiguousarray(c.reshape(-1, order="F"))
        out = np.empty(self.n_amp * n_vec)
        self._check(self.lib.ccsd_gpu_jacobian(self.ctx, n_vec, _dp(flat), _dp(out)))
        return out if c.ndim == 1 else out.reshape(self.n_amp, n_vec, order="F")

    def jacobian_transpose_transformation(self, b):
        b = np.asarray(b, dtype=np.float64)
        n_vec = 1 if b.ndim == 1 else b.shape[1]
        flat = np.ascontiguousarray(b.reshape(-1, order="F"))
        out = np.empty(self.n_amp * n_vec)
        self._check(self.lib.ccsd_gpu_jacobian_transpose(self.ctx, n_vec, _dp(flat), _dp(out)))
        return out if b.ndim == 1 else out.reshape(self.n_amp, n_vec, order="F")

    def prepare_for_jacobian(self, side: int = 0):
        """prepare_for_jacobian (side 0) / prepare_for_jacobian_transpose (side 1): record the
        residual once at the current amplitudes for the transformations that follow; side -1
        releases it.  Dropped automatically when the amplitudes, integrals or precision change."""
        self._check(self.lib.ccsd_gpu_prepare_jacobian(self.ctx, int(side)))

    def jacobian_device(self, n_vec: int, d_c: int, d_rho: int, transpose: bool = False):
        """rho = A c (or sigma = b^T A) on device pointers of (n_amp x n_vec) column blocks."""
        fn = self.lib.ccsd_gpu_jacobian_transpose_device if transpose else self.lib.ccsd_gpu_jacobian_device
        self._check(fn(self.ctx, n_vec, _VP(d_c), _VP(d_rho)))

    def vjp(self, b, *, want_L=False, want_h=False):
        """b^T dOmega/dt (no D scaling), and optionally b^T dOmega/dL_mo (J,p,q) and b^T dOmega/dh_mo."""
        b = _f64(b, self.n_amp)
        dt = np.empty(self.n_amp)
        dL = np.empty(self.n_J * self.n_mo * self.n_mo) if want_L else None
        dh = np.empty(self.n_mo * self.n_mo) if want_h else None
        self._check(self.lib.ccsd_gpu_vjp(self.ctx, _dp(b), _dp(dt), _dp(dL) if want_L else None,
                                          _dp(dh) if want_h else None))
        out = [dt]
        if want_L:
            out.append(dL.reshape(self.n_J, self.n_mo, self.n_mo, order="F"))
        if want_h:
            out.append(dh.reshape(self.n_mo, self.n_mo, order="F"))
        return out[0] if len(out) == 1 else tuple(out)

    def excited_states(self, n_states, *, left=False, max_iterations=100, block=0, max_reduced_dim=0,
                       residual_threshold=1e-6, energy_threshold=1e-6, vectors=False, start=None,
                       raise_on_failure=True):
        """eigen_davidson_solver on the device: (omegas, vectors or None, iterations).

        ``start`` ((n_amp, n_states)) seeds the trial space, e.g. with mixed-precision eigenvectors.
        With ``raise_on_failure=False`` a run that reaches ``max_iterations`` returns its current
        roots (a fixed number of refinement iterations)."""
        opt = DavidsonOptions(max_iterations=max_iterations, block=block, max_reduced_dim=max_reduced_dim,
                              residual_threshold=residual_threshold, energy_threshold=energy_threshold,
                              start_from_vectors=int(start is not None))
        om = np.zeros(n_states)
        if start is not None:
            vectors = True
            vec = np.ascontiguousarray(np.asarray(start, dtype=np.float64).reshape(-1, order="F"))
        else:
            vec = np.zeros(self.n_amp * n_states) if vectors else None
        it = ctypes.c_int32()
        rc = self.lib.ccsd_gpu_eom_davidson(self.ctx, n_states, int(bool(left)), ctypes.byref(opt), _dp(om),
                                            _dp(vec) if vectors else None, ctypes.byref(it))
        if rc != 0 and (raise_on_failure or rc != -5):
            self._check(rc)
        return om, (vec.reshape(self.n_amp, n_states, order="F") if vectors else None), it.value

    def one_electron_density(self, tbar):
        """Unrelaxed CCSD one-electron density in the MO basis (n_mo x n_mo): d(E + tbar^T Omega)/dh
        at the current amplitudes (eT: construct_gs_density_doubles, in the T1 basis)."""
        tb = _f64(tbar, self.n_amp)
        D = np.zeros(self.n_mo * self.n_mo)
        self._check(self.lib.ccsd_gpu_one_electron_density(self.ctx, _dp(tb), _dp(D)))
        return D.reshape(self.n_mo, self.n_mo, order="F")

    def construct_eta(self):
        out = np.empty(self.n_amp)
        self._check(self.lib.ccsd_gpu_construct_eta(self.ctx, _dp(out)))
        return out

    def solve_multipliers(self, *, max_iterations=100, residual_threshold=1e-6, max_reduced_dim=0):
        """A^T tbar = -eta on the device: (tbar, iterations)."""
        opt = DavidsonOptions(max_iterations=max_iterations, residual_threshold=residual_threshold,
                              max_reduced_dim=max_reduced_dim)
        out = np.empty(self.n_amp)
        it = ctypes.c_int32()
        self._check(self.lib.ccsd_gpu_solve_multipliers(self.ctx, ctypes.byref(opt), _dp(out), ctypes.byref(it)))
        return out, it.value

    def solve_ground_state(self, *, max_iterations=100, diis_dimension=8, omega_threshold=1e-5,
                           energy_threshold=1e-5, refine_threshold=1e-4, refine_target=0.0, refresh_digits=0,
                           raise_on_failure=True):
        """run_diis_cc_gs on the device; returns (energy, iterations, history[(E, |Omega|)], status).

        Mixed precision only: ``refine_threshold`` is |Omega| of the first FP64 refresh,
        ``refine_target`` the true residual the refreshes aim at (0: ``omega_threshold``),
        ``refresh_digits`` the arithmetic of the FP64 evaluations (4..7: int8 digit GEMM on the
        tensor cores, -1: cuBLAS DGEMM, 0: the library default)."""
        opt = SolverOptions(max_iterations=max_iterations, diis_dimension=diis_dimension,
                            omega_threshold=omega_threshold, energy_threshold=energy_threshold,
                            refine_threshold=refine_threshold, refine_target=refine_target,
                            refresh_digits=refresh_digits)
        e = ctypes.c_double()
        it = ctypes.c_int32()
        hist = np.zeros(2 * max_iterations)
        rc = self.lib.ccsd_gpu_solve_gs(self.ctx, ctypes.byref(opt), ctypes.byref(e), ctypes.byref(it), _dp(hist))
        if rc != 0 and (raise_on_failure or rc != -5):
            self._check(rc)
        return e.value, it.value, hist[: 2 * it.value].reshape(-1, 2), rc

    def set_graphs(self, on: bool):
        """Residual evaluations as captured CUDA graphs (off by default; CCSD_GPU_GRAPHS=1)."""
        self._check(self.lib.ccsd_gpu_set_graphs(self.ctx, 1 if on else 0))

    def set_fp64_integrals(self, resident: bool):
        """FP64 residual from resident integrals of the untransformed vectors (default, when they
        fit) or from T1-transformed integrals formed in every call (eT's omega_ccsd_a2)."""
        self._check(self.lib.ccsd_gpu_set_fp64_integrals(self.ctx, 1 if resident else 0))

    def set_fp64_digits(self, digits: int, min_flops: float = 0.0):
        """FP64 products of at least ``min_flops`` (0: 1e10) on the int8 tensor cores with 4..7
        digits per operand (0: cuBLAS DGEMM)."""
        self._check(self.lib.ccsd_gpu_set_fp64_digits(self.ctx, int(digits), float(min_flops)))

    def digit_gemm_profile(self):
        """(launches, device ms, int8 ops) of the digit GEMM since profiling was enabled."""
        n = ctypes.c_int64()
        ms = ctypes.c_double()
        ops = ctypes.c_double()
        self._check(self.lib.ccsd_gpu_digit_gemm_profile(self.ctx, ctypes.byref(n), ctypes.byref(ms),
                                                         ctypes.byref(ops)))
        return n.value, ms.value, ops.value

    def set_term_timing(self, on: bool):
        """Per-term device times under eT's timing labels; on starts a fresh log."""
        self._check(self.lib.ccsd_gpu_set_term_timing(self.ctx, 1 if on else 0))

    def term_timings(self) -> dict:
        """{eT timing label: {"calls": n, "ms": total device ms}} since set_term_timing(True)."""
        need = ctypes.c_int64()
        self._check(self.lib.ccsd_gpu_term_timing_report(self.ctx, None, 0, ctypes.byref(need)))
        buf = ctypes.create_string_buffer(int(need.value))
        self._check(self.lib.ccsd_gpu_term_timing_report(self.ctx, buf, int(need.value), ctypes.byref(need)))
        return json.loads(buf.value.decode())

    def graph_stats(self):
        """(residual evaluations served by a graph launch, GEMM routes held by the process)."""
        r, n = ctypes.c_int64(), ctypes.c_int64()
        self._check(self.lib.ccsd_gpu_graph_stats(self.ctx, ctypes.byref(r), ctypes.byref(n)))
        return int(r.value), int(n.value)

    def stats(self):
        """(kernel launches of this library, GEMM flops issued) since creation."""
        n = ctypes.c_int64()
        f = ctypes.c_double()
        self._check(self.lib.ccsd_gpu_stats(self.ctx, ctypes.byref(n), ctypes.byref(f)))
        return n.value, f.value

    def set_profiling(self, on: bool):
        self._check(self.lib.ccsd_gpu_set_profiling(self.ctx, int(bool(on))))

    def gemm_profile(self):
        """(launches, device ms, tensor flops) of the tensor-core GEMMs since profiling was enabled."""
        n = ctypes.c_int64()
        ms = ctypes.c_double()
        fl = ctypes.c_double()
        self._check(self.lib.ccsd_gpu_gemm_profile(self.ctx, ctypes.byref(n), ctypes.byref(ms), ctypes.byref(fl)))
        return n.value, ms.value, fl.value

    def selftest_gemm(self, A, B, C=None, *, alpha=1.0, beta=0.0, transA=False, transB=False, mixed=True):
        """C = alpha op(A) op(B) + beta C on the device (diagnostics of the GEMM back ends).

        ``mixed``: False/0 = FP64 DGEMM, True/1 = split-BF16 with 2 planes, 2 = with 3 planes."""
        A = np.asfortranarray(A, dtype=np.float64)
        B = np.asfortranarray(B, dtype=np.float64)
        m = A.shape[1] if transA else A.shape[0]
        k = A.shape[0] if transA else A.shape[1]
        n = B.shape[0] if transB else B.shape[1]
        Cf = np.asfortranarray(np.zeros((m, n)) if C is None else C, dtype=np.float64).copy(order="F")
        self._check(self.lib.ccsd_gpu_selftest_gemm(
            self.ctx, int(mixed), int(transA), int(transB), m, n, k, alpha, A.ctypes.data_as(_DP), A.shape[0],
            B.ctypes.data_as(_DP), B.shape[0], beta, Cf.ctypes.data_as(_DP), m))
        return Cf

    def selftest_gemm_stall(self, m=256, n=256, k=256, wait_cycles=20_000_000) -> int:
        """Failure-path diagnostics: one tensor-core GEMM whose producer withholds a pipeline stage,
        so a bounded barrier wait runs out by design.  Returns the status code (-9 when the kernel
        reported the time-out as designed) without raising."""
        return int(self.lib.ccsd_gpu_selftest_gemm_stall(self.ctx, m, n, k, wait_cycles))

    def omega_flops(self) -> float:
        return float(self.lib.ccsd_gpu_omega_flops(self.ctx))



def solve_ground_states(systems, *, precision=FP64, device=0, workers=8, max_iterations=100, diis_dimension=8,
                        omega_threshold=1e-5, energy_threshold=1e-5, refine_threshold=1e-4, refine_target=0.0,
                        mixed_min_flops=0, autotune=0, amplitudes=False):
    """Ground states of independent systems on `workers` concurrent contexts (ccsd_gpu_solve_gs_batch).

    ``systems``: sequence of (L_mo[J, p, q], h_mo, eps, n_o, e_hf) host arrays and sizes.  Each system
    starts from its MP2 guess.  Returns (energies, iterations, statuses, amplitudes or None); status
    -5 means that system did not converge within ``max_iterations``."""
    lib = load_library()
    n = len(systems)
    arr = (BatchSystem * max(n, 1))()
    keep, t_outs = [], []
    for k, (L, h, eps, n_o, e_hf) in enumerate(systems):
        L = np.asarray(L, dtype=np.float64)
        n_J, n_mo = L.shape[0], L.shape[1]
        flat = L.reshape(-1, order="F")                                   # (J, p, q), J fastest
        if not flat.flags.c_contiguous:
            flat = np.ascontiguousarray(flat)
        hf = np.ascontiguousarray(np.asarray(h, dtype=np.float64).reshape(-1, order="F"))
        ef = np.ascontiguousarray(np.asarray(eps, dtype=np.float64))
        keep += [flat, hf, ef]
        arr[k].n_o, arr[k].n_v, arr[k].n_J = int(n_o), int(n_mo - n_o), int(n_J)
        arr[k].L_mo, arr[k].h_mo, arr[k].eps = _dp(flat), _dp(hf), _dp(ef)
        arr[k].e_hf = float(e_hf)
        if amplitudes:
            n1 = int(n_o) * int(n_mo - n_o)
            t = np.zeros(n1 + n1 * (n1 + 1) // 2)
            t_outs.append(t)
            arr[k].t_out = _dp(t)
    opt = Options(device=device, precision=precision, mixed_min_flops=mixed_min_flops, autotune=autotune)
    sopt = SolverOptions(max_iterations=max_iterations, diis_dimension=diis_dimension,
                         omega_threshold=omega_threshold, energy_threshold=energy_threshold,
                         refine_threshold=refine_threshold, refine_target=refine_target)
    e = np.zeros(max(n, 1))
    it = np.zeros(max(n, 1), dtype=np.int32)
    st = np.zeros(max(n, 1), dtype=np.int32)
    rc = lib.ccsd_gpu_solve_gs_batch(n, arr, ctypes.byref(opt), ctypes.byref(sopt), int(workers), _dp(e),
                                     it.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                     st.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))
    if rc not in (0, -5):
        raise CCSDGPUError(int(rc), "batch solve failed for system %d" % int(np.flatnonzero(st[:n])[0]))
    return e[:n], it[:n], st[:n], (t_outs if amplitudes else None)
