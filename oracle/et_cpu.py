"""CPU restatement of eT's own algorithm for the CCSD residual, at the benchmark's sizes.

TEST INFRASTRUCTURE ONLY.  This is the CPU baseline that ``bench.py`` times (its ``cpu_baseline``
and its ``--impl reference`` arm); it is never imported by the product library.

eT itself cannot be built in this image (no Fortran compiler, no Libint, no system BLAS), so the
baseline restates eT's algorithm: every contraction is a BLAS call through numpy (OpenBLAS, all
host threads), and the bandwidth-bound steps eT runs as OpenMP loops (packing, squareup, the
+/- index algebra of the A2 ladder) are C + OpenMP (``oracle/et_cpu.c``).  The A2 ladder follows
``omega_ccsd_a2`` (src/wavefunctions/ccsd/omega_ccsd.F90:113-480) step by step: t+/t- once per
call, then for every (a, b) batch pair with b-batch <= a-batch the integrals g_acbd of the batch
are formed from the T1-transformed Cholesky vectors (eri_t1%get('vvvv'), one DGEMM over N_J), their
+/- combinations built, two DGEMMs against t+/t-, and the result added into the packed residual.
So the v^4 integrals are never stored (they would be 84 GB at o=32, v=320), as in eT.  The other
terms are those of ``oracle/ccsd.py`` (each cites its eT routine).

``ETSystem`` is a ``CCSDSystem`` whose residual, energy and packing use these paths, so
``oracle.ccsd.solve_gs`` runs eT's quasi-Newton + DIIS iteration on it.  Results equal the
oracle's (``tests/test_oracle_et_cpu.py``).
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

from . import ccsd as oc

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_I64 = ctypes.c_int64
_DP = ctypes.POINTER(ctypes.c_double)
_LP = ctypes.POINTER(ctypes.c_int64)


def _lib():
    global _LIB
    if _LIB is None:
        from .build import build_et_cpu
        lib = ctypes.CDLL(build_et_cpu())
        lib.et_squareup.argtypes = [_DP, _DP, _I64]
        lib.et_pack_half.argtypes = [_DP, _DP, _I64, ctypes.c_double, ctypes.c_int]
        lib.et_permute4.argtypes = [_DP, _LP, _DP, _LP, ctypes.c_double, ctypes.c_double]
        lib.et_t_pm.argtypes = [_DP, _I64, _I64, _DP, _DP]
        lib.et_g_pm_block.argtypes = [_DP, _I64, _I64, _I64, _I64, _I64, _LP, _LP, _DP, _DP]
        lib.et_add_pm.argtypes = [_DP, _DP, _DP, _I64, _I64, _I64, _LP, _LP]
        for f in (lib.et_squareup, lib.et_pack_half, lib.et_permute4, lib.et_t_pm, lib.et_g_pm_block,
                  lib.et_add_pm):
            f.restype = None
        _LIB = lib
    return _LIB


def _p(a):
    assert a.flags.c_contiguous or a.flags.f_contiguous
    return a.ctypes.data_as(_DP)


def _ip(a):
    return a.ctypes.data_as(_LP)


def squareup(t2p, n_v, n_o):
    """squareup_real (reordering.F90:4174): packed -> full t[a,i,b,j] (Fortran order)."""
    n = n_v * n_o
    full = np.empty(n * n)
    _lib().et_squareup(_p(t2p), _p(full), n)
    return full.reshape(n_v, n_o, n_v, n_o, order="F")


def pack_half(full, n_v, n_o, *, sym=False, alpha=1.0, out=None):
    """packin after scale_diagonal(1/2) (omega_ccsd.F90:100-102); with sym, of full + full^T
    (symmetric_sum, reordering.F90:416), else ``full`` must be symmetric.  Adds into ``out``."""
    n = n_v * n_o
    f = np.asfortranarray(full).reshape(-1, order="F")
    if out is None:
        out = np.zeros(n * (n + 1) // 2)
    _lib().et_pack_half(_p(f), _p(out), n, alpha, 1 if sym else 0)
    return out


def permute(x, perm):
    """Fortran-ordered y with y.shape[k] = x.shape[perm[k]], y[..] = x[permuted ..] (eT's sort_*)."""
    x = np.asarray(x, dtype=np.float64)
    assert x.ndim == 4
    if not (x.flags.c_contiguous or x.flags.f_contiguous):
        x = np.ascontiguousarray(x)
    st = np.array(x.strides, dtype=np.int64) // 8
    dims = np.array([x.shape[p] for p in perm], dtype=np.int64)
    s = np.array([st[p] for p in perm], dtype=np.int64)
    out = np.empty(int(np.prod(dims)))
    _lib().et_permute4(_p(x), _ip(s), _p(out), _ip(dims), 1.0, 0.0)
    return out.reshape(tuple(dims), order="F")


def permute3(x, perm):
    """permute() for a 3-index array (a unit fourth index)."""
    y = permute(np.asarray(x)[..., None], tuple(perm) + (3,))
    return y.reshape(y.shape[:3], order="F")


def fmm(A, B):
    """A @ B returned in Fortran order, for Fortran-ordered (or transposed C-ordered) operands:
    one BLAS call, no copies (the products of eT's dgemm calls)."""
    return (B.T @ A.T).T


def eri(Lp, Lq):
    """g_pqrs = sum_J L_pq L_rs from blocks in eT's layout (J, p, q) (eri_tool_class.F90:145-157,
    dgemm('T','N')); Fortran order (p, q, r, s)."""
    nJ = Lp.shape[0]
    g = fmm(Lp.reshape(nJ, -1, order="F").T, Lq.reshape(nJ, -1, order="F"))
    return g.reshape(Lp.shape[1], Lp.shape[2], Lq.shape[1], Lq.shape[2], order="F")


def _m(x, rows):
    """Fortran-ordered x as a (rows x rest) matrix (a view)."""
    return x.reshape(rows, -1, order="F")


def omega_a2_batched(t2p, L_vv, n_o, *, batch=None, memory=4.0e9):
    """omega_ccsd_a2 (omega_ccsd.F90:113-480), right = .true., batched over (a, b) as eT does.

    L_vv: the T1-transformed vv block (J, a, c) in eT's layout (Fortran order).  Returns the
    packed contribution.  ``batch`` is the a (and b) batch length; by default the
    largest that keeps one batch pair's integrals g_acbd (batch^2 n_v^2 doubles) within ``memory``
    bytes (eT's mem%batch_setup picks it from its memory budget).
    """
    lib = _lib()
    nJ, n_v = L_vv.shape[0], L_vv.shape[1]
    nvp, nvm = n_v * (n_v + 1) // 2, n_v * (n_v - 1) // 2
    nop, nom = n_o * (n_o + 1) // 2, n_o * (n_o - 1) // 2
    # t+ and t- once per call (construct_plus_minus_2413_from_packed, scale_double_packed_blocks)
    tp = np.empty(nop * nvp)
    tm = np.empty(max(nom * nvm, 1))
    lib.et_t_pm(_p(t2p), n_o, n_v, _p(tp), _p(tm))
    tpT = tp.reshape(nvp, nop)                   # C-order view of the column-major (nop x nvp)
    tmT = tm[: nom * nvm].reshape(nvm, nom)
    # L~_vv with rows (a, c) of one a-batch contiguous: (J, c, a) in Fortran order is (a, c, J) in C
    # order, rows a * n_v + c of length N_J
    Lv2 = permute3(L_vv, (0, 2, 1)).reshape(-1, order="F").reshape(n_v * n_v, nJ)
    if batch is None:
        batch = int(max(1, min(n_v, np.sqrt(memory / (8.0 * n_v * n_v)))))
    starts = list(range(0, n_v, batch))
    om2 = np.zeros(oc.n_t2(n_o, n_v))
    for ia, a0 in enumerate(starts):
        a1 = min(n_v, a0 + batch)
        for b0 in starts[: ia + 1]:
            b1 = min(n_v, b0 + batch)
            # eri_t1%get('vvvv', a-batch, all c, b-batch, all d): G[(a,c),(b,d)] = sum_J L_ac L_bd
            G = Lv2[a0 * n_v:a1 * n_v] @ Lv2[b0 * n_v:b1 * n_v].T
            if b0 == a0:
                pa, pb = np.tril_indices(a1 - a0)
            else:
                pa, pb = np.meshgrid(np.arange(a1 - a0), np.arange(b1 - b0), indexing="ij")
            pa = np.ascontiguousarray((pa + a0).ravel(), dtype=np.int64)
            pb = np.ascontiguousarray((pb + b0).ravel(), dtype=np.int64)
            npair = pa.size
            gp = np.empty((npair, nvp))
            gm = np.empty((npair, max(nvm, 1)))
            lib.et_g_pm_block(_p(G), n_v, a0, b0, b1 - b0, npair, _ip(pa), _ip(pb), _p(gp), _p(gm))
            del G
            # omega+-_ij,ab = 1/2 sum_cd t+-_ij,cd g+-_cd,ab (the two DGEMMs of omega_ccsd_a2)
            wpT = 0.5 * (gp @ tpT)                   # (npair x nop) = column-major (nop x npair)
            if nom > 0 and nvm > 0:
                wmT = 0.5 * (gm[:, :nvm] @ tmT)
            else:
                wmT = np.zeros((npair, max(nom, 1)))
            lib.et_add_pm(_p(om2), _p(np.ascontiguousarray(wpT)), _p(np.ascontiguousarray(wmT)), n_o, n_v, npair,
                          _ip(pa), _ip(pb))
    return om2


def t1_cholesky(L, t1):
    """construct_t1_cholesky (t1_ccs.F90:208-499) block by block, one GEMM per term as eT does.
    L: the MO blocks {'oo','ov','vo','vv'} in eT's layout (J, p, q), Fortran order."""
    nJ, n_o, n_v = L["ov"].shape
    t1 = np.asfortranarray(t1)
    Lt = {"ov": L["ov"]}
    # oo: L_ij + sum_a L_ia t_aj                                      (:251-290)
    Lt["oo"] = L["oo"] + fmm(_m(L["ov"], nJ * n_o), t1).reshape(nJ, n_o, n_o, order="F")
    # vo: L_ai + sum_b L_ab t_bi - sum_j t_aj (L_ji + sum_b L_jb t_bi)  (:293-440); the bracket is L~_oo
    vo = L["vo"] + fmm(_m(L["vv"], nJ * n_v), t1).reshape(nJ, n_v, n_o, order="F")
    x = fmm(t1, _m(permute3(Lt["oo"], (1, 0, 2)), n_o)).reshape(n_v, nJ, n_o, order="F")
    Lt["vo"] = vo - permute3(x, (1, 0, 2))
    # vv: L_ab - sum_j t_aj L_jb                                      (:443-499)
    x = fmm(t1, _m(permute3(L["ov"], (1, 0, 2)), n_o)).reshape(n_v, nJ, n_v, order="F")
    Lt["vv"] = L["vv"] - permute3(x, (1, 0, 2))
    return Lt


def fock(h_mo, Lt, t1, n_o):
    """T1 Fock F_pq = h~_pq + sum_k (2 g~_pqkk - g~_pkkq) (fock_ccsd.F90:34-78, fock_ccs.F90:242-1107)."""
    nJ = Lt["oo"].shape[0]
    F = oc.t1_transform(h_mo, t1, n_o)
    X = np.einsum("Jkk->J", Lt["oo"])
    o, v = slice(0, n_o), slice(n_o, None)
    for (rp, rq, key) in ((o, o, "oo"), (o, v, "ov"), (v, o, "vo"), (v, v, "vv")):
        F[rp, rq] += 2.0 * (X @ _m(Lt[key], nJ)).reshape(Lt[key].shape[1:], order="F")
    for (rp, rq, left, right) in ((o, o, "oo", "oo"), (o, v, "oo", "ov"), (v, o, "vo", "oo"), (v, v, "vo", "ov")):
        # - sum_Jk L~_pk L~_kq: (p, J k) x (J k, q)
        lp = permute3(Lt[left], (1, 0, 2))
        F[rp, rq] -= fmm(_m(lp, lp.shape[0]), _m(Lt[right], nJ * n_o))
    return F


def omega_et(t1, t2p, L0, Lt, F, n_o, *, batch=None):
    """construct_omega_ccsd (omega_ccsd.F90:39-110) in eT's order: singles A1/B1/C1 of the doubles
    class, E2 then symmetric_sum, B2, packing with the diagonal halved, C2/D2, and the batched A2.
    L0 / Lt: the MO / T1-transformed Cholesky blocks in eT's layout."""
    n_v = t1.shape[0]
    nov = n_v * n_o
    nJ = Lt["oo"].shape[0]
    o = slice(0, n_o)
    v = slice(n_o, None)
    om1 = np.array(F[v, o], copy=True, order="F")                     # omega_ccs_a1 (omega_ccs.F90:62)
    t = squareup(t2p, n_v, n_o)
    u = 2.0 * t - permute(t, (0, 3, 2, 1))                            # construct_u_aibj (:881-914)
    # omega_doubles_a1 (omega_doubles.F90:36-138): X_Jbi = sum_cj L_Jcj u_cjbi, sum_Jb L~_Jab X_Jbi
    X = fmm(_m(L0["vo"], nJ), _m(u, nov))                              # (J, b i)
    om1 += fmm(_m(permute3(Lt["vv"], (1, 0, 2)), n_v), X.reshape(nJ * n_v, n_o, order="F"))
    # omega_doubles_b1 (:141-204): - sum_jbk u_ajbk g_kbji
    g = eri(Lt["ov"], Lt["oo"])                                        # g[k,b,j,i]
    om1 -= fmm(_m(u, n_v), _m(permute(g, (2, 1, 0, 3)), n_o * n_v * n_o).reshape(-1, n_o, order="F"))
    # omega_doubles_c1 (:207-258): sum_bj u_aibj F_jb
    om1 += (_m(u, nov) @ np.asfortranarray(F[o, v]).T.reshape(-1, order="F")).reshape(n_v, n_o, order="F")
    # omega_ccsd_e2 (:712-878), unsymmetrised, then symmetric_sum + scale_diagonal(1/2) + packin
    g_ldkc = eri(Lt["ov"], Lt["ov"])
    u_bldk = 2.0 * permute(t, (0, 3, 2, 1)) - t
    X_bc = F[v, v] - fmm(_m(u_bldk, n_v), _m(g_ldkc, n_o * n_v * n_o).reshape(-1, n_v, order="F"))
    Y_kj = F[o, o] + fmm(_m(g_ldkc, n_o), _m(u_bldk, n_v * n_o * n_v).reshape(-1, n_o, order="F"))
    om = fmm(X_bc, _m(t, n_v)).reshape(n_v, n_o, n_v, n_o, order="F")
    om -= fmm(_m(t, n_v * n_o * n_v), Y_kj).reshape(n_v, n_o, n_v, n_o, order="F")
    om2 = pack_half(om, n_v, n_o, sym=True)
    del om, u_bldk
    # omega_ccsd_b2 (:483-583): g_aibj + sum_kl t_akbl (g_kilj + sum_cd t_cidj g_kcld)
    t_abij = permute(t, (0, 2, 1, 3))
    g_klij = permute(eri(Lt["oo"], Lt["oo"]), (0, 2, 1, 3))
    g_klcd = permute(g_ldkc, (0, 2, 1, 3))
    g_klij = g_klij + fmm(_m(g_klcd, n_o * n_o), _m(t_abij, n_v * n_v)).reshape(g_klij.shape, order="F")
    om_abij = fmm(_m(t_abij, n_v * n_v), _m(g_klij, n_o * n_o)).reshape(n_v, n_v, n_o, n_o, order="F")
    b2 = eri(Lt["vo"], Lt["vo"]) + permute(om_abij, (0, 2, 1, 3))
    pack_half(b2, n_v, n_o, out=om2)
    del b2, om_abij, t_abij, g_klcd
    om2 += _c2_d2(t, Lt, g_ldkc, n_o)                                 # omega_ccsd_c2_d2 (:586-709)
    om2 += omega_a2_batched(t2p, Lt["vv"], n_o, batch=batch)          # omega_ccsd_a2 (:113-480)
    return np.concatenate([om1.reshape(nov, order="F"), om2])


def _c2_d2(t, Lt, g_kcld, n_o):
    """omega_ccsd_c2_d2 in eT's contravariant DSYMM form (omega_ccsd.F90:586-709), as
    oracle.ccsd.omega_ccsd_c2_d2 but on eT's layouts with multi-threaded sorts and packing."""
    n_v = Lt["vv"].shape[1]
    nov = n_v * n_o

    def mat(x):
        return _m(x, nov)

    def ten(m):
        return m.reshape(n_v, n_o, n_v, n_o, order="F")

    C = permute(eri(Lt["vv"], Lt["oo"]), (1, 2, 0, 3))                # sort_1234_to_2314: C[c,k,a,j]
    D = 2.0 * permute(eri(Lt["vo"], Lt["ov"]), (3, 2, 0, 1)) - C      # add_3421_to_1234
    g = permute(g_kcld, (1, 2, 3, 0))                                 # sort_1234_to_2341: g[c,l,d,k]
    YU = mat(permute(t, (0, 3, 2, 1)))                                # construct_1432_and_contra
    YL = mat(2.0 * t) - YU
    Cm = mat(C) - 0.5 * fmm(mat(g), YU)                               # dsymm('R','U', -1/2)
    del C
    gc = 2.0 * permute(g, (0, 3, 2, 1)) - g                           # construct_full_contra_in_place
    Dm = mat(D) + 0.5 * fmm(mat(gc), YL)                              # dsymm('R','L', +1/2)
    del D, gc, g
    x = ten(-1.5 * fmm(YU, Cm))                                       # dsymm('L','U', -3/2)
    z = (x + 2.0 * permute(x, (0, 3, 2, 1))) / 3.0                    # symmetrize_and_pack (contra)
    out = pack_half(z, n_v, n_o, sym=True)
    del x, z
    x = ten(0.5 * fmm(YL, Dm))                                        # dsymm('L','L', +1/2)
    pack_half(x, n_v, n_o, sym=True, out=out)
    return out


def _blocks(L_mo, n_o):
    """The four MO blocks of L[J, p, q] in eT's layout (abstract_eri_cholesky_class.F90:290-327)."""
    o, v = slice(0, n_o), slice(n_o, None)
    return {k: np.asfortranarray(L_mo[:, a, b]) for k, a, b in (("oo", o, o), ("ov", o, v), ("vo", v, o), ("vv", v, v))}


class ETSystem(oc.CCSDSystem):
    """A CCSDSystem whose residual and energy run eT's algorithm at full size (batched A2), with the
    Cholesky vectors kept in eT's four blocks."""

    def __init__(self, L_mo, h_mo, eps, n_o, e_hf=0.0, *, batch=None):
        self.batch = batch
        self.n_o = int(n_o)
        self.L0 = _blocks(np.asarray(L_mo, dtype=np.float64), self.n_o)
        self.h_mo = np.asarray(h_mo, dtype=np.float64)
        self.eps = np.asarray(eps, dtype=np.float64)
        self.n_mo = self.h_mo.shape[0]
        self.n_v = self.n_mo - self.n_o
        self.n_J = self.L0["oo"].shape[0]
        self.e_hf = float(e_hf)
        self.n_t1 = self.n_o * self.n_v
        self.n_t2 = oc.n_t2(self.n_o, self.n_v)
        self.n_amp = self.n_t1 + self.n_t2
        self.set_amplitudes(np.zeros(self.n_amp))

    def set_amplitudes(self, amp):
        amp = np.asarray(amp)
        self.t1 = amp[: self.n_t1].reshape(self.n_v, self.n_o, order="F").copy()
        self.t2 = amp[self.n_t1:].copy()
        self.Lt = t1_cholesky(self.L0, self.t1)
        self.fock = fock(self.h_mo, self.Lt, self.t1, self.n_o)

    def omega(self, ladder="batched"):
        return omega_et(self.t1, self.t2, self.L0, self.Lt, self.fock, self.n_o, batch=self.batch)

    def energy(self):
        """calculate_energy_ccsd (mean_value_ccsd.F90:36-99):
        sum_aibj (t_aibj + t_ai t_bj)(2 g_iajb - g_ibja)."""
        nov = self.n_t1
        g = eri(self.Lt["ov"], self.Lt["ov"])                         # g[i,a,j,b]
        Lg = _m(permute(2.0 * g - permute(g, (0, 3, 2, 1)), (1, 0, 3, 2)), nov)   # as [ai, bj]
        t1 = self.t1.reshape(-1, order="F")
        e = float(np.dot(squareup(self.t2, self.n_v, self.n_o).reshape(-1, order="F"), Lg.reshape(-1, order="F")))
        return self.e_hf + e + float(t1 @ (Lg @ t1))

    def orbital_differences(self):
        """eps_ai and eps_aibj = e_a + e_b - e_i - e_j packed (doubles_class.F90:421-470)."""
        d1 = (self.eps[self.n_o:, None] - self.eps[None, :self.n_o]).reshape(-1, order="F")
        d2 = pack_half(np.add.outer(d1, d1), self.n_v, self.n_o, alpha=0.5, sym=True)
        d2[oc.diag_positions(self.n_v, self.n_o)] *= 2.0
        return np.concatenate([d1, d2])

    def mp2_start(self):
        """set_initial_amplitudes_guess_ccsd (ccsd_class.F90:357-410, 478-533) without restart."""
        self.set_amplitudes(np.zeros(self.n_amp))
        g = eri(self.Lt["vo"], self.Lt["vo"])                         # g_aibj (symmetric)
        t2 = pack_half(g, self.n_v, self.n_o)                         # packin ...
        t2[oc.diag_positions(self.n_v, self.n_o)] *= 2.0              # ... without the halved diagonal
        den = -self.orbital_differences()[self.n_t1:]
        self.set_amplitudes(np.concatenate([np.zeros(self.n_t1), t2 / den]))
