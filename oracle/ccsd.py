"""CPU restatement (FP64, numpy) of eT's Cholesky-factored CCSD hot path.

TEST INFRASTRUCTURE ONLY.  This module is the oracle that the CUDA path is
checked against; it is imported by ``tests/``, by ``__graft_entry__.smoke()``
and by the CPU-baseline leg of ``bench.py``, never by the product library.

Every function restates one eT routine (paths relative to the eT source tree)
and keeps eT's conventions:

* Cholesky vectors ``L[J, p, q]`` over the full MO range (occupied first), so
  ``g_pqrs = sum_J L[J,p,q] L[J,r,s]`` (src/eri_tool/eri_tool_class.F90:92-163).
* singles ``t1[a, i]`` (v, o); doubles upper-packed over the compound index
  ``ai = a + n_v*i`` with ``idx = M(M+1)/2 + m`` for ``M = max(ai, bj)``,
  ``m = min(ai, bj)`` (0-based form of src/tools/reordering.F90:4174-4198).
* dense 4-index arrays are indexed exactly like eT's Fortran arrays
  (``t_aibj[a, i, b, j]``); Fortran matrix views are emulated with
  ``reshape(order="F")``.

Parity of this restatement is pinned end to end against eT's committed test
outputs (tests/ccsd_gs_energy, tests/ccsd_right_es_energies): see
``tests/test_oracle_golden.py``.
"""

from __future__ import annotations

import numpy as np

# --------------------------------------------------------------------------
# packing helpers (src/tools/reordering.F90)
# --------------------------------------------------------------------------


def n_t2(n_o: int, n_v: int) -> int:
    nov = n_o * n_v
    return nov * (nov + 1) // 2


def _pair_index(n_v: int, n_o: int) -> np.ndarray:
    nov = n_v * n_o
    ai = np.arange(nov)
    big = np.maximum.outer(ai, ai)
    small = np.minimum.outer(ai, ai)
    return big * (big + 1) // 2 + small


def squareup(t2p: np.ndarray, n_v: int, n_o: int) -> np.ndarray:
    """Packed (ai>=bj) -> full symmetric t[a,i,b,j]; reordering.F90:4174 (squareup_real)."""
    idx = _pair_index(n_v, n_o)
    mat = t2p[..., idx] if t2p.ndim == 1 else None
    if mat is None:
        raise ValueError("squareup expects a 1-D packed vector")
    return mat.reshape(n_v, n_o, n_v, n_o, order="F")


def packin(full: np.ndarray, n_v: int, n_o: int) -> np.ndarray:
    """Full [a,i,b,j] -> packed lower triangle (ai>=bj); reordering.F90:4267 (packin_real)."""
    nov = n_v * n_o
    mat = full.reshape(nov, nov, order="F")
    r, c = np.tril_indices(nov)
    out = np.empty(nov * (nov + 1) // 2, dtype=full.dtype)
    out[r * (r + 1) // 2 + c] = mat[r, c]
    return out


def pack_half_diag(full: np.ndarray, n_v: int, n_o: int) -> np.ndarray:
    """packin after scale_diagonal(1/2): the packing eT applies to every Omega_2 piece.

    omega_ccsd.F90:100-102 (scale_diagonal(half) + packin), and the
    (1 - delta/2) factor of symmetrize_and_pack (packed_array_utilities_r.F90:586).
    """
    out = packin(full, n_v, n_o)
    nov = n_v * n_o
    d = np.arange(nov)
    out[d * (d + 1) // 2 + d] *= 0.5
    return out


def diag_positions(n_v: int, n_o: int) -> np.ndarray:
    """Packed positions of the doubles diagonal (ai == bj)."""
    d = np.arange(n_v * n_o)
    return d * (d + 1) // 2 + d


def scale_amplitudes(vec: np.ndarray, n_o: int, n_v: int, factor: float = 2.0) -> np.ndarray:
    """scale_amplitudes_ccsd (src/wavefunctions/ccsd/ccsd_class.F90:648-671): t2_aiai *= 2."""
    out = vec.copy()
    n_t1 = n_o * n_v
    out[n_t1 + diag_positions(n_v, n_o)] *= factor
    return out


def eri(Lp: np.ndarray, Lq: np.ndarray) -> np.ndarray:
    """g_pqrs = sum_J L^J_pq L^J_rs; eri_tool_class.F90:145-157 (dgemm 'T','N')."""
    return np.einsum("Jpq,Jrs->pqrs", Lp, Lq, optimize=True)


# --------------------------------------------------------------------------
# T1 transformation (src/wavefunctions/ccs/t1_ccs.F90)
# --------------------------------------------------------------------------


def t1_transform(Z: np.ndarray, t1: np.ndarray, n_o: int) -> np.ndarray:
    """Z <- X Z Y^T with X = I - t1, Y = I + t1^T; t1_ccs.F90:34-95."""
    n_mo = Z.shape[-1]
    X = np.eye(n_mo, dtype=np.result_type(Z, t1))
    Y = np.eye(n_mo, dtype=np.result_type(Z, t1))
    X[n_o:, :n_o] = -t1
    Y[:n_o, n_o:] = t1.T
    return X @ Z @ Y.T


def construct_t1_cholesky(L_mo: np.ndarray, t1: np.ndarray, n_o: int) -> np.ndarray:
    """Block-wise T1-transformed Cholesky vectors; t1_ccs.F90:208-499.

    oo: L_ij + sum_a L_ia t_aj                                  (:251-290)
    vo: L_ai + sum_b L_ab t_bi - sum_j t_aj (L_ji + sum_b L_jb t_bi)   (:293-440)
    vv: L_ab - sum_j t_aj L_jb                                  (:443-499)
    ov: unchanged
    """
    o = slice(0, n_o)
    v = slice(n_o, None)
    Lt = np.array(L_mo, dtype=np.result_type(L_mo, t1), copy=True)
    L_oo = L_mo[:, o, o]
    L_ov = L_mo[:, o, v]
    L_vo = L_mo[:, v, o]
    L_vv = L_mo[:, v, v]
    Lt[:, o, o] = L_oo + np.einsum("Jia,aj->Jij", L_ov, t1)
    Lp_ji = L_oo + np.einsum("Jjb,bi->Jji", L_ov, t1)
    Lt[:, v, o] = L_vo + np.einsum("Jab,bi->Jai", L_vv, t1) - np.einsum("aj,Jji->Jai", t1, Lp_ji)
    Lt[:, v, v] = L_vv - np.einsum("aj,Jjb->Jab", t1, L_ov)
    return Lt


def construct_fock(h_mo: np.ndarray, L_t1: np.ndarray, t1: np.ndarray, n_o: int) -> np.ndarray:
    """T1 Fock F_pq = h~_pq + sum_k (2 g~_pqkk - g~_pkkq); fock_ccsd.F90:34-78, fock_ccs.F90:242-1107."""
    h = t1_transform(h_mo, t1, n_o)
    X_J = np.einsum("Jkk->J", L_t1[:, :n_o, :n_o])
    coul = 2.0 * np.einsum("Jpq,J->pq", L_t1, X_J)
    exch = np.einsum("Jpk,Jkq->pq", L_t1[:, :, :n_o], L_t1[:, :n_o, :], optimize=True)
    return h + coul - exch


# --------------------------------------------------------------------------
# energy, guess, preconditioner
# --------------------------------------------------------------------------


def correlation_energy(t1: np.ndarray, t2p: np.ndarray, L_t1: np.ndarray, n_o: int) -> float:
    """sum (t_aibj + t_ai t_bj)(2 g_iajb - g_ibja); mean_value_ccsd.F90:36-99."""
    n_v = t1.shape[0]
    L_ov = L_t1[:, :n_o, n_o:]
    g_iajb = eri(L_ov, L_ov)
    t = squareup(t2p, n_v, n_o) + np.einsum("ai,bj->aibj", t1, t1)
    Lg = 2.0 * g_iajb - g_iajb.transpose(0, 3, 2, 1)   # 2 g_iajb - g_ibja
    return float(np.einsum("aibj,iajb->", t, Lg, optimize=True))


def orbital_differences(eps: np.ndarray, n_o: int) -> np.ndarray:
    """eps_ai and eps_aibj = e_a + e_b - e_i - e_j; doubles_class.F90:421-470."""
    e_o = eps[:n_o]
    e_v = eps[n_o:]
    n_v = e_v.size
    d1 = (e_v[:, None] - e_o[None, :])
    d2 = d1[:, :, None, None] + d1[None, None, :, :]
    return np.concatenate([d1.reshape(-1, order="F"), packin(d2, n_v, n_o)])


def mp2_guess(L_t1: np.ndarray, eps: np.ndarray, n_o: int) -> np.ndarray:
    """t_aibj = g_aibj / (e_i + e_j - e_a - e_b); ccsd_class.F90:478-533 (set_t2_to_cc2_guess)."""
    n_v = eps.size - n_o
    L_vo = L_t1[:, n_o:, :n_o]
    g = eri(L_vo, L_vo)
    den = -orbital_differences(eps, n_o)[n_o * n_v:]
    return packin(g, n_v, n_o) / den


# --------------------------------------------------------------------------
# Omega (src/wavefunctions/ccsd/omega_ccsd.F90 and the doubles/ccs parents)
# --------------------------------------------------------------------------


def omega_ccsd(t1, t2p, L_mo, L_t1, F, n_o, *, ladder="dense"):
    """Omega = <mu| exp(-T) H exp(T) |R>; construct_omega_ccsd, omega_ccsd.F90:39-110.

    Returns the eT vector [Omega_1 (v,o) column-major, Omega_2 packed].
    ``ladder`` selects the dense restatement of the A2 term or the literal
    +/- algorithm of omega_ccsd.F90:113-480 (identical results).
    """
    n_v = t1.shape[0]
    nov = n_v * n_o
    o = slice(0, n_o)
    v = slice(n_o, None)
    dt = np.result_type(t1, t2p, L_t1, F)

    # omega_ccs_a1 (omega_ccs.F90:62): Omega_ai += F_ai
    om1 = np.array(F[v, o], dtype=dt, copy=True)

    t = squareup(t2p, n_v, n_o)
    u = 2.0 * t - np.einsum("ajbi->aibj", t)              # construct_u_aibj, omega_ccsd.F90:881-914

    # omega_doubles_a1 (omega_doubles.F90:36-138): sum_ckd u_bicj g_abjc via L
    X_Jbi = np.einsum("Jcj,cjbi->Jbi", L_mo[:, v, o], u, optimize=True)
    om1 += np.einsum("Jab,Jbi->ai", L_t1[:, v, v], X_Jbi, optimize=True)
    # omega_doubles_b1 (omega_doubles.F90:141-204): - sum_ckl g_kbji u_ajbk
    g_kbji = eri(L_t1[:, o, v], L_t1[:, o, o])
    om1 -= np.einsum("ajbk,kbji->ai", u, g_kbji, optimize=True)
    # omega_doubles_c1 (omega_doubles.F90:207-258): sum_bj u_aibj F_jb
    om1 += np.einsum("aibj,jb->ai", u, F[o, v], optimize=True)

    # ---- doubles on the full (v,o,v,o) array ----
    om = omega_ccsd_e2(t, L_t1, F, n_o)                     # omega_ccsd.F90:712-878
    om = om + np.einsum("bjai->aibj", om)                   # symmetric_sum (reordering.F90:416)
    om += omega_ccsd_b2(t, L_t1, n_o)                       # omega_ccsd.F90:483-583 (already symmetric)
    om2 = pack_half_diag(om, n_v, n_o)                      # scale_diagonal(1/2) + packin (:100-102)

    om2 += omega_ccsd_c2_d2(t2p, L_t1, n_o)                 # omega_ccsd.F90:586-709
    if ladder == "dense":
        om2 += omega_ccsd_a2_dense(t, L_t1, n_o)            # omega_ccsd.F90:113-480
    else:
        om2 += omega_ccsd_a2_pm(t2p, L_t1, n_o)
    return np.concatenate([om1.reshape(nov, order="F"), om2])


def omega_ccsd_e2(t, L_t1, F, n_o):
    """Unsymmetrised E2 term; omega_ccsd.F90:712-878.

    E2: sum_c t_ij^ac (F_bc - sum_dkl g_ldkc u_kl^bd) - sum_k t_ik^ab (F_kj + sum_cdl g_ldkc u_lj^dc)
    """
    o = slice(0, n_o)
    v = slice(n_o, None)
    u_bldk = -t + 2.0 * np.einsum("bkdl->bldk", t)          # copy_and_scale + add_1432_to_1234
    g_ldkc = eri(L_t1[:, o, v], L_t1[:, o, v])
    X_bc = F[v, v] - np.einsum("bldk,ldkc->bc", u_bldk, g_ldkc, optimize=True)
    om = np.einsum("bc,cjai->bjai", X_bc, t, optimize=True)  # E2.1, ordered (b,j,a,i)
    Y_kj = F[o, o] + np.einsum("kdlc,dlcj->kj", g_ldkc, u_bldk, optimize=True)
    om = om - np.einsum("aibk,kj->aibj", t, Y_kj, optimize=True)   # E2.2
    return om


def omega_ccsd_b2(t, L_t1, n_o):
    """B2 = g_aibj + sum_kl t_akbl (g_kilj + sum_cd t_cidj g_kcld); omega_ccsd.F90:483-583.

    Returned in (a,i,b,j) order (eT works on the 1324-sorted array).
    """
    o = slice(0, n_o)
    v = slice(n_o, None)
    g_aibj = eri(L_t1[:, v, o], L_t1[:, v, o])
    g_klij = np.einsum("kilj->klij", eri(L_t1[:, o, o], L_t1[:, o, o]))
    g_klcd = np.einsum("kcld->klcd", eri(L_t1[:, o, v], L_t1[:, o, v]))
    t_abij = np.einsum("aibj->abij", t)
    g_klij = g_klij + np.einsum("klcd,cdij->klij", g_klcd, t_abij, optimize=True)
    om_abij = np.einsum("abkl,klij->abij", t_abij, g_klij, optimize=True)
    return g_aibj + np.einsum("abij->aibj", om_abij)


def omega_ccsd_c2_d2(t2p, L_t1, n_o):
    """C2 and D2 in eT's contravariant DSYMM form; omega_ccsd.F90:586-709.

    C2: ~Omega^ab_ij = -3/2 P(sum_ck t^bc_ki (g_kjac - 1/2 sum_dl t^ad_lj g_kdlc))
    D2:  Omega^ab_ij =  1/2 P(sum_ck u^bc_jk (L_aikc + 1/2 sum_dl u^ad_il L_ldkc))
    Returns the packed contribution.
    """
    o = slice(0, n_o)
    v = slice(n_o, None)
    n_v = L_t1.shape[1] - n_o
    nov = n_v * n_o
    t = squareup(t2p, n_v, n_o)

    def mat(x):
        return x.reshape(nov, nov, order="F")

    def ten(m):
        return m.reshape(n_v, n_o, n_v, n_o, order="F")

    g_vvoo = eri(L_t1[:, v, v], L_t1[:, o, o])
    C = np.einsum("ackj->ckaj", g_vvoo)                      # sort_1234_to_2314
    D = -C
    g_voov = eri(L_t1[:, v, o], L_t1[:, o, v])
    D = D + 2.0 * np.einsum("aikc->ckai", g_voov)            # add_3421_to_1234
    g = np.einsum("kcld->cldk", eri(L_t1[:, o, v], L_t1[:, o, v]))   # sort_1234_to_2341
    YU = mat(np.einsum("ajbi->aibj", t))                     # construct_1432_and_contra, upper
    YL = mat(2.0 * t - np.einsum("ajbi->aibj", t))           # ... lower (u)
    Cm = mat(C) - 0.5 * mat(g) @ YU                          # dsymm('R','U', -1/2)
    gc = 2.0 * np.einsum("psrq->pqrs", g) - g                # construct_full_contra_in_place(psrq)
    Dm = mat(D) + 0.5 * mat(gc) @ YL                         # dsymm('R','L', +1/2)
    x = ten(-1.5 * YU @ Cm)                                  # dsymm('L','U', -3/2)
    z = (x + 2.0 * np.einsum("psrq->pqrs", x)) / 3.0         # symmetrize_and_pack(contra, psrq)
    out = pack_half_diag(z + np.einsum("rspq->pqrs", z), n_v, n_o)
    x = ten(0.5 * YL @ Dm)                                   # dsymm('L','L', +1/2)
    out += pack_half_diag(x + np.einsum("rspq->pqrs", x), n_v, n_o)
    return out


def omega_ccsd_a2_dense(t, L_t1, n_o, *, diagonal_factor=None):
    """A2 ladder sum_cd g_acbd t^cd_ij as a dense contraction.

    Equivalent to the +/- algorithm of omega_ccsd.F90:113-480: expanding its
    t+/t-/g+/g- combinations gives sum_cd g_acbd t_cidj for every packed
    element with ai != bj and half of it on the ai == bj diagonal, i.e.
    pack_half_diag of the full contraction.  ``diagonal_factor`` scales the
    t diagonal first (the right-hand Jacobian call, jacobian_ccsd.F90:174).
    """
    n_v = L_t1.shape[1] - n_o
    v = slice(n_o, None)
    if diagonal_factor is not None:
        t = t.copy()
        a = np.arange(n_v)[:, None]
        i = np.arange(n_o)[None, :]
        t[a, i, a, i] *= diagonal_factor
    g_vvvv = eri(L_t1[:, v, v], L_t1[:, v, v])
    full = np.einsum("acbd,cidj->aibj", g_vvvv, t, optimize=True)
    return pack_half_diag(full, n_v, n_o)


def omega_ccsd_a2_pm(t2p, L_t1, n_o):
    """Literal single-batch +/- algorithm of omega_ccsd.F90:113-480 (right=.true.).

    t+_{ij,cd} = (1-d_cd/2)(1-d_ij/2)(t_cidj + t_cjdi), t-_{ij,cd} = t_cidj - t_cjdi
    g+-_{cd,ab} = g_acbd +- g_adbc; omega+-_{ij,ab} = 1/2 sum t+- g+-,
    omega+ diagonal (a=b) scaled by 1/2, then added with add_double_packed_plus_minus.
    """
    n_v = L_t1.shape[1] - n_o
    v = slice(n_o, None)
    t = squareup(t2p, n_v, n_o)
    g = eri(L_t1[:, v, v], L_t1[:, v, v])               # g[a,c,b,d]
    ip, jp = np.tril_indices(n_o)                         # i >= j
    cp, dp = np.tril_indices(n_v)                         # c >= d
    im, jm = np.tril_indices(n_o, -1)
    cm, dm = np.tril_indices(n_v, -1)
    t_p = t[cp[None, :], ip[:, None], dp[None, :], jp[:, None]] + t[cp[None, :], jp[:, None], dp[None, :], ip[:, None]]
    t_p = t_p * np.where(cp == dp, 0.5, 1.0)[None, :] * np.where(ip == jp, 0.5, 1.0)[:, None]
    t_m = t[cm[None, :], im[:, None], dm[None, :], jm[:, None]] - t[cm[None, :], jm[:, None], dm[None, :], im[:, None]]
    ap, bp = cp, dp                                       # a >= b uses the same triangle
    am, bm = cm, dm
    g_p = g[ap[None, :], cp[:, None], bp[None, :], dp[:, None]] + g[ap[None, :], dp[:, None], bp[None, :], cp[:, None]]
    g_m = g[am[None, :], cm[:, None], bm[None, :], dm[:, None]] - g[am[None, :], dm[:, None], bm[None, :], cm[:, None]]
    om_p = 0.5 * t_p @ g_p                                # (ij_p, ab_p)
    om_m = 0.5 * t_m @ g_m
    om_p = om_p * np.where(ap == bp, 0.5, 1.0)[None, :]
    full = np.zeros((n_v, n_o, n_v, n_o), dtype=om_p.dtype)
    # add_double_packed_plus_minus: x(a i b j) += w+ + w-, x(a j b i) += w+ - w-
    # (for i == j or a == b only w+ is added, to both positions)
    res = np.zeros(n_t2(n_o, n_v), dtype=om_p.dtype)
    mi = {(int(a), int(b)): k for k, (a, b) in enumerate(zip(im, jm))}
    ma = {(int(a), int(b)): k for k, (a, b) in enumerate(zip(am, bm))}
    for kij, (i, j) in enumerate(zip(ip, jp)):
        for kab, (a, b) in enumerate(zip(ap, bp)):
            wp = om_p[kij, kab]
            if i != j and a != b:
                wm = om_m[mi[(int(i), int(j))], ma[(int(a), int(b))]]
                x1, x2 = wp + wm, wp - wm
            else:
                x1 = x2 = wp
            for (aa, ii, bb, jj, val) in ((a, i, b, j, x1), (a, j, b, i, x2)):
                p = aa + n_v * ii
                q = bb + n_v * jj
                big, small = max(p, q), min(p, q)
                res[big * (big + 1) // 2 + small] += val
    del full
    return res


# --------------------------------------------------------------------------
# the system object: an eT ccsd wavefunction restricted to the hot path
# --------------------------------------------------------------------------


class CCSDSystem:
    """Holds L_mo, h_mo, orbital energies and amplitudes; mirrors the ccsd TBPs used by the solvers."""

    def __init__(self, L_mo, h_mo, eps, n_o, e_hf=0.0):
        self.L_mo = np.asarray(L_mo, dtype=np.float64)
        self.h_mo = np.asarray(h_mo, dtype=np.float64)
        self.eps = np.asarray(eps, dtype=np.float64)
        self.n_o = int(n_o)
        self.n_mo = self.h_mo.shape[0]
        self.n_v = self.n_mo - self.n_o
        self.n_J = self.L_mo.shape[0]
        self.e_hf = float(e_hf)
        self.n_t1 = self.n_o * self.n_v
        self.n_t2 = n_t2(self.n_o, self.n_v)
        self.n_amp = self.n_t1 + self.n_t2
        self.set_amplitudes(np.zeros(self.n_amp))

    # ccs_class / ccsd set_amplitudes + construct_t1_cholesky + construct_fock
    def set_amplitudes(self, amp):
        amp = np.asarray(amp)
        self.t1 = amp[: self.n_t1].reshape(self.n_v, self.n_o, order="F").copy()
        self.t2 = amp[self.n_t1:].copy()
        self.L_t1 = construct_t1_cholesky(self.L_mo, self.t1, self.n_o)
        self.fock = construct_fock(self.h_mo, self.L_t1, self.t1, self.n_o)

    def get_amplitudes(self):
        return np.concatenate([self.t1.reshape(-1, order="F"), self.t2])

    def mp2_start(self):
        """set_initial_amplitudes_guess_ccsd (ccsd_class.F90:357-410) without restart."""
        self.set_amplitudes(np.zeros(self.n_amp))
        t2 = mp2_guess(self.L_t1, self.eps, self.n_o)
        self.set_amplitudes(np.concatenate([np.zeros(self.n_t1), t2]))

    def energy(self):
        return self.e_hf + correlation_energy(self.t1, self.t2, self.L_t1, self.n_o)

    def omega(self, ladder="dense"):
        return omega_ccsd(self.t1, self.t2, self.L_mo, self.L_t1, self.fock, self.n_o, ladder=ladder)

    def omega_at(self, amp):
        """Omega as a pure function of the amplitude vector (real or complex)."""
        amp = np.asarray(amp)
        t1 = amp[: self.n_t1].reshape(self.n_v, self.n_o, order="F")
        t2 = amp[self.n_t1:]
        L_t1 = construct_t1_cholesky(self.L_mo, t1, self.n_o)
        F = construct_fock(self.h_mo, L_t1, t1, self.n_o)
        return omega_ccsd(t1, t2, self.L_mo, L_t1, F, self.n_o)

    def orbital_differences(self):
        return orbital_differences(self.eps, self.n_o)

    # ---- Jacobian and its transpose ----
    def diag_scaling(self):
        """D = 1 except 2 on the packed doubles diagonal: rho = (dOmega/dt) D c.

        jacobian_ccsd.F90:74-176 documents rho_mu = sum A_mu,ck c_ck +
        1/2 sum A_mu,ckdl c_ckdl (1 + delta_ck,dl); with Omega a function of
        the packed amplitudes this is the directional derivative along the
        vector c whose doubles diagonal is doubled (scale_diagonal(two, c_aibj)
        at :122-123 and diagonal_factor=two in the A2 call at :174).
        """
        d = np.ones(self.n_amp)
        d[self.n_t1 + diag_positions(self.n_v, self.n_o)] = 2.0
        return d

    def jacobian_transformation(self, c, h=1e-30):
        """rho = A c by complex-step differentiation of omega_at (exact to rounding)."""
        amp = self.get_amplitudes().astype(np.complex128)
        dc = np.asarray(c, dtype=np.float64) * self.diag_scaling()
        return np.imag(self.omega_at(amp + 1j * h * dc)) / h

    def jacobian_matrix(self):
        """Dense A (small systems only)."""
        n = self.n_amp
        A = np.empty((n, n))
        for k in range(n):
            e = np.zeros(n)
            e[k] = 1.0
            A[:, k] = self.jacobian_transformation(e)
        return A


def one_electron_density(sysm, tbar, h=1e-30):
    """Unrelaxed CCSD one-electron density in the MO basis of h:
    D_pq = d(E + tbar^T Omega)/dh_pq at fixed amplitudes and orbitals.

    eT forms the same density in the T1 basis (construct_gs_density_doubles,
    src/wavefunctions/doubles/mean_value_doubles.F90:78-114: D = <Lambda| E_pq |CC>); with
    h~ = (1 - t1) h (1 + t1) the two are related by D_T1 = (1 + t1^T) D (1 - t1^T).  The energy
    depends on h through the reference (2 on the occupied diagonal) and through the singles term
    2 sum_ai F_ia t_ai (F_ia = h_ia + ...; it vanishes at a Hartree-Fock reference but not its
    derivative); tbar^T dOmega/dh is taken by complex-step differentiation."""
    n_o, n_v = sysm.n_o, sysm.n_v
    n = n_o + n_v
    D = np.zeros((n, n))
    D[:n_o, :n_o] += 2.0 * np.eye(n_o)
    D[:n_o, n_o:] += 2.0 * sysm.t1.T
    L_t1 = construct_t1_cholesky(sysm.L_mo, sysm.t1, n_o)
    for p in range(n):
        for q in range(n):
            hc = sysm.h_mo.astype(np.complex128)
            hc[p, q] += 1j * h
            F = construct_fock(hc, L_t1, sysm.t1, n_o)
            om = omega_ccsd(sysm.t1, sysm.t2, sysm.L_mo, L_t1, F, n_o)
            D[p, q] += tbar @ (np.imag(om) / h)
    return D


def construct_eta(F, L_t1, n_o):
    """eta = [2 F_ia ; pack(4 g_iajb - 2 g_ibja)]; construct_eta_ccsd, multiplier_equation_ccsd.F90:50-113."""
    n_v = F.shape[0] - n_o
    eta1 = 2.0 * F[:n_o, n_o:].T                                  # eta_ai = 2 F_ia
    L_ov = L_t1[:, :n_o, n_o:]
    g = eri(L_ov, L_ov)                                            # g[i,a,j,b]
    eta2 = 4.0 * np.einsum("iajb->aibj", g) - 2.0 * np.einsum("ibja->aibj", g)
    return np.concatenate([eta1.reshape(-1, order="F"), packin(eta2, n_v, n_o)])


def multiplier_guess(t1, t2p, n_o):
    """t1bar = t1, t2bar = 2 t_aibj - t_ajbi packed (set_initial_multipliers_guess_ccsd, ccsd_class.F90:411-475)."""
    n_v = t1.shape[0]
    t = squareup(t2p, n_v, n_o)
    return np.concatenate([t1.reshape(-1, order="F"), packin(2.0 * t - np.einsum("ajbi->aibj", t), n_v, n_o)])


# --------------------------------------------------------------------------
# solvers: quasi-Newton + DIIS ground state (src/solvers/cc/diis_cc_gs_class.F90)
# --------------------------------------------------------------------------


class DIIS:
    """diis_tool (src/solver_tools/diis_tool_class.F90:302-640), records in memory."""

    def __init__(self, dimension=8):
        self.dimension = dimension
        self.errors: list[np.ndarray] = []
        self.params: list[np.ndarray] = []
        self.G = np.zeros((0, 0))

    def update(self, e, x):
        if len(self.errors) == self.dimension:
            self.errors.pop(0)
            self.params.pop(0)
            self.G = self.G[1:, 1:]
        self.errors.append(e.copy())
        self.params.append(x.copy())
        n = len(self.errors)
        G = np.zeros((n, n))
        G[: n - 1, : n - 1] = self.G
        for k in range(n):
            G[n - 1, k] = G[k, n - 1] = float(np.dot(e, self.errors[k]))
        self.G = G
        P = np.zeros((n + 1, n + 1))
        P[:n, :n] = G
        P[n, :n] = -1.0
        P[:n, n] = -1.0
        H = np.zeros(n + 1)
        H[n] = -1.0
        w = np.linalg.solve(P, H)[:n]                 # dgesv (diis_tool_class.F90:621)
        return sum(wk * pk for wk, pk in zip(w, self.params))


def solve_gs(system: CCSDSystem, *, max_iterations=100, omega_threshold=1e-10,
             energy_threshold=1e-10, diis_dimension=8, history=None):
    """run_diis_cc_gs (diis_cc_gs_class.F90:209-315) with the quasi-Newton updater.

    Returns (energy, iterations, converged); appends (E, |Omega|) per iteration to ``history``.
    """
    diis = DIIS(diis_dimension)
    previous = 0.0
    eps = system.orbital_differences()
    for it in range(1, max_iterations + 1):
        energy = system.energy()
        omega = system.omega()
        norm = float(np.linalg.norm(omega))
        if history is not None:
            history.append((energy, norm))
        # convergence_tool: residual and (when requested) energy change
        if norm < omega_threshold and abs(energy - previous) < energy_threshold:
            return energy, it, True
        amp = system.get_amplitudes()
        residual = -omega / eps                          # quasi_newton_updater_class.F90
        update = scale_amplitudes(residual, system.n_o, system.n_v)
        amp = amp + update                               # amplitude_updater_class.F90
        residual = scale_amplitudes(residual, system.n_o, system.n_v)
        amp = diis.update(residual, amp)
        system.set_amplitudes(amp)
        previous = energy
    return system.energy(), max_iterations, False


def davidson_right(system: CCSDSystem, n_states, *, max_iterations=100, threshold=1e-10,
                   max_dim=None):
    """Lowest right eigenpairs of A (eigen_davidson_solver_class.F90:122-229, restated).

    Plain non-symmetric Davidson with the orbital-difference preconditioner;
    the reduced problem is solved with numpy's geev.
    """
    n = system.n_amp
    eps = system.orbital_differences()
    order = np.argsort(eps)
    V = np.zeros((n, 0))
    AV = np.zeros((n, 0))
    guesses = []
    for k in range(n_states):
        e = np.zeros(n)
        e[order[k]] = 1.0
        guesses.append(e)
    max_dim = max_dim or max(100, 10 * n_states)
    omegas = None
    new = guesses
    for it in range(max_iterations):
        for vec in new:
            vec = vec - V @ (V.T @ vec)
            vec = vec - V @ (V.T @ vec)
            nrm = np.linalg.norm(vec)
            if nrm < 1e-12:
                continue
            vec = vec / nrm
            V = np.column_stack([V, vec])
            AV = np.column_stack([AV, system.jacobian_transformation(vec)])
        red = V.T @ AV
        w, s = np.linalg.eig(red)
        idx = np.argsort(w.real)[:n_states]
        omegas = w.real[idx]
        X = V @ s[:, idx].real
        R = AV @ s[:, idx].real - X * omegas
        norms = np.linalg.norm(R, axis=0)
        if np.all(norms < threshold):
            return omegas, X, it + 1
        new = []
        for k in range(n_states):
            if norms[k] >= threshold:
                den = omegas[k] - eps
                den = np.where(np.abs(den) < 1e-8, 1e-8, den)
                new.append(R[:, k] / den)
        if V.shape[1] + len(new) > max_dim:
            V = X / np.linalg.norm(X, axis=0)
            V, _ = np.linalg.qr(V)
            AV = np.column_stack([system.jacobian_transformation(V[:, k]) for k in range(V.shape[1])])
    return omegas, None, max_iterations
