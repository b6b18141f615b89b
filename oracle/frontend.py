"""Molecular front end for the oracle: basis -> AO integrals -> RHF -> Cholesky -> MO vectors.

TEST INFRASTRUCTURE ONLY.  eT builds the MO Cholesky vectors that feed the
CCSD hot path from Libint integrals, an RHF reference and a pivoted Cholesky
decomposition of the AO ERI matrix (src/solvers/cholesky/eri_cd_class.F90,
construct_cholesky_mo_vectors at :3132).  This module restates that chain for
small molecules (s, p, d shells; spherical d) so the CPU oracle can be pinned
against eT's committed test outputs.  The AO integrals come from the
McMurchie-Davidson code in ``integrals.c`` (built into ``oracle/_lib`` by
``oracle/build.py``).
"""

from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BOHR_PER_ANGSTROM = 1.0 / 0.52917721092      # the conversion eT prints (tests/*/result/*.out)
CHARGES = {"H": 1, "He": 2, "Li": 3, "Be": 4, "B": 5, "C": 6, "N": 7, "O": 8, "F": 9, "Ne": 10}
L_OF = {"S": 0, "P": 1, "D": 2}


def _lib():
    path = os.path.join(HERE, "_lib", "libintegrals.so")
    if not os.path.exists(path):
        from oracle.build import build_oracle
        build_oracle()
    lib = ctypes.CDLL(path)
    dp = ctypes.POINTER(ctypes.c_double)
    ip = ctypes.POINTER(ctypes.c_int)
    lib.one_electron.argtypes = [ctypes.c_int, ip, dp, dp, ctypes.c_int, dp, dp, dp, dp, dp]
    lib.dipole.argtypes = [ctypes.c_int, ip, dp, dp, dp, dp, dp, dp]
    lib.eri_all.argtypes = [ctypes.c_int, ip, dp, dp, dp]
    return lib


def parse_g94(text: str, elements) -> dict:
    """Contracted shells per element from a Gaussian-94 basis file: {el: [(l, [(alpha, c)])]}."""
    out = {}
    lines = [ln.strip() for ln in text.splitlines()]
    i = 0
    while i < len(lines):
        tok = lines[i].split()
        if len(tok) == 2 and tok[0] in elements and tok[1] == "0":
            el = tok[0]
            shells = []
            i += 1
            while not lines[i].startswith("****"):
                head = lines[i].split()
                kind, nprim = head[0].upper(), int(head[1])
                rows = [lines[i + 1 + k].replace("D", "E").split() for k in range(nprim)]
                if kind == "SP":
                    # an s and a p shell sharing exponents (s first, as the basis lists them)
                    shells.append((0, [(float(r[0]), float(r[1])) for r in rows]))
                    shells.append((1, [(float(r[0]), float(r[2])) for r in rows]))
                else:
                    shells.append((L_OF[kind], [(float(r[0]), float(r[1])) for r in rows]))
                i += nprim + 1
            out[el] = shells
        i += 1
    return out


def _dfact(n):
    r = 1.0
    while n > 1:
        r *= n
        n -= 2
    return r


_SPH_D = np.array([[0, 1, 0, 0, 0, 0],       # xy
                   [0, 0, 0, 0, 1, 0],       # yz
                   [-1, 0, 0, -1, 0, 2],     # 2zz - xx - yy
                   [0, 0, 1, 0, 0, 0],       # xz
                   [1, 0, 0, -1, 0, 0]],     # xx - yy
                  dtype=float)


@dataclass
class Molecule:
    symbols: list
    coords_bohr: np.ndarray      # (natom, 3)

    @property
    def charges(self):
        return np.array([CHARGES[s] for s in self.symbols], dtype=float)

    def nuclear_repulsion(self):
        Z = self.charges
        e = 0.0
        for a in range(len(Z)):
            for b in range(a):
                e += Z[a] * Z[b] / np.linalg.norm(self.coords_bohr[a] - self.coords_bohr[b])
        return e


def molecule_from_angstrom(symbols, coords):
    return Molecule(list(symbols), np.asarray(coords, dtype=float) * BOHR_PER_ANGSTROM)


def _contracted(mol: Molecule, basis: dict):
    """Primitive Cartesian shells and the (unnormalised) map T from them to the contracted spherical AOs."""
    prim_l, prim_a, prim_c = [], [], []
    rows = []          # contracted spherical AO -> list of (prim cart index, coefficient)
    ncart_off = 0
    for atom, el in enumerate(mol.symbols):
        for l, prims in basis[el]:
            nc = (l + 1) * (l + 2) // 2
            offs = []
            for a, c in prims:
                prim_l.append(l)
                prim_a.append(a)
                prim_c.append(mol.coords_bohr[atom])
                offs.append((ncart_off, a, c))
                ncart_off += nc
            if l == 0:
                sph = np.ones((1, 1))
            elif l == 1:
                sph = np.eye(3)
            else:
                sph = _SPH_D
            for m in range(sph.shape[0]):
                row = {}
                for off, a, c in offs:
                    norm = (2 * a / np.pi) ** 0.75 * (4 * a) ** (l / 2) / np.sqrt(_dfact(2 * l - 1))
                    for k in range(nc):
                        if sph[m, k] != 0.0:
                            row[off + k] = row.get(off + k, 0.0) + c * norm * sph[m, k]
                rows.append(row)
    T = np.zeros((len(rows), ncart_off))
    for r, row in enumerate(rows):
        for k, val in row.items():
            T[r, k] = val
    return (np.array(prim_l, dtype=np.int32), np.array(prim_a, dtype=np.float64),
            np.ascontiguousarray(np.array(prim_c, dtype=np.float64)), T)


def ao_dipole(mol: Molecule, basis: dict, origin=(0.0, 0.0, 0.0)):
    """<mu| r - origin |nu> over the normalised contracted AOs of ao_integrals: array (3, n_ao, n_ao), bohr."""
    l_arr, a_arr, c_arr, T = _contracted(mol, basis)
    n_prim = T.shape[1]
    lib = _lib()
    dp = ctypes.POINTER(ctypes.c_double)
    ip = ctypes.POINTER(ctypes.c_int)
    S = np.zeros((n_prim, n_prim))
    Tk = np.zeros((n_prim, n_prim))
    V = np.zeros((n_prim, n_prim))
    Z = np.zeros(1)
    cpos = np.zeros(3)
    lib.one_electron(len(l_arr), l_arr.ctypes.data_as(ip), a_arr.ctypes.data_as(dp), c_arr.ctypes.data_as(dp),
                     0, Z.ctypes.data_as(dp), cpos.ctypes.data_as(dp), S.ctypes.data_as(dp), Tk.ctypes.data_as(dp),
                     V.ctypes.data_as(dp))
    M = [np.zeros((n_prim, n_prim)) for _ in range(3)]
    o = np.ascontiguousarray(np.asarray(origin, dtype=np.float64))
    lib.dipole(len(l_arr), l_arr.ctypes.data_as(ip), a_arr.ctypes.data_as(dp), c_arr.ctypes.data_as(dp),
               o.ctypes.data_as(dp), M[0].ctypes.data_as(dp), M[1].ctypes.data_as(dp), M[2].ctypes.data_as(dp))
    nrm = 1.0 / np.sqrt(np.diag(T @ S @ T.T))
    Tn = T * nrm[:, None]
    return np.stack([Tn @ m @ Tn.T for m in M])


def ao_integrals(mol: Molecule, basis: dict):
    """S, T, V and the AO ERI tensor over spherical, normalised contracted functions."""
    l_arr, a_arr, c_arr, T = _contracted(mol, basis)
    n_prim = T.shape[1]
    lib = _lib()
    nsh = len(l_arr)
    dp = ctypes.POINTER(ctypes.c_double)
    ip = ctypes.POINTER(ctypes.c_int)
    S = np.zeros((n_prim, n_prim))
    Tk = np.zeros((n_prim, n_prim))
    V = np.zeros((n_prim, n_prim))
    Z = mol.charges
    cpos = np.ascontiguousarray(mol.coords_bohr)
    lib.one_electron(nsh, l_arr.ctypes.data_as(ip), a_arr.ctypes.data_as(dp), c_arr.ctypes.data_as(dp),
                     len(Z), Z.ctypes.data_as(dp), cpos.ctypes.data_as(dp),
                     S.ctypes.data_as(dp), Tk.ctypes.data_as(dp), V.ctypes.data_as(dp))
    eri_p = np.zeros((n_prim,) * 4)
    lib.eri_all(nsh, l_arr.ctypes.data_as(ip), a_arr.ctypes.data_as(dp), c_arr.ctypes.data_as(dp),
                eri_p.ctypes.data_as(dp))
    S = T @ S @ T.T
    nrm = 1.0 / np.sqrt(np.diag(S))
    T = T * nrm[:, None]
    S = S * np.outer(nrm, nrm)
    Tk = T @ Tk @ T.T
    V = T @ V @ T.T
    eri = np.einsum("pi,qj,rk,sl,ijkl->pqrs", T, T, T, T, eri_p, optimize=True)
    return S, Tk, V, eri


def rhf(S, H, eri, n_occ, e_nuc, *, conv=1e-12, max_iter=200):
    """Closed-shell RHF with DIIS; returns (E_HF, C, eps)."""
    s, U = np.linalg.eigh(S)
    X = U / np.sqrt(s)
    F = H
    e, Cp = np.linalg.eigh(X.T @ F @ X)
    C = X @ Cp
    errs, focks = [], []
    e_old = 0.0
    for it in range(max_iter):
        D = C[:, :n_occ] @ C[:, :n_occ].T
        J = np.einsum("pqrs,rs->pq", eri, D)
        K = np.einsum("prqs,rs->pq", eri, D)
        F = H + 2 * J - K
        E = float(np.sum(D * (H + F))) + e_nuc
        err = F @ D @ S - S @ D @ F
        errs.append(err)
        focks.append(F)
        if len(errs) > 8:
            errs.pop(0)
            focks.pop(0)
        if np.abs(err).max() < conv and abs(E - e_old) < conv * 1e-2:
            break
        e_old = E
        n = len(errs)
        B = -np.ones((n + 1, n + 1))
        B[n, n] = 0.0
        for i in range(n):
            for j in range(n):
                B[i, j] = np.sum(errs[i] * errs[j])
        rhs = np.zeros(n + 1)
        rhs[n] = -1.0
        w = np.linalg.solve(B, rhs)[:n]
        Fd = sum(wi * fi for wi, fi in zip(w, focks))
        e, Cp = np.linalg.eigh(X.T @ Fd @ X)
        C = X @ Cp
    D = C[:, :n_occ] @ C[:, :n_occ].T
    J = np.einsum("pqrs,rs->pq", eri, D)
    K = np.einsum("prqs,rs->pq", eri, D)
    F = H + 2 * J - K
    e, Cp = np.linalg.eigh(X.T @ F @ X)
    C = X @ Cp
    D = C[:, :n_occ] @ C[:, :n_occ].T
    E = float(np.sum(D * (H + F))) + e_nuc
    return E, C, e


def pivoted_cholesky(eri, threshold, pivots=False):
    """Pivoted Cholesky of the (n^2 x n^2) ERI matrix: returns L[J, mu, nu] (and, with pivots=True,
    the pivot pairs as indices of the flattened (mu, nu) index, in selection order)."""
    n = eri.shape[0]
    M = eri.reshape(n * n, n * n)
    diag = np.diag(M).copy()
    vecs, piv = [], []
    while True:
        p = int(np.argmax(diag))
        if diag[p] <= threshold:
            break
        piv.append(p)
        col = M[:, p].copy()
        for v in vecs:
            col -= v * v[p]
        v = col / np.sqrt(diag[p])
        vecs.append(v)
        diag -= v * v
        diag[p] = 0.0
    L = np.array(vecs).reshape(len(vecs), n, n)
    return (L, np.array(piv)) if pivots else L


def build_system(symbols, coords_angstrom, basis, *, cd_threshold=1e-12):
    """Full chain for a neutral closed-shell molecule; returns a dict of MO quantities.

    ``basis`` is either Gaussian-94 text or an already parsed {element: shells} dict.
    """
    mol = molecule_from_angstrom(symbols, coords_angstrom)
    if isinstance(basis, str):
        basis = parse_g94(basis, set(symbols))
    S, Tk, V, eri = ao_integrals(mol, basis)
    n_el = int(round(mol.charges.sum()))
    n_o = n_el // 2
    e_nuc = mol.nuclear_repulsion()
    E_hf, C, eps = rhf(S, Tk + V, eri, n_o, e_nuc)
    L_ao = pivoted_cholesky(eri, cd_threshold)
    L_mo = np.einsum("mp,Jmn,nq->Jpq", C, L_ao, C, optimize=True)
    h_mo = C.T @ (Tk + V) @ C
    return dict(L_mo=L_mo, h_mo=h_mo, eps=eps, n_o=n_o, e_hf=E_hf, e_nuc=e_nuc)


GOLDEN = os.path.join(os.path.dirname(HERE), "tests", "golden")


def golden_values() -> dict:
    import json
    with open(os.path.join(GOLDEN, "et_reference_values.json")) as f:
        return json.load(f)


def golden_basis(name: str = "cc-pvdz") -> dict:
    import json
    with open(os.path.join(GOLDEN, f"basis_{name}.json")) as f:
        shells = json.load(f)["shells"]
    return {el: [(int(l), [tuple(p) for p in prims]) for l, prims in sh] for el, sh in shells.items()}


def et_test_system(name: str, cd_threshold=None):
    """MO data of one of eT's committed regression molecules (from the golden fixtures)."""
    v = golden_values()[name]
    sym = [a[0] for a in v["atoms"]]
    xyz = [a[1:] for a in v["atoms"]]
    thr = v["cd_threshold"] if cd_threshold is None else cd_threshold
    return build_system(sym, xyz, golden_basis(), cd_threshold=thr)


def et_restart_system() -> dict:
    """eT's H2O+He/cc-pVDZ restart test (tests/restart_ccsd_v1.0) in eT's own MO basis.

    The MO coefficients come from the restart files eT wrote, so L_mo and h_mo are expressed in
    exactly the orbitals of eT's amplitudes; the Cholesky threshold is the test's 1e-12.  Also
    returns eT's converged t, multipliers tbar, right/left EOM vectors r, l (rows) and the
    excitation energies omega."""
    v = golden_values()["restart_ccsd_v1.0"]
    z = np.load(os.path.join(GOLDEN, "et_restart_h2o_he.npz"))
    mol = molecule_from_angstrom([a[0] for a in v["atoms"]], [a[1:] for a in v["atoms"]])
    S, Tk, V, eri = ao_integrals(mol, golden_basis())
    C = z["C"]
    n_o = int(z["n_o"])
    L_ao = pivoted_cholesky(eri, v["cd_threshold"])
    L_mo = np.einsum("mp,Jmn,nq->Jpq", C, L_ao, C, optimize=True)
    h_mo = C.T @ (Tk + V) @ C
    L_oo = L_mo[:, :n_o, :n_o]
    fock_oo = (h_mo[:n_o, :n_o] + 2.0 * np.einsum("Jpq,Jkk->pq", L_oo, L_oo)
               - np.einsum("Jpk,Jkq->pq", L_oo, L_oo))
    e_nuc = mol.nuclear_repulsion()
    e_hf = e_nuc + float(np.trace(h_mo[:n_o, :n_o]) + np.trace(fock_oo))
    return dict(L_mo=L_mo, h_mo=h_mo, eps=z["eps"].copy(), n_o=n_o, e_hf=e_hf, e_nuc=e_nuc, C=C, S=S,
                t=z["t"].copy(), tbar=z["tbar"].copy(), r=z["r"].copy(), l=z["l"].copy(),
                omega=z["omega"].copy(), e_ccsd=v["e_ccsd"])


def et_dipole_system() -> dict:
    """eT's tests/ccsd_dipole molecule (H2O and He, STO-3G, Cholesky threshold 1e-11): MO data plus
    the dipole integrals <p| r |q> in the MO basis (origin 0, bohr) and the nuclear dipole."""
    v = golden_values()["ccsd_dipole"]
    sym = [a[0] for a in v["atoms"]]
    xyz = [a[1:] for a in v["atoms"]]
    basis = golden_basis(v["basis"])
    mol = molecule_from_angstrom(sym, xyz)
    S, Tk, V, eri = ao_integrals(mol, basis)
    n_o = int(round(mol.charges.sum())) // 2
    e_nuc = mol.nuclear_repulsion()
    E_hf, C, eps = rhf(S, Tk + V, eri, n_o, e_nuc)
    L_ao = pivoted_cholesky(eri, v["cd_threshold"])
    L_mo = np.einsum("mp,Jmn,nq->Jpq", C, L_ao, C, optimize=True)
    h_mo = C.T @ (Tk + V) @ C
    mu_mo = np.einsum("mp,xmn,nq->xpq", C, ao_dipole(mol, basis), C, optimize=True)
    nuc = (mol.charges[:, None] * mol.coords_bohr).sum(axis=0)
    return dict(L_mo=L_mo, h_mo=h_mo, eps=eps, n_o=n_o, e_hf=E_hf, e_nuc=e_nuc, mu_mo=mu_mo, nuclear_dipole=nuc,
                reference=v)


# H2O at O (0,0,0), H (0, +-0.757, 0.587) Angstrom, cc-pVDZ, Cholesky threshold 1e-8:
# the plain-FP64 drop-in workload (5 occupied, 19 virtual orbitals).
WATER_SYMBOLS = ["O", "H", "H"]
WATER_ANGSTROM = [[0.0, 0.0, 0.0], [0.0, 0.757, 0.587], [0.0, -0.757, 0.587]]


def water_system(cd_threshold=1e-8):
    return build_system(WATER_SYMBOLS, WATER_ANGSTROM, golden_basis(), cd_threshold=cd_threshold)
