"""Seeded synthetic Cholesky-factored CCSD systems.

The generator follows the recipe the benchmark configurations are quoted on:

* ``L^J_pq = s_J (X + X^T)/2`` with ``X ~ N(0,1)/sqrt(n_o+n_v)`` (n_mo x n_mo)
  and ``s_J = exp(-8 J / N_J)`` for ``J = 0 .. N_J-1`` (0-based J);
* a diagonal MO Fock matrix, occupied energies ``U[-1.2, -0.4]`` Eh and
  virtual energies ``U[0.1, 2.5]`` Eh (sorted ascending);
* ``h_pq = F_pq - sum_k (2 g_pqkk - g_pkkq)`` so that the T1 Fock matrix that
  eT rebuilds from h and L equals the chosen diagonal at t1 = 0;
* ``E_HF`` = 0 (energies are reported as correlation energies).

``coupling`` (kappa) multiplies X.  kappa = 1 is the literal recipe; with it the
CCSD iterations diverge already at o=8, v=80 (the MP2 energy grows like
o^2 v^2 N_J / (o+v)^2 and reaches ~-1e3 Eh at o=32, v=320), so the default
kappa = 0.15 keeps every shape, flop count and data layout and gives a
convergent, molecule-like system (E_MP2 of a few Eh at o=32, v=320).

Randomness: numpy PCG64 seeded with ``seed``; the same arrays feed the CUDA
path and the CPU oracle.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class System:
    n_o: int
    n_v: int
    n_J: int
    L_mo: np.ndarray      # (n_J, n_mo, n_mo), L[J, p, q]
    h_mo: np.ndarray      # (n_mo, n_mo)
    eps: np.ndarray       # (n_mo,)
    e_hf: float = 0.0

    @property
    def n_mo(self) -> int:
        return self.n_o + self.n_v


DEFAULT_COUPLING = 0.15


def make_system(n_o: int, n_v: int, n_J: int, seed: int = 2026, coupling: float = DEFAULT_COUPLING) -> System:
    rng = np.random.Generator(np.random.PCG64(seed))
    n_mo = n_o + n_v
    # eT's layout of the MO Cholesky vectors, L(J, pq) with J fastest (Fortran order), so that the
    # host arrays go to the library without a reordering copy
    L = np.empty((n_J, n_mo, n_mo), dtype=np.float64, order="F")
    scale = coupling / np.sqrt(n_o + n_v)
    for J in range(n_J):
        X = rng.standard_normal((n_mo, n_mo)) * scale
        L[J] = np.exp(-8.0 * J / n_J) * 0.5 * (X + X.T)
    e_occ = np.sort(rng.uniform(-1.2, -0.4, n_o))
    e_vir = np.sort(rng.uniform(0.1, 2.5, n_v))
    eps = np.concatenate([e_occ, e_vir])
    Lk = np.einsum("Jkk->J", L[:, :n_o, :n_o])
    coul = 2.0 * np.einsum("Jpq,J->pq", L, Lk)
    Lo = L[:, :, :n_o]
    exch = np.einsum("Jpk,Jqk->pq", Lo, Lo, optimize=True)   # L_kq = L_qk (symmetric L)
    h = np.diag(eps) - coul + exch
    return System(n_o=n_o, n_v=n_v, n_J=n_J, L_mo=L, h_mo=h, eps=eps, e_hf=0.0)


# Workload shapes (o, v, N_J) of the benchmark configurations.
GS_SYNTHETIC = dict(n_o=32, n_v=320, n_J=1200)      # ground state, 30 DIIS iterations
EOM_SYNTHETIC = dict(n_o=24, n_v=240, n_J=792)      # 12 roots, blocks of 24 trials
ADJOINT_SYNTHETIC = dict(n_o=16, n_v=128, n_J=432)  # VJP vs finite differences
