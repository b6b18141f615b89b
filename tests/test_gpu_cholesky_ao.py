"""MO Cholesky vectors built on the device from (wx|K) and (K|L) against the host MO transform,
for eT's H2O+He/cc-pVDZ test molecule (Cholesky threshold 1e-12)."""

import numpy as np
import pytest

from oracle import ccsd as oc

pytestmark = pytest.mark.gpu


def test_cholesky_mo_vectors_from_ao_integrals():
    from et_b200 import CCSD
    from oracle import frontend as fe
    v = fe.golden_values()["ccsd_gs_energy"]
    mol = fe.molecule_from_angstrom([a[0] for a in v["atoms"]], [a[1:] for a in v["atoms"]])
    S_ao, Tk, V, eri = fe.ao_integrals(mol, fe.golden_basis())
    n_ao = S_ao.shape[0]
    n_o = int(round(mol.charges.sum())) // 2
    E_hf, C, eps = fe.rhf(S_ao, Tk + V, eri, n_o, mol.nuclear_repulsion())
    L_ao, piv = fe.pivoted_cholesky(eri, v["cd_threshold"], pivots=True)
    M = eri.reshape(n_ao * n_ao, n_ao * n_ao)
    W = M[:, piv].reshape(n_ao, n_ao, len(piv))          # (wx|K)
    S = M[np.ix_(piv, piv)]                               # (K|L)
    L_mo = np.einsum("mp,Jmn,nq->Jpq", C, L_ao, C, optimize=True)
    h_mo = C.T @ (Tk + V) @ C
    n_J, n_mo = len(piv), C.shape[1]
    amp = None
    out = []
    for via_ao in (False, True):
        with CCSD(n_o, n_mo - n_o, n_J) as g:
            if via_ao:
                g.set_cholesky_ao(W, S, C)
            else:
                g.set_cholesky_mo(L_mo)
            g.set_h_mo(h_mo, eps, E_hf)
            g.set_initial_amplitudes_guess()
            if amp is None:
                amp = g.get_amplitudes() * (1.0 + 0.1 * np.random.default_rng(0).standard_normal(g.n_amp))
            g.set_amplitudes(amp)
            out.append((g.calculate_energy(), g.construct_omega()))
    assert abs(out[0][0] - out[1][0]) < 1e-11
    assert np.abs(out[0][1] - out[1][1]).max() < 1e-11 * max(1.0, np.abs(out[0][1]).max())


def test_cholesky_ao_rejects_an_indefinite_basis_overlap():
    from et_b200 import CCSD, CCSDGPUError
    with CCSD(2, 3, 4) as g:
        W = np.zeros((5, 5, 4))
        S = -np.eye(4)
        with pytest.raises(CCSDGPUError):
            g.set_cholesky_ao(W, S, np.eye(5))
