"""The identity behind the device ladder (mixed precision, and FP64 with resident integrals), checked
with the oracle on the CPU: with the T1-transformed vv block L~_ac = L_ac - sum_k t_ak L_kc,

    sum_cd g~_acbd t_cidj = X0 - (A + A^T) + T4,
    X0_aibj = sum_cd g_acbd t_cidj,         A_aibj = sum_k t_ak Y_kibj,  Y_kibj = sum_cd g_kcbd t_cidj,
    T4_aibj = sum_kl t_ak t_bl Q_kilj,      Q_kilj = sum_cd g_kcld t_cidj,

all with integrals of the untransformed vectors, equals eT's A2 ladder on T1-transformed integrals
(omega_ccsd.F90:113-480, restated by the oracle's omega_ccsd_a2_dense)."""

import numpy as np
import pytest

from et_b200.synthetic import make_system
from oracle import ccsd as oc


def ladder_untransformed(t, t1, L, n_o):
    v = slice(n_o, None)
    o = slice(0, n_o)
    g_vvvv = oc.eri(L[:, v, v], L[:, v, v])
    g_ovvv = oc.eri(L[:, o, v], L[:, v, v])          # g_kcbd
    g_ovov = oc.eri(L[:, o, v], L[:, o, v])          # g_kcld
    X0 = np.einsum("acbd,cidj->aibj", g_vvvv, t, optimize=True)
    Y = np.einsum("kcbd,cidj->kibj", g_ovvv, t, optimize=True)
    A = np.einsum("ak,kibj->aibj", t1, Y, optimize=True)
    Q = np.einsum("kcld,cidj->kilj", g_ovov, t, optimize=True)
    T4 = np.einsum("ak,bl,kilj->aibj", t1, t1, Q, optimize=True)
    return X0 - (A + A.transpose(2, 3, 0, 1)) + T4


@pytest.mark.parametrize("dims", [(2, 5, 9), (3, 8, 20), (4, 11, 30)])
def test_untransformed_ladder_with_t1_corrections_equals_transformed_ladder(dims):
    n_o, n_v, n_J = dims
    s = make_system(n_o, n_v, n_J, seed=31)
    rng = np.random.default_rng(8)
    sysm = oc.CCSDSystem(s.L_mo, s.h_mo, s.eps, n_o)
    amp = 0.1 * rng.standard_normal(sysm.n_amp)
    sysm.set_amplitudes(amp)
    t = oc.squareup(sysm.t2, n_v, n_o)
    ref = oc.omega_ccsd_a2_dense(t, sysm.L_t1, n_o)
    got = oc.pack_half_diag(ladder_untransformed(t, sysm.t1, np.asarray(s.L_mo), n_o), n_v, n_o)
    assert np.abs(got - ref).max() <= 1e-13 * max(1.0, np.abs(ref).max())


def test_y_with_transformed_vv_block_is_y0_minus_t1_q():
    """The Jacobian's t1 terms use Y with the transformed vv block: Y~ = Y0 - sum_l t_bl Q_kilj."""
    n_o, n_v, n_J = 3, 9, 22
    s = make_system(n_o, n_v, n_J, seed=33)
    sysm = oc.CCSDSystem(s.L_mo, s.h_mo, s.eps, n_o)
    sysm.set_amplitudes(0.1 * np.random.default_rng(9).standard_normal(sysm.n_amp))
    t = oc.squareup(sysm.t2, n_v, n_o)
    L, Lt = np.asarray(s.L_mo), sysm.L_t1
    o, v = slice(0, n_o), slice(n_o, None)
    Y_t = np.einsum("kcbd,cidj->kibj", oc.eri(Lt[:, o, v], Lt[:, v, v]), t, optimize=True)
    Y0 = np.einsum("kcbd,cidj->kibj", oc.eri(L[:, o, v], L[:, v, v]), t, optimize=True)
    Q = np.einsum("kcld,cidj->kilj", oc.eri(L[:, o, v], L[:, o, v]), t, optimize=True)
    got = Y0 - np.einsum("bl,kilj->kibj", sysm.t1, Q, optimize=True)
    assert np.abs(got - Y_t).max() <= 1e-13 * max(1.0, np.abs(Y_t).max())
