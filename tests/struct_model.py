"""CPU model of the structured (channel-layout) CCSD iteration.

It follows the decomposition of the CUDA kernels in
``nulattice_b200/csrc/ccsd_struct.cu`` step by step (prep, G intermediates,
T2 update, T1 update) on the compact T2 of :mod:`nulattice_b200.structure`,
so the channel algebra can be checked against the dense oracle on the CPU.
Test helper only.
"""
import numpy as np


def prep(plan, t1, f_pp, f_ph, f_hh):
    Q = f_ph.T @ t1                          # Q[k,j] = sum_c f_ck t1_cj
    S = (f_ph * t1).sum(1)                   # S[a] = sum_k f_ak t1_ak
    return dict(Q=Q, Xh2=-f_hh - Q, Xh1=-f_hh - 0.5 * Q,
                dXp2=np.diag(f_pp) - S, dXp1=np.diag(f_pp) - 0.5 * S)


def _fpp_sub(plan, g):
    n = len(plan.p_of[g])
    m = np.zeros((n, n))
    b = plan.p_base[g]
    for r in range(n):
        s, e = plan.fpp_ptr[b + r], plan.fpp_ptr[b + r + 1]
        m[r, plan.fpp_col[s:e]] += plan.fpp_val[s:e]
    return m


def _fph_sub(plan, g):
    n, nh = len(plan.p_of[g]), len(plan.h_of[g])
    m = np.zeros((n, nh))
    b = plan.h_base[g]
    for k in range(nh):
        s, e = plan.fph_ptr[b + k], plan.fph_ptr[b + k + 1]
        m[plan.fph_col[s:e], k] += plan.fph_val[s:e]
    return m


def g_terms(plan, B):
    """Gb[ch][a',k',i',j'] = sum_c f_ck B[a',c',i',j'] (k in H_g2) and
    Ga[ch][b',k',i',j'] = sum_c f_ck B[c',b',i',j'] (k in H_g1)."""
    Gb, Ga = [], []
    for ch in plan.channels:
        blk = B[ch.offset:ch.offset + ch.size].reshape(ch.np1, ch.np2, ch.nh1, ch.nh2)
        F2, F1 = _fph_sub(plan, ch.g2), _fph_sub(plan, ch.g1)
        Gb.append(np.einsum("ck,acij->akij", F2, blk))
        Ga.append(np.einsum("ck,cbij->bkij", F1, blk))
    return Gb, Ga


def t2_update(plan, B, t1, pr, Gb, Ga, mixing):
    out = np.zeros_like(B)
    for n, ch in enumerate(plan.channels):
        P1, P2, H1, H2 = plan.p_of[ch.g1], plan.p_of[ch.g2], plan.h_of[ch.g1], plan.h_of[ch.g2]
        blk = B[ch.offset:ch.offset + ch.size].reshape(ch.np1, ch.np2, ch.nh1, ch.nh2)
        t11, t12 = t1[np.ix_(P1, H1)], t1[np.ix_(P2, H2)]
        tau = blk + np.einsum("ak,bl->abkl", t11, t12)
        R = np.einsum("bc,acij->abij", _fpp_sub(plan, ch.g2), blk)
        R += np.einsum("ac,cbij->abij", _fpp_sub(plan, ch.g1), blk)
        R -= np.einsum("bk,akij->abij", t12, Gb[n])
        R -= np.einsum("ak,bkij->abij", t11, Ga[n])
        X1 = pr["Xh2"][np.ix_(H1, H1)]
        X2 = pr["Xh2"][np.ix_(H2, H2)]
        R += np.einsum("ki,abkj->abij", X1, blk)
        R += np.einsum("kj,abik->abij", X2, blk)
        tau2 = tau.reshape(ch.np1, ch.np2, ch.nh1 * ch.nh2)
        Rv = R.reshape(ch.np1, ch.np2, ch.nh1 * ch.nh2)
        ptr, col, val = plan.hh_ptr[n], plan.hh_col[n], plan.hh_val[n]
        for hp in range(ch.nh1 * ch.nh2):
            for e in range(ptr[hp], ptr[hp + 1]):
                Rv[:, :, hp] += val[e] * tau2[:, :, col[e]]
        tauab = tau.reshape(ch.np1 * ch.np2, ch.nh1, ch.nh2)
        Rab = R.reshape(ch.np1 * ch.np2, ch.nh1, ch.nh2)
        ptr, col, val = plan.pp_ptr[n], plan.pp_col[n], plan.pp_val[n]
        for ab in range(ch.np1 * ch.np2):
            for e in range(ptr[ab], ptr[ab + 1]):
                Rab[ab] += val[e] * tauab[col[e]]
        dp, dh = pr["dXp2"], np.diag(pr["Xh2"])
        D = -(dp[P1][:, None, None, None] + dp[P2][None, :, None, None]
              + dh[H1][None, None, :, None] + dh[H2][None, None, None, :])
        out[ch.offset:ch.offset + ch.size] = (blk + (1.0 - mixing) * R / D).ravel()
    return out


def t1_update(plan, t1, pr, f_pp, f_ph, Gb, Ga, mixing):
    p, h = t1.shape
    F2 = np.zeros((p, h))
    for n, ch in enumerate(plan.channels):
        P1, P2, H1, H2 = plan.p_of[ch.g1], plan.p_of[ch.g2], plan.h_of[ch.g1], plan.h_of[ch.g2]
        # a in P1, i in H1: sum_k' Gb[a',k',i',k']
        F2[np.ix_(P1, H1)] += np.einsum("akik->ai", Gb[n])
        # a in P2, i in H2: sum_k' Ga[a',k',k',i']
        F2[np.ix_(P2, H2)] += np.einsum("akki->ai", Ga[n])
    H1 = f_ph + F2 + f_pp @ t1 - 0.5 * t1 @ pr["Q"] + t1 @ pr["Xh1"]
    D1 = -(pr["dXp1"][:, None] + np.diag(pr["Xh1"])[None, :])
    t1n = t1 + H1 / D1
    out = mixing * t1 + (1.0 - mixing) * t1n
    return np.where(plan.t1_mask(), out, 0.0)


def iterate(plan, fock, t1, B, mixing):
    f_pp, f_ph, f_hh = fock
    pr = prep(plan, t1, f_pp, f_ph, f_hh)
    Gb, Ga = g_terms(plan, B)
    Bn = t2_update(plan, B, t1, pr, Gb, Ga, mixing)
    t1n = t1_update(plan, t1, pr, f_pp, f_ph, Gb, Ga, mixing)
    return t1n, Bn
