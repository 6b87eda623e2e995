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


# ---------------------------------------------------------------------------
# adjoint (CC Lambda) on the compact layout
# ---------------------------------------------------------------------------
def _blk(plan, ch, X):
    return X[ch.offset:ch.offset + ch.size].reshape(ch.np1, ch.np2, ch.nh1, ch.nh2)


def lambda_residual(plan, fock, t1, B, lam1, Lam):
    """(Z1, Z2, U, T): gradient of L = E + <lam1, R1> + <Lam, R2> with
    respect to (t1, compact t2) at (t1, B), plus the hole-hole contractions
    U = t1^T lam1 and T (sum over channels of Lam . B along i and j) that the
    coupling derivative needs."""
    f_pp, f_ph, f_hh = [np.asarray(f) for f in fock]
    pr = prep(plan, t1, f_pp, f_ph, f_hh)
    Q, Xh = pr["Q"], pr["Xh2"]
    U = t1.T @ lam1
    Z1 = f_ph.copy() + f_pp @ lam1 - lam1 @ f_hh.T - lam1 @ Q.T - f_ph @ U
    Z2 = np.zeros_like(Lam)
    T = np.zeros_like(f_hh)
    for n, ch in enumerate(plan.channels):
        P1, P2, H1, H2 = plan.p_of[ch.g1], plan.p_of[ch.g2], plan.h_of[ch.g1], plan.h_of[ch.g2]
        Lb, Bb = _blk(plan, ch, Lam), _blk(plan, ch, B)
        F1, F2s = _fpp_sub(plan, ch.g1), _fpp_sub(plan, ch.g2)
        f1, f2 = _fph_sub(plan, ch.g1), _fph_sub(plan, ch.g2)
        t1a, t1b = t1[np.ix_(P1, H1)], t1[np.ix_(P2, H2)]
        X1, X2 = Xh[np.ix_(H1, H1)], Xh[np.ix_(H2, H2)]
        Z = np.einsum("bc,acij->abij", F2s, Lb) + np.einsum("ac,cbij->abij", F1, Lb)
        Hb = np.einsum("ck,acij->akij", t1b, Lb)
        Ha = np.einsum("ck,cbij->kbij", t1a, Lb)
        Z -= np.einsum("bk,akij->abij", f2, Hb)
        Z -= np.einsum("ak,kbij->abij", f1, Ha)
        Z += np.einsum("ik,abkj->abij", X1, Lb) + np.einsum("jk,abik->abij", X2, Lb)
        Lv = Lb.reshape(ch.np1, ch.np2, -1)
        Zv = Z.reshape(ch.np1, ch.np2, -1)
        ptr, col, val = plan.hh_ptr[n], plan.hh_col[n], plan.hh_val[n]
        for hp in range(ch.nh1 * ch.nh2):
            for e in range(ptr[hp], ptr[hp + 1]):
                Zv[:, :, col[e]] += val[e] * Lv[:, :, hp]
        La = Lb.reshape(ch.np1 * ch.np2, ch.nh1, ch.nh2)
        Za = Z.reshape(ch.np1 * ch.np2, ch.nh1, ch.nh2)
        ptr, col, val = plan.pp_ptr[n], plan.pp_col[n], plan.pp_val[n]
        for ab in range(ch.np1 * ch.np2):
            for e in range(ptr[ab], ptr[ab + 1]):
                Za[col[e]] += val[e] * La[ab]
        Z += np.einsum("am,bn->abmn", lam1[np.ix_(P1, H1)], f2) + np.einsum("bn,am->abmn", lam1[np.ix_(P2, H2)], f1)
        Z2[ch.offset:ch.offset + ch.size] = Z.ravel()
        # T1-side pieces
        Gb = np.einsum("ck,acij->akij", f2, Bb)
        Ga = np.einsum("ck,cbij->kbij", f1, Bb)
        Z1[np.ix_(P2, H2)] -= np.einsum("axij,amij->xm", Lb, Gb)
        Z1[np.ix_(P1, H1)] -= np.einsum("xbij,mbij->xm", Lb, Ga)
        T[np.ix_(H1, H1)] += np.einsum("abij,abkj->ki", Lb, Bb)
        T[np.ix_(H2, H2)] += np.einsum("abij,abik->kj", Lb, Bb)
        ptr, col, val = plan.hh_ptr[n], plan.hh_col[n], plan.hh_val[n]
        for hp in range(ch.nh1 * ch.nh2):
            for e in range(ptr[hp], ptr[hp + 1]):
                kq, lq = divmod(col[e], ch.nh2)
                Z1[P1, H1[kq]] += val[e] * Lv[:, :, hp] @ t1b[:, lq]
                Z1[P2, H2[lq]] += val[e] * Lv[:, :, hp].T @ t1a[:, kq]
        ptr, col, val = plan.pp_ptr[n], plan.pp_col[n], plan.pp_val[n]
        for ab in range(ch.np1 * ch.np2):
            for e in range(ptr[ab], ptr[ab + 1]):
                cq, dq = divmod(col[e], ch.np2)
                Z1[P1[cq], H1] += val[e] * La[ab] @ t1b[dq, :]
                Z1[P2[dq], H2] += val[e] * La[ab].T @ t1a[cq, :]
    Z1 -= f_ph @ T
    Z1 = np.where(plan.t1_mask(), Z1, 0.0)
    return Z1, Z2, U, T


def lambda_solve(plan, fock, t1, B, mixing=0.5, tol=1e-12, max_iter=5000):
    """Jacobi on Z = 0 with the amplitude equations' denominators."""
    f_pp, f_ph, f_hh = [np.asarray(f) for f in fock]
    pr = prep(plan, t1, f_pp, f_ph, f_hh)
    D1 = -(pr["dXp1"][:, None] + np.diag(pr["Xh1"])[None, :])
    D2 = np.zeros(plan.n_t2)
    for ch in plan.channels:
        P1, P2, H1, H2 = plan.p_of[ch.g1], plan.p_of[ch.g2], plan.h_of[ch.g1], plan.h_of[ch.g2]
        dp, dh = pr["dXp2"], np.diag(pr["Xh2"])
        D2[ch.offset:ch.offset + ch.size] = -(dp[P1][:, None, None, None] + dp[P2][None, :, None, None]
                                              + dh[H1][None, None, :, None] + dh[H2][None, None, None, :]).ravel()
    lam1 = np.zeros_like(t1)
    Lam = np.zeros(plan.n_t2)
    for it in range(max_iter):
        Z1, Z2, U, T = lambda_residual(plan, fock, t1, B, lam1, Lam)
        d1 = np.where(plan.t1_mask(), (1 - mixing) * Z1 / D1, 0.0)
        d2 = (1 - mixing) * Z2 / D2
        lam1 = lam1 + d1
        Lam = Lam + d2
        if np.sqrt(np.sum(d1 ** 2) + 4 * np.sum(d2 ** 2)) < tol * max(1.0, np.sqrt(np.sum(lam1 ** 2))):
            break
    return lam1, Lam, it + 1


def coupling_gradient(plan, dfock, dtwo, de_ref, t1, B, lam1, Lam):
    """dE/dc = dE_ref/dc + <lam1, R1(t; dH)> + <Lam, R2(t; dH)> for a
    derivative Hamiltonian dH with zero f_pp and f_ph (closed sites)."""
    df_pp, df_ph, df_hh = [np.asarray(f) for f in dfock]
    assert not np.any(df_pp) and not np.any(df_ph)
    from nulattice_b200 import structure as S
    _, _, U, T = lambda_residual(plan, [np.zeros_like(df_pp), np.zeros_like(df_ph), np.zeros_like(df_hh)],
                                 t1, B, lam1, Lam)
    g = de_ref - np.sum(U * df_hh) - np.sum(T * df_hh)
    pp_idx, pp_val = S._coo(dtwo[0])
    hh_idx, hh_val = S._coo(dtwo[5])
    for ch in plan.channels:
        P1, P2, H1, H2 = plan.p_of[ch.g1], plan.p_of[ch.g2], plan.h_of[ch.g1], plan.h_of[ch.g2]
        Lb, Bb = _blk(plan, ch, Lam), _blk(plan, ch, B)
        t1a, t1b = t1[np.ix_(P1, H1)], t1[np.ix_(P2, H2)]
        tau = Bb + np.einsum("ak,bl->abkl", t1a, t1b)
        for (k, l, i, j), v in zip(hh_idx.tolist(), hh_val):
            if plan.h_label[k] == ch.g1 and plan.h_label[l] == ch.g2 and plan.h_label[i] == ch.g1 \
                    and plan.h_label[j] == ch.g2:
                g += v * np.sum(Lb[:, :, plan.h_loc[i], plan.h_loc[j]] * tau[:, :, plan.h_loc[k], plan.h_loc[l]])
        for (a, b, c, d), v in zip(pp_idx.tolist(), pp_val):
            if plan.p_label[a] == ch.g1 and plan.p_label[b] == ch.g2 and plan.p_label[c] == ch.g1 \
                    and plan.p_label[d] == ch.g2:
                g += v * np.sum(Lb[plan.p_loc[a], plan.p_loc[b]] * tau[plan.p_loc[c], plan.p_loc[d]])
    return g
