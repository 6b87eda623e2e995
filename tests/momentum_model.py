"""CPU model of the momentum-block residual (test helper).

It follows the decomposition of the CUDA kernels in
``nulattice_b200/csrc/momentum.cu`` on the blocked t2 of
:class:`nulattice_b200.momentum.MomentumPlan`: M sums over the particle
momentum, row dots for X_pp, X_hh from M, the dressed hole-hole matrix W_K
per block, the particle-hole intermediates R, U, G, and every term of the
residual per block, so the blocked algebra can be checked against the dense
oracle on the CPU.
"""
import numpy as np

from nulattice_b200 import momentum as MB


def _blocks(plan, t):
    return [t[plan.blk_off[q]:plan.blk_off[q + 1]].reshape(int(plan.nr[q]), int(plan.nc[q]))
            for q in range(len(plan.Ks))]


def _group_momenta(plan, q):
    """Particle-momentum indices (first, second) of each row group and
    hole-momentum indices (first, second) of each column group of block q."""
    L, K = plan.L, plan.Ks[q]
    ma = plan.pm_list[plan.pm0[q]:plan.pm0[q] + plan.nr[q] // 16]
    mb = plan.pinv[MB._madd(L, K, MB._mneg(L, plan.pmom[ma]))]
    mi = plan.hm_list[plan.hm0[q]:plan.hm0[q] + plan.nc[q] // 16]
    mj = plan.hinv[MB._madd(L, K, MB._mneg(L, plan.hmom[mi]))]
    return ma, mb, mi, mj


def residual(plan, V, fpp, fhh, t):
    """Blocked T2 residual H (before the antisymmetric projection) and the
    X_pp / X_hh blocks, ``(H, Xpp[n_pmom,4,4], Xhh[n_hmom,4,4])``."""
    V = np.asarray(V, dtype=np.float64).reshape(4, 4, 4, 4)
    Vf = V.reshape(16, 16)
    T = _blocks(plan, np.asarray(t, dtype=np.float64))
    nb, npm, nhm, L = len(plan.Ks), len(plan.pmom), len(plan.hmom), plan.L
    M = [TK.reshape(-1, 16, TK.shape[1]).sum(0) for TK in T]
    grp = [_group_momenta(plan, q) for q in range(nb)]
    # X_pp[m][s_b, s_c] = f_pp - 1/2 sum_K sum_{s_d} sum_col V[s_c s_d][col spins] T[(m s_b s_d)][col]
    Xpp = np.array(fpp, dtype=np.float64).reshape(npm, 4, 4).copy()
    for q in range(nb):
        ma, mb, mi, mj = grp[q]
        cs = np.tile(np.arange(16), len(mi))
        Y = (T[q] @ Vf[:, cs].T).reshape(len(ma), 4, 4, 4, 4)     # [pa, s_b, s_d, s_c, s_d']
        np.add.at(Xpp, ma, -0.5 * np.einsum("pbdcd->pbc", Y))
    # X_hh[m][s_k, s_j] = -f_hh - 1/2 sum_{m_l, s_l} sum_sigma V[sigma][s_k s_l] M[sigma][(m s_j s_l)]
    Xhh = -np.array(fhh, dtype=np.float64).reshape(nhm, 4, 4)
    for q in range(nb):
        ma, mb, mi, mj = grp[q]
        Wh = (Vf.T @ M[q]).reshape(4, 4, len(mi), 4, 4)           # [s_k, s_l, pi, s_j, s_l']
        np.add.at(Xhh, mi, -0.5 * np.einsum("klpjl->pkj", Wh))
    # R[a, i][s_c, s_k] = sum_{k_k} t2[a, (k_k + k_i - k_a, s_c), i, (k_k, s_k)]
    R = np.zeros((npm, 4, nhm, 4, 4, 4))                         # [ma, sa, mi, si, sc, sk]
    for xa in range(npm):
        ka = plan.pmom[xa]
        for xi in range(nhm):
            ki = plan.hmom[xi]
            for kk in plan.hmom:
                kc = MB._madd(L, MB._madd(L, kk, ki), MB._mneg(L, ka))
                if plan.pinv[kc] < 0:
                    continue
                b = plan.kblk[MB._madd(L, ka, kc)]
                pa, pi = plan.ppos[b, ka], plan.hpos[b, ki]
                blk = T[b].reshape(-1, 4, 4, int(plan.nc[b]) // 16, 4, 4)[pa, :, :, pi]   # [sa, sc, si, sk]
                R[xa, :, xi] += blk.transpose(0, 2, 1, 3)
    R = R.reshape(npm * 4, nhm * 4, 4, 4)
    G = -np.einsum("bkcj,aick->aibj", V, R)
    U = np.einsum("aick,cdkl->aidl", R, V)
    G6 = G.reshape(npm, 4, nhm, 4, 4, 4)                         # [ma, sa, mi, si, sb, sj]
    U6, R6 = U.reshape(npm, 4, nhm, 4, 16), R.reshape(npm, 4, nhm, 4, 16)
    H = np.zeros(plan.n_t2)
    for q in range(nb):
        ma, mb, mi, mj = grp[q]
        TK = T[q]
        nr, nc = TK.shape
        npa, nhg = nr // 16, nc // 16
        rs, cs = np.tile(np.arange(16), npa), np.tile(np.arange(16), nhg)
        # v_pphh, 1/2 v_pppp t2 through M, hole ladders through W_K
        Wq = 0.5 * Vf[cs][:, cs] + 0.25 * Vf[:, cs].T @ M[q]
        HK = Vf[rs][:, cs] + 0.5 * Vf[rs] @ M[q] + TK @ Wq
        T6 = TK.reshape(npa, 4, 4, nhg, 4, 4)                    # [pa, sa, sb, pi, si, sj]
        xp = np.einsum("pbc,pacPij->pabPij", Xpp[mb], T6) + np.einsum("pac,pcbPij->pabPij", Xpp[ma], T6)
        xh = np.einsum("Pkj,pabPik->pabPij", Xhh[mj], T6) + np.einsum("Pki,pabPkj->pabPij", Xhh[mi], T6)
        ring = (G6[ma][:, :, mi].transpose(0, 1, 4, 2, 3, 5) - G6[mb][:, :, mi].transpose(0, 4, 1, 2, 3, 5)
                - G6[ma][:, :, mj].transpose(0, 1, 4, 2, 5, 3) + G6[mb][:, :, mj].transpose(0, 4, 1, 2, 5, 3))
        quad = (np.einsum("paPix,pbPjx->pabPij", U6[ma][:, :, mi], R6[mb][:, :, mj])
                - np.einsum("pbPix,paPjx->pabPij", U6[mb][:, :, mi], R6[ma][:, :, mj]))
        HK = HK + (xp + xh + ring + quad).reshape(nr, nc)
        H[plan.blk_off[q]:plan.blk_off[q + 1]] = HK.ravel()
    return H, Xpp, Xhh


def step(plan, V, fpp, fhh, t, mixing=0.5):
    """One Jacobi step with mixing on the blocked amplitudes: the residual,
    the denominators -(X_pp[a,a] + X_pp[b,b] + X_hh[i,i] + X_hh[j,j]) from
    the diagonals of the 4x4 blocks, ``m t + (1 - m)(t + H / D)``."""
    t = np.asarray(t, dtype=np.float64)
    H, Xpp, Xhh = residual(plan, V, fpp, fhh, t)
    dp, dh = np.einsum("mss->ms", Xpp), np.einsum("mss->ms", Xhh)
    D = np.zeros(plan.n_t2)
    for q in range(len(plan.Ks)):
        ma, mb, mi, mj = _group_momenta(plan, q)
        npa, nhg = len(ma), len(mi)
        drow = (dp[ma][:, :, None] + dp[mb][:, None, :]).reshape(npa * 16)     # [pa, sa, sb]
        dcol = (dh[mi][:, :, None] + dh[mj][:, None, :]).reshape(nhg * 16)     # [pi, si, sj]
        D[plan.blk_off[q]:plan.blk_off[q + 1]] = (-(drow[:, None] + dcol[None, :])).ravel()
    return mixing * t + (1.0 - mixing) * (t + H / D)
