"""CPU FP64 oracle for NuLattice's CCSD iteration -- TEST INFRASTRUCTURE ONLY.

This module restates, in plain numpy, the algorithm of the reference solver:

* ``CCM/coupled_cluster.py:265-286``  ``ccsd_energy``
* ``CCM/coupled_cluster.py:319-340``  ``t1Init`` (MP2 guess for T1)
* ``CCM/coupled_cluster.py:342-414``  ``t1Iter`` (dressed Jacobi step for T1)
* ``CCM/coupled_cluster.py:416-439``  ``t2Init`` (MP2 guess for T2)
* ``CCM/coupled_cluster.py:442-545``  ``t2Iter`` (dressed Jacobi step for T2)
* ``CCM/coupled_cluster.py:547-687``  ``ccsd_solver`` (mixing, convergence test)
* ``CCM/soa/coupled_cluster.py:479-567`` pulsed DIIS of the torch solver
* ``CCM/ccDgrams.py:13-578``          the individual diagrams

Only the test-suite, ``__graft_entry__.smoke`` and ``bench.py``'s CPU-baseline
leg may import it, always as the checker.  The product solver never calls it.

Layout conventions are the reference's: ``t1[a,i]``, ``t2[a,b,i,j]``,
``f_pp[a,b]``, ``f_ph[a,i]``, ``f_hh[i,j]``, ``v_pphh[a,b,i,j] = <ab||ij>``,
``v_phph[a,i,b,j] = <ai||bj>``, ``v_phhh[a,i,j,k] = <ai||jk>``,
``v_hhhh[i,j,k,l] = <ij||kl>``; ``v_pppp`` is a list/array of rows
``[a,b,c,d,val]`` and ``v_ppph`` of rows ``[c,d,a,k,val]`` (``<cd||ak>``);
repeated keys are summed (``CCM/coupled_cluster.py:254-260``).

Every diagram is written as an entry of a term table: a coefficient, an
einsum over named operands and the antisymmetrisers to apply.  Parity with
the reference is pinned by ``tests/golden/*.npz`` (made by running the
reference itself, ``tests/golden/make_goldens.py``).
"""
from __future__ import annotations

import numpy as np

__all__ = [
    "Hamiltonian", "pab", "pij", "ppph_intermediates", "pppp_ladders",
    "DIAGRAMS", "t1_init", "t2_init", "t1_step", "t2_step", "energy", "solve",
    "jacobi_gap",
]


def pab(x):
    """Antisymmetriser over the two particle indices (``ccDgrams.py:193-202``)."""
    return x - x.transpose(1, 0, 2, 3)


def pij(x):
    """Antisymmetriser over the two hole indices (``ccDgrams.py:204-213``)."""
    return x - x.transpose(0, 1, 3, 2)


_PERM = {"": lambda x: x, "ab": pab, "ij": pij, "abij": lambda x: pij(pab(x))}


def _ein(spec, *ops):
    return np.einsum(spec, *ops, optimize="greedy")


# name -> (coefficient, einsum, operands, antisymmetriser).  The name is the
# reference's function name in CCM/ccDgrams.py; the line of its definition is
# given beside each entry.
DIAGRAMS = {
    # T1 equation, H1 parts
    "dgram_akci_ck": (-1.0, "akci,ck->ai", ("v_phph", "t1"), ""),            # :48
    "dgram_ck_acik": (1.0, "ck,acik->ai", ("f_ph", "t2"), ""),               # :61
    "dgram_cikl_cakl": (-0.5, "cikl,cakl->ai", ("v_phhh", "t2"), ""),        # :74
    "dgram_cdkl_ck_dali": (1.0, "cdkl,ck,dali->ai", ("v_pphh", "t1", "t2"), ""),  # :87
    # T1 equation, dressing of the Fock matrices
    "dgram_ck_ci": (-0.5, "ck,ci->ki", ("f_ph", "t1"), ""),                  # :102
    "dgram_ck_ak": (-0.5, "ck,ak->ac", ("f_ph", "t1"), ""),                  # :115
    "dgram_bijk_bj": (-1.0, "bijk,bj->ki", ("v_phhh", "t1"), ""),            # :128
    "dgram_cdlk_cdli": (-0.5, "cdlk,cdli->ki", ("v_pphh", "t2"), ""),        # :141
    "dgram_dckl_dakl": (-0.5, "dckl,dakl->ac", ("v_pphh", "t2"), ""),        # :154
    "dgram_cdlk_cl_di": (-0.5, "cdlk,cl,di->ki", ("v_pphh", "t1", "t1"), ""),  # :167
    "dgram_cdkl_dk_al": (0.5, "cdkl,dk,al->ac", ("v_pphh", "t1", "t1"), ""),   # :180
    # T2 equation
    "dgram_klij_abkl": (0.5, "klij,abkl->abij", ("v_hhhh", "t2"), ""),       # :240
    "dgram_bkcj_acik": (-1.0, "bkcj,acik->abij", ("v_phph", "t2"), "abij"),  # :253
    "dgram_bkij_ak": (1.0, "bkij,ak->abij", ("v_phhh", "t1"), "ab"),         # :266
    "dgram_cdkl_acik_dblj": (0.5, "cdkl,acik,dblj->abij", ("v_pphh", "t2", "t2"), "abij"),  # :279
    "dgram_cdkl_cdij_abkl": (0.25, "cdkl,cdij,abkl->abij", ("v_pphh", "t2", "t2"), ""),     # :292
    "dgram_klij_ak_bl": (0.5, "klij,ak,bl->abij", ("v_hhhh", "t1", "t1"), "ab"),            # :305
    "dgram_bkci_ak_cj": (-1.0, "bkci,ak,cj->abij", ("v_phph", "t1", "t1"), "abij"),         # :318
    "dgram_cikl_ck_ablj": (-1.0, "cikl,ck,ablj->abij", ("v_phhh", "t1", "t2"), "ij"),       # :331
    "dgram_da_dbij": (-1.0, "da,dbij->abij", ("x_pp", "t2"), "ab"),                         # :346
    "dgram_acik_bcjk": (1.0, "acik,bcjk->abij", ("x_pphh", "t2"), "abij"),                  # :359
    "dgram_cikl_al_bcjk": (-1.0, "cikl,al,bcjk->abij", ("v_phhh", "t1", "t2"), "abij"),     # :372
    "dgram_cjkl_ci_abkl": (0.5, "cjkl,ci,abkl->abij", ("v_phhh", "t1", "t2"), "ij"),        # :387
    "dgram_bijk_ak1": (0.5, "bijk,ak->abij", ("x_phhh", "t1"), "ab"),                       # :405
    "dgram_bijk_ak2": (0.5, "bijk,ak->abij", ("x_phhh", "t1"), "abij"),                     # :418
    "dgram_cjkl_ci_ak_bl": (0.5, "cjkl,ci,ak,bl->abij", ("v_phhh", "t1", "t1", "t1"), "abij"),  # :431
    "dgram_cdkl_ci_dj_abkl": (0.25, "cdkl,ci,dj,abkl->abij", ("v_pphh", "t1", "t1", "t2"), "ij"),  # :444
    "dgram_cdkl_ak_bl_cdij": (0.25, "cdkl,ak,bl,cdij->abij", ("v_pphh", "t1", "t1", "t2"), "ab"),  # :459
    "dgram_cdkl_ci_bl_adkj": (1.0, "cdkl,ci,bl,adkj->abij", ("v_pphh", "t1", "t1", "t2"), "abij"),  # :474
    "dgram_cdkl_ci_ak_dj_bl": (0.25, "cdkl,ci,ak,dj,bl->abij",
                               ("v_pphh", "t1", "t1", "t1", "t1"), "abij"),                 # :489
    "dgram_cdkl_bdkl": (-0.5, "cdkl,bdkl->bc", ("v_pphh", "t2"), ""),        # :502
    "dgram_cdkl_cdjl": (-0.5, "cdkl,cdjl->kj", ("v_pphh", "t2"), ""),        # :515
    "dgram_ck_bk": (-1.0, "ck,bk->bc", ("f_ph", "t1"), ""),                  # :528
    "dgram_ck_cj": (-1.0, "ck,cj->kj", ("f_ph", "t1"), ""),                  # :541
    "dgram_cdlk_cl_dj": (-1.0, "cdlk,cl,dj->kj", ("v_pphh", "t1", "t1"), ""),  # :554
    "dgram_cdlk_dk_bl": (-1.0, "cdlk,dk,bl->bc", ("v_pphh", "t1", "t1"), ""),  # :567
}


def diagram(name, **ops):
    """Evaluate one diagram of the table on named numpy operands."""
    coef, spec, names, perm = DIAGRAMS[name]
    return coef * _PERM[perm](_ein(spec, *[ops[n] for n in names]))


def _rows(lst):
    """Split a [k0,k1,k2,k3,val] row list (or an (N,5) array) into (idx, val)."""
    a = np.asarray(lst, dtype=np.float64).reshape(-1, 5)
    return a[:, :4].astype(np.int64), a[:, 4].copy()


class Hamiltonian:
    """Normal-ordered Fock and two-body blocks in the reference's layout."""

    def __init__(self, fock_mats, two_body_int):
        self.f_pp, self.f_ph, self.f_hh = [np.asarray(f, dtype=np.float64) for f in fock_mats]
        v_pppp, v_ppph, self.v_pphh, self.v_phph, self.v_phhh, self.v_hhhh = two_body_int
        self.v_pphh, self.v_phph, self.v_phhh, self.v_hhhh = [
            np.asarray(v, dtype=np.float64) for v in (self.v_pphh, self.v_phph, self.v_phhh, self.v_hhhh)]
        self.pppp_idx, self.pppp_val = _rows(v_pppp)
        self.ppph_idx, self.ppph_val = _rows(v_ppph)
        self.p, self.h = self.f_ph.shape

    def ops(self, t1, t2, **extra):
        d = dict(f_pp=self.f_pp, f_ph=self.f_ph, f_hh=self.f_hh, v_pphh=self.v_pphh,
                 v_phph=self.v_phph, v_phhh=self.v_phhh, v_hhhh=self.v_hhhh, t1=t1, t2=t2)
        d.update(extra)
        return d


def ppph_intermediates(idx, val, t1, t2):
    """The seven v_ppph intermediates of ``CCM/ccDgrams.py:13-45``.

    Rows are ``(c, d, a, k)`` with value ``<cd||ak>``.  Returned in the
    reference's order (r0 .. r6) with the reference's shapes.
    """
    p, h = t1.shape
    r0 = np.zeros((p, h)); r1 = np.zeros((p, p)); r2 = np.zeros((p, p, h, h))
    r3 = np.zeros((p, p)); r4 = np.zeros((p, p, h, h))
    r5 = np.zeros((p, h, h, h)); r6 = np.zeros((p, h, h, h))
    if len(val) == 0:
        return r0, r1, r2, r3, r4, r5, r6
    c, d, a, k = idx.T
    v = val
    np.add.at(r0, a, -0.5 * v[:, None] * t2[c, d, k, :])
    np.add.at(r1, (a, d), -v * t1[c, k])
    np.add.at(r3, (d, a), v * t1[c, k])
    # r2[c,d,:,k] += v t1[a,:] ; r4[a,d,:,k] += v t1[c,:]
    np.add.at(r2.transpose(0, 1, 3, 2), (c, d, k), v[:, None] * t1[a, :])
    np.add.at(r4.transpose(0, 1, 3, 2), (a, d, k), v[:, None] * t1[c, :])
    # r5[a,:,:,k] += v t2[c,d,:,:] ; r6[a,:,:,k] += v t1[c,:] t1[d,:]^T
    np.add.at(r5.transpose(0, 3, 1, 2), (a, k), v[:, None, None] * t2[c, d, :, :])
    np.add.at(r6.transpose(0, 3, 1, 2), (a, k), v[:, None, None] * (t1[c, :, None] * t1[d, None, :]))
    return r0, r1, r2, r3, r4, r5, r6


def pppp_ladders(idx, val, t1, t2):
    """The two sparse v_pppp ladders of ``CCM/ccDgrams.py:215-237``:
    ``sum_cd v_abcd t2_cdij`` and ``sum_cd v_abcd t1_ci t1_dj`` (no 1/2)."""
    p, h = t1.shape
    l1 = np.zeros((p, p, h, h)); l2 = np.zeros((p, p, h, h))
    if len(val) == 0:
        return l1, l2
    a, b, c, d = idx.T
    np.add.at(l1, (a, b), val[:, None, None] * t2[c, d])
    np.add.at(l2, (a, b), val[:, None, None] * (t1[c, :, None] * t1[d, None, :]))
    return l1, l2


# Skip diagrams whose operand block is identically zero (they add exact
# zeros).  The CPU-baseline timing turns this off so that the port does the
# same work as the reference, which evaluates every diagram.
SKIP_ZERO_BLOCKS = True


def _nz(x):
    if not SKIP_ZERO_BLOCKS:
        return x is not None
    return x is not None and np.any(x)


def t1_init(H, delta=0.0):
    """MP2 guess ``t1 = f_ph / (f_ii - f_aa + delta)`` (``coupled_cluster.py:319-340``)."""
    den = np.diag(H.f_hh)[None, :] - np.diag(H.f_pp)[:, None] + delta
    with np.errstate(divide="ignore", invalid="ignore"):
        return H.f_ph / den


def t2_init(H, delta=0.0):
    """MP2 guess ``t2 = v_pphh / (e_i + e_j - e_a - e_b + delta)`` (``:416-439``)."""
    ep, eh = np.diag(H.f_pp), np.diag(H.f_hh)
    den = (-ep[:, None, None, None] - ep[None, :, None, None]
           + eh[None, None, :, None] + eh[None, None, None, :] + delta)
    with np.errstate(divide="ignore", invalid="ignore"):
        return H.v_pphh / den


def _t1_parts(H, t1, t2, r):
    """H1 without the dressed Fock products, and the T1-equation X_pp, X_hh."""
    o = H.ops(t1, t2)
    h1 = H.f_ph.copy()
    xhh = -H.f_hh.copy()
    xpp = H.f_pp.copy()
    h1 += diagram("dgram_ck_acik", **o)
    xhh += diagram("dgram_ck_ci", **o)
    xpp += diagram("dgram_ck_ak", **o)
    if _nz(H.v_phph):
        h1 += diagram("dgram_akci_ck", **o)
    if _nz(H.v_phhh):
        h1 += diagram("dgram_cikl_cakl", **o)
        xhh += diagram("dgram_bijk_bj", **o)
    if _nz(H.v_pphh):
        h1 += diagram("dgram_cdkl_ck_dali", **o)
        xhh += diagram("dgram_cdlk_cdli", **o) + diagram("dgram_cdlk_cl_di", **o)
        xpp += diagram("dgram_dckl_dakl", **o) + diagram("dgram_cdkl_dk_al", **o)
    h1 += r[0]
    xpp += r[1]
    return h1, xpp, xhh


def t1_residual(H, t1, t2, r=None):
    """Full T1 residual H1 of ``t1Iter`` (``coupled_cluster.py:372-408``)."""
    if r is None:
        r = ppph_intermediates(H.ppph_idx, H.ppph_val, t1, t2)
    h1, xpp, xhh = _t1_parts(H, t1, t2, r)
    return h1 + xpp @ t1 + t1 @ xhh, xpp, xhh


def t1_step(H, t1, t2, r=None):
    """One unmixed Jacobi step for T1 (``coupled_cluster.py:342-414``)."""
    h1, xpp, xhh = t1_residual(H, t1, t2, r)
    den = -(np.diag(xpp)[:, None] + np.diag(xhh)[None, :])
    return t1 + h1 / den


def t2_residual(H, t1, t2, r=None):
    """Full T2 residual H2 of ``t2Iter`` (``coupled_cluster.py:476-536``)."""
    if r is None:
        r = ppph_intermediates(H.ppph_idx, H.ppph_val, t1, t2)
    o = H.ops(t1, t2, x_pp=r[3], x_pphh=r[4])
    h2 = H.v_pphh.copy()
    h2 += diagram("dgram_klij_abkl", **o) + diagram("dgram_klij_ak_bl", **o)
    if _nz(H.v_phph):
        h2 += diagram("dgram_bkcj_acik", **o) + diagram("dgram_bkci_ak_cj", **o)
    if _nz(H.v_phhh):
        for n in ("dgram_bkij_ak", "dgram_cikl_ck_ablj", "dgram_cikl_al_bcjk",
                  "dgram_cjkl_ci_abkl", "dgram_cjkl_ci_ak_bl"):
            h2 += diagram(n, **o)
    if _nz(H.v_pphh):
        for n in ("dgram_cdkl_acik_dblj", "dgram_cdkl_cdij_abkl", "dgram_cdkl_ci_dj_abkl",
                  "dgram_cdkl_ak_bl_cdij", "dgram_cdkl_ci_bl_adkj", "dgram_cdkl_ci_ak_dj_bl"):
            h2 += diagram(n, **o)
    xhh = -H.f_hh + diagram("dgram_ck_cj", **o)
    xpp = H.f_pp + diagram("dgram_ck_bk", **o)
    if _nz(H.v_pphh):
        xhh = xhh + diagram("dgram_cdkl_cdjl", **o) + diagram("dgram_cdlk_cl_dj", **o)
        xpp = xpp + diagram("dgram_cdkl_bdkl", **o) + diagram("dgram_cdlk_dk_bl", **o)
    if len(H.ppph_val):
        h2 += pij(r[2])
        h2 += diagram("dgram_da_dbij", **o) + diagram("dgram_acik_bcjk", **o)
        h2 += diagram("dgram_bijk_ak1", **H.ops(t1, t2, x_phhh=r[5]))
        h2 += diagram("dgram_bijk_ak2", **H.ops(t1, t2, x_phhh=r[6]))
    l1, l2 = pppp_ladders(H.pppp_idx, H.pppp_val, t1, t2)
    h2 += 0.5 * l1 + 0.5 * pij(l2)
    h2 += pab(_ein("bc,acij->abij", xpp, t2)) + pij(_ein("kj,abik->abij", xhh, t2))
    return h2, xpp, xhh


def t2_step(H, t1, t2, r=None):
    """One unmixed Jacobi step for T2 (``coupled_cluster.py:442-545``)."""
    h2, xpp, xhh = t2_residual(H, t1, t2, r)
    dp, dh = np.diag(xpp), np.diag(xhh)
    den = -(dp[:, None, None, None] + dp[None, :, None, None]
            + dh[None, None, :, None] + dh[None, None, None, :])
    return t2 + h2 / den


def energy(H, t1, t2):
    """CCSD correlation energy (``coupled_cluster.py:265-286``)."""
    e = float(np.sum(H.f_ph * t1))
    if _nz(H.v_pphh):
        e += 0.25 * float(np.sum(H.v_pphh * t2))
        e += 0.5 * float(_ein("abij,ai,bj->", H.v_pphh, t1, t1))
    return e


def jacobi_gap(H, t1, t2):
    """Norms of one unmixed Jacobi step at (t1, t2); zero at the CCSD fixed point."""
    r = ppph_intermediates(H.ppph_idx, H.ppph_val, t1, t2)
    return (float(np.linalg.norm(t1_step(H, t1, t2, r) - t1)),
            float(np.linalg.norm(t2_step(H, t1, t2, r) - t2)))


def solve(fock_mats, two_body_int, t1initial=None, eps=1e-8, maxSteps=1000, max_diis=10,
          delta=0.0, mixing=0.5, ccs=False, criterion="soa", history=None):
    """The solver loop.

    ``criterion="soa"`` follows ``CCM/soa/coupled_cluster.py:440-575``: the
    energy test ``|dE| / max(1, |E|) < eps`` and pulsed DIIS every
    ``max_diis`` steps.  ``criterion="numpy"`` follows
    ``CCM/coupled_cluster.py:547-687``: the test ``|dE| / |E| < eps`` (or both
    energies exactly zero) and no DIIS (that branch never fires there).
    Returns ``(E_corr, t1, t2, iterations, status)`` with status ``"converged"``,
    ``"max_iter"`` or ``"diverged"``.
    """
    H = Hamiltonian(fock_mats, two_body_int)
    t1 = t1_init(H, delta) if t1initial is None else np.array(t1initial, dtype=np.float64)
    t2 = np.zeros_like(H.v_pphh) if (ccs or t1initial is not None) else t2_init(H, delta)
    use_diis = criterion == "soa" and max_diis > 0
    if use_diis:
        hist1, hist2, errs = [t1.copy()], [t2.copy()], []
    prev = energy(H, t1, t2)
    e = prev
    for it in range(maxSteps):
        old1, old2 = t1, t2
        r = ppph_intermediates(H.ppph_idx, H.ppph_val, t1, t2)
        t1 = mixing * t1 + (1.0 - mixing) * t1_step(H, t1, t2, r)
        if not ccs:
            t2 = mixing * t2 + (1.0 - mixing) * t2_step(H, old1, t2, r)
        e = energy(H, t1, t2)
        if history is not None:
            history.append(e)
        if criterion == "soa":
            done = abs(e - prev) / max(1.0, abs(e)) < eps
        else:
            done = (e == 0 and prev == 0) or abs(e - prev) / abs(e) < eps
        if done:
            return e, t1, t2, it + 1, "converged"
        if use_diis:
            hist1.append(t1.copy()); hist2.append(t2.copy())
            errs.append(np.concatenate([(t1 - old1).ravel(), (t2 - old2).ravel()]))
            if len(errs) == max_diis:
                n = len(errs)
                B = np.array([[float(np.dot(errs[a], errs[b])) for b in range(n)] for a in range(n)])
                B = B / (np.abs(B).max() + 1e-16)
                A = -np.ones((n + 1, n + 1)); A[:n, :n] = B; A[n, n] = 0.0
                rhs = np.zeros(n + 1); rhs[n] = -1.0
                try:
                    c = np.linalg.solve(A, rhs)[:n]
                    t1 = sum(c[k] * hist1[k + 1] for k in range(n))
                    if not ccs:
                        t2 = sum(c[k] * hist2[k + 1] for k in range(n))
                except np.linalg.LinAlgError:
                    pass
                hist1, hist2, errs = [t1.copy()], [t2.copy()], []
        if abs(e) > 1e10 or np.isnan(e):
            return e, t1, t2, it + 1, "diverged"
        prev = e
    return e, t1, t2, maxSteps, "max_iter"
