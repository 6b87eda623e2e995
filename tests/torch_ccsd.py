"""Plain FP64 PyTorch CCSD, differentiable -- test infrastructure.

The reference's factorised residuals (``CCM/coupled_cluster.py:342-545``,
diagram table shared with ``oracle.ccsd_oracle``) written with
``torch.einsum`` and ``index_put`` so that autograd can differentiate the
converged energy with respect to the couplings, and the residual with
respect to the amplitudes.  Used to check the hand-written adjoint.
"""
import numpy as np
import torch

from oracle.ccsd_oracle import DIAGRAMS


def _pab(x):
    return x - x.permute(1, 0, 2, 3)


def _pij(x):
    return x - x.permute(0, 1, 3, 2)


_PERM = {"": lambda x: x, "ab": _pab, "ij": _pij, "abij": lambda x: _pij(_pab(x))}


def _d(name, ops):
    coef, spec, names, perm = DIAGRAMS[name]
    return coef * _PERM[perm](torch.einsum(spec, *[ops[n] for n in names]))


class TorchHam:
    """H(v, w) = H_kin + v * H_v + w * H_w with torch scalars v, w.

    ``parts`` are the builder outputs at (kinetic only), (unit contact, no
    kinetic) and (unit three-body contact, no kinetic)."""

    def __init__(self, parts, v, w, device="cpu"):
        (ek, fk, tk), (ev, fv, tv), (ew, fw, tw) = parts
        T = lambda a: torch.as_tensor(np.asarray(a, dtype=np.float64), device=device)  # noqa: E731
        self.e_ref = ek + v * ev + w * ew
        self.f = [T(a) + v * T(b) + w * T(c) for a, b, c in zip(fk, fv, fw)]
        dense = lambda blk: T(blk.to_dense() if hasattr(blk, "to_dense") else blk)  # noqa: E731
        self.v = {}
        for k, name in enumerate(("v_pphh", "v_phph", "v_phhh", "v_hhhh")):
            self.v[name] = dense(tk[2 + k]) + v * dense(tv[2 + k]) + w * dense(tw[2 + k])
        rows = [np.asarray(x, dtype=np.float64).reshape(-1, 5) for x in (tk[0], tv[0], tw[0])]
        idx = np.concatenate([r[:, :4] for r in rows]).astype(np.int64)
        vals = torch.cat([T(rows[0][:, 4]), v * T(rows[1][:, 4]), w * T(rows[2][:, 4])])
        self.pppp = (torch.as_tensor(idx, device=device), vals)
        for x in (tk[1], tv[1], tw[1]):
            assert len(np.asarray(x).reshape(-1, 5)) == 0, "v_ppph not supported here"

    def ops(self, t1, t2):
        f_pp, f_ph, f_hh = self.f
        return dict(f_pp=f_pp, f_ph=f_ph, f_hh=f_hh, t1=t1, t2=t2, **self.v)


def residuals(H, t1, t2):
    """(R1, R2, X1pp, X1hh, X2pp, X2hh): the H1/H2 of t1Iter/t2Iter."""
    o = H.ops(t1, t2)
    nz = {k: bool(torch.any(v != 0)) for k, v in H.v.items()}
    h1 = o["f_ph"] + _d("dgram_ck_acik", o)
    xhh1 = -o["f_hh"] + _d("dgram_ck_ci", o)
    xpp1 = o["f_pp"] + _d("dgram_ck_ak", o)
    if nz["v_phph"]:
        h1 = h1 + _d("dgram_akci_ck", o)
    if nz["v_phhh"]:
        h1 = h1 + _d("dgram_cikl_cakl", o)
        xhh1 = xhh1 + _d("dgram_bijk_bj", o)
    if nz["v_pphh"]:
        h1 = h1 + _d("dgram_cdkl_ck_dali", o)
        xhh1 = xhh1 + _d("dgram_cdlk_cdli", o) + _d("dgram_cdlk_cl_di", o)
        xpp1 = xpp1 + _d("dgram_dckl_dakl", o) + _d("dgram_cdkl_dk_al", o)
    r1 = h1 + xpp1 @ t1 + t1 @ xhh1
    h2 = o["v_pphh"] + _d("dgram_klij_abkl", o) + _d("dgram_klij_ak_bl", o)
    if nz["v_phph"]:
        h2 = h2 + _d("dgram_bkcj_acik", o) + _d("dgram_bkci_ak_cj", o)
    if nz["v_phhh"]:
        for n in ("dgram_bkij_ak", "dgram_cikl_ck_ablj", "dgram_cikl_al_bcjk", "dgram_cjkl_ci_abkl",
                  "dgram_cjkl_ci_ak_bl"):
            h2 = h2 + _d(n, o)
    if nz["v_pphh"]:
        for n in ("dgram_cdkl_acik_dblj", "dgram_cdkl_cdij_abkl", "dgram_cdkl_ci_dj_abkl",
                  "dgram_cdkl_ak_bl_cdij", "dgram_cdkl_ci_bl_adkj", "dgram_cdkl_ci_ak_dj_bl"):
            h2 = h2 + _d(n, o)
    xhh2 = -o["f_hh"] + _d("dgram_ck_cj", o)
    xpp2 = o["f_pp"] + _d("dgram_ck_bk", o)
    if nz["v_pphh"]:
        xhh2 = xhh2 + _d("dgram_cdkl_cdjl", o) + _d("dgram_cdlk_cl_dj", o)
        xpp2 = xpp2 + _d("dgram_cdkl_bdkl", o) + _d("dgram_cdlk_dk_bl", o)
    idx, val = H.pppp
    a, b, c, d = idx.T
    l1 = torch.zeros_like(t2).index_put((a, b), val[:, None, None] * t2[c, d], accumulate=True)
    l2 = torch.zeros_like(t2).index_put((a, b), val[:, None, None] * (t1[c, :, None] * t1[d, None, :]),
                                        accumulate=True)
    h2 = h2 + 0.5 * l1 + 0.5 * _pij(l2)
    h2 = h2 + _pab(torch.einsum("bc,acij->abij", xpp2, t2)) + _pij(torch.einsum("kj,abik->abij", xhh2, t2))
    return r1, h2, xpp1, xhh1, xpp2, xhh2


def energy(H, t1, t2):
    e = torch.sum(H.f[1] * t1) + 0.25 * torch.sum(H.v["v_pphh"] * t2)
    return e + 0.5 * torch.einsum("abij,ai,bj->", H.v["v_pphh"], t1, t1)


def solve(H, eps=1e-12, max_steps=3000, mixing=0.5):
    """Jacobi + mixing to |dE|/|E| < eps, keeping the autograd graph."""
    f_pp, f_ph, f_hh = H.f
    ep, eh = torch.diagonal(f_pp), torch.diagonal(f_hh)
    t1 = f_ph / (eh[None, :] - ep[:, None])
    den2 = -ep[:, None, None, None] - ep[None, :, None, None] + eh[None, None, :, None] + eh[None, None, None, :]
    t2 = H.v["v_pphh"] / den2
    prev = energy(H, t1, t2)
    e = prev
    for it in range(max_steps):
        r1, r2, xpp1, xhh1, xpp2, xhh2 = residuals(H, t1, t2)
        d1 = -(torch.diagonal(xpp1)[:, None] + torch.diagonal(xhh1)[None, :])
        dp, dh = torch.diagonal(xpp2), torch.diagonal(xhh2)
        d2 = -(dp[:, None, None, None] + dp[None, :, None, None] + dh[None, None, :, None] + dh[None, None, None, :])
        t1, t2 = (mixing * t1 + (1 - mixing) * (t1 + r1 / d1), mixing * t2 + (1 - mixing) * (t2 + r2 / d2))
        e = energy(H, t1, t2)
        if abs(float(e.detach() - prev.detach())) < eps * abs(float(e.detach())):
            return e, t1, t2, it + 1
        prev = e
    return e, t1, t2, max_steps
