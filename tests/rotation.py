"""Orbital rotations of a normal-ordered Hamiltonian (test helper).

A rotation within the particle space and, separately, within the hole space
(as a Hartree-Fock or any other basis change that keeps the reference
determinant) leaves the CCSD correlation energy unchanged, while every block
of the Hamiltonian becomes dense."""
import numpy as np


def _dense_rows(rows, shape):
    out = np.zeros(shape)
    r = np.asarray(rows, dtype=np.float64).reshape(-1, 5)
    if len(r):
        np.add.at(out, tuple(r[:, :4].astype(np.int64).T), r[:, 4])
    return out


def rotate(fock, two, seed):
    f_pp, f_ph, f_hh = [np.asarray(f) for f in fock]
    p, h = f_ph.shape
    rng = np.random.default_rng(seed)
    up = np.linalg.qr(rng.standard_normal((p, p)))[0]
    uh = np.linalg.qr(rng.standard_normal((h, h)))[0]
    fr = [up.T @ f_pp @ up, up.T @ f_ph @ uh, uh.T @ f_hh @ uh]
    blocks = [_dense_rows(two[0], (p, p, p, p)), _dense_rows(two[1], (p, p, p, h))]
    blocks += [b.to_dense() if hasattr(b, "to_dense") else np.asarray(b) for b in two[2:]]
    kinds = ["pppp", "ppph", "pphh", "phph", "phhh", "hhhh"]
    out = []
    for blk, kind in zip(blocks, kinds):
        us = [up if c == "p" else uh for c in kind]
        out.append(np.einsum(blk, [0, 1, 2, 3], us[0], [0, 4], us[1], [1, 5], us[2], [2, 6], us[3], [3, 7],
                             [4, 5, 6, 7], optimize=True))
    return fr, out


def rows_of(dense):
    """The reference's sparse row-list form [k0, k1, k2, k3, val] of a 4-D block."""
    idx = np.argwhere(dense != 0)
    return np.concatenate([idx.astype(np.float64), dense[tuple(idx.T)][:, None]], 1)
