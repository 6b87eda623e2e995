"""Plane-wave (momentum-basis) inputs for the lattice contact Hamiltonian.

The reference solves the lattice Hamiltonian in the position basis
(``lattice.py``); its CCSD entry point takes any Hamiltonian in its list
conventions.  This module builds the same Hamiltonian in the plane-wave basis
of the periodic L^3 lattice -- the exact Fourier transform of the
position-basis builder of :mod:`nulattice_b200.hamiltonian` with couplings
``(vT1, vS1, w3)`` -- and normal-orders it with respect to closed momentum
shells, in the input layout of :func:`nulattice_b200.ccsd.ccsd_solver`:

* single-particle index ``((nx*L + ny)*L + nz)*4 + 2*tz + sz`` with the
  momentum ``2 pi n / L``;
* kinetic energy ``sum_d (2 - 2 cos(2 pi n_d / L))`` on the diagonal, every
  diagonal entry present (also the zeros), so the Fock matrix receives the
  hole traces on its whole diagonal;
* two-body ``<ij||kl> = v_loc[s_i s_j s_k s_l] / L^3`` when the momenta add
  up modulo L, ``v_loc`` the antisymmetrised on-site spin-isospin tensor of
  ``lattice.py:421-627`` (:func:`hamiltonian._local_contact_channels`);
* three-body ``<ijk||lmn> = w3 sgn(perm) / L^6`` when the spin-isospin labels
  of the ket are a permutation of the bra's (all distinct) and the momenta
  add up.  With every hole momentum filled in all four spin-isospin states
  its normal-ordered parts are, for ``n_k`` hole momenta: ``E_3 = (1/6)
  #(ordered hole triples with distinct labels) w3 / L^6 = 4 n_k^3 w3 / L^6``,
  ``f_3 = (1/2) #(ordered hole pairs with labels distinct from each other and
  from the state) w3 / L^6`` on the diagonal, and a two-body part equal to an
  SU(4) contact of strength ``2 n_k w3 / L^3`` (the sums of
  ``CCM/three_body_utils.py:229-377`` evaluated in closed form).

The normal ordering itself follows ``CCM/coupled_cluster.py:21-317`` as in
:func:`hamiltonian.normal_ordered_hamiltonian`: Fock = kinetic + hole trace
of the two-body part + ``f_3``; blocks = two-body + the normal-ordered
three-body part; ``E_ref`` = trace of the hole Fock block minus half the
hole-hole block plus ``E_3``.

Unlike the position basis, the plane-wave ``v_pphh``, ``v_phph`` and
``v_phhh`` blocks are not zero, and the one-body part is diagonal, so no
label survives the structure test and :func:`ccsd_solver` uses its general
engine for these inputs.
"""
from __future__ import annotations

import numpy as np

from . import hamiltonian as _ham

UNIT_SHELL = [(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)]


def momentum_holes(L, A):
    """Closed momentum shells: A=4 fills n=0, A=28 also the six unit momenta
    (all four spin-isospin states each)."""
    if A == 4:
        ks = UNIT_SHELL[:1]
    elif A == 28:
        ks = UNIT_SHELL
    else:
        raise ValueError("momentum_holes: A must be 4 or 28")
    out = []
    for k in ks:
        for tz in range(2):
            for sz in range(2):
                out.append([k[0] % L, k[1] % L, k[2] % L, tz, sz])
    # the six unit momenta are distinct only for L > 2
    uniq = {tuple(x) for x in out}
    if len(uniq) != len(out):
        raise ValueError("momentum_holes: the unit shell needs L > 2")
    return out


def _vloc_tensor(vT1, vS1):
    """Full antisymmetric on-site tensor v[s1, s2, s3, s4] (4^4 entries)."""
    v = np.zeros((4, 4, 4, 4))
    for p, q, r, s, val in _ham._local_contact_channels(vT1, vS1):
        p, q, r, s = int(p), int(q), int(r), int(s)
        v[p, q, r, s] = val
        v[q, p, r, s] = -val
        v[p, q, s, r] = -val
        v[q, p, s, r] = val
    return v


def two_body_rows(vT1, vS1, L, k_full=None, is_hole=None):
    """Rows ``[p, q, r, s, <pq||rs>]`` (p<q, r<s) of the contact in the
    plane-wave basis: momentum conservation modulo L, value ``v_loc / L^3``.

    ``k_full`` (bool per total momentum K, with ``is_hole`` per state): at
    the K where it is False only rows whose bra and ket pairs both hold a
    hole are emitted (the p-h blocks need every K; the pure-particle and
    three-particle rows there only ever meet amplitudes that vanish)."""
    n = 4 * L ** 3
    v = _vloc_tensor(vT1, vS1) / L ** 3
    i, j = np.triu_indices(n, 1)
    si, sj = i % 4, j % 4
    ki, kj = i // 4, j // 4

    def kvec(k):
        return k // (L * L), (k // L) % L, k % L

    xi, yi, zi = kvec(ki)
    xj, yj, zj = kvec(kj)
    K = (((xi + xj) % L) * L + (yi + yj) % L) * L + (zi + zj) % L
    order = np.argsort(K, kind="stable")
    Ks = K[order]
    bounds = np.searchsorted(Ks, np.arange(L ** 3 + 1))
    rows = []
    for k in range(L ** 3):
        sel = order[bounds[k]:bounds[k + 1]]
        if k_full is not None and not k_full[k]:
            sel = sel[is_hole[i[sel]] | is_hole[j[sel]]]
        if len(sel) == 0:
            continue
        a, b = i[sel], j[sel]
        sa, sb = si[sel], sj[sel]
        val = v[sa[:, None], sb[:, None], sa[None, :], sb[None, :]]
        bi, ki2 = np.nonzero(val)
        rows.append(np.stack([a[bi], b[bi], a[ki2], b[ki2], val[bi, ki2]], 1))
    return np.concatenate(rows) if rows else np.zeros((0, 5))


def kinetic_rows(L):
    """Diagonal rows ``[p, p, sum_d (2 - 2 cos(2 pi n_d / L))]``, zeros kept."""
    n = 4 * L ** 3
    s = np.arange(n)
    k = s // 4
    t = np.zeros(n)
    for m in (k // (L * L), (k // L) % L, k % L):
        t += 2.0 - 2.0 * np.cos(2.0 * np.pi * m / L)
    return np.stack([s, s, t], 1).astype(np.float64)


def plane_wave_hamiltonian(L, holes, vT1, vS1, w3=0.0, dense=True, prune=True):
    """Normal-ordered plane-wave Hamiltonian, returned like
    :func:`hamiltonian.normal_ordered_hamiltonian`:
    ``(E_ref, [f_pp, f_ph, f_hh], [v_pppp, v_ppph, v_pphh, v_phph, v_phhh, v_hhhh])``.

    ``holes`` are ``[nx, ny, nz, tz, sz]`` rows (:func:`momentum_holes`);
    every hole momentum must hold all four spin-isospin states.  ``prune``
    leaves out the v_pppp / v_ppph rows at total momenta no hole pair has
    (they never meet a non-zero amplitude; ``prune=False`` keeps every row)."""
    holes = np.asarray(holes, dtype=np.int64).reshape(-1, 5)
    hole, part = _ham.ph_split(holes, L)
    h, p = len(hole), len(part)
    n = 4 * L ** 3
    hk = {}
    for x in holes:
        hk.setdefault(tuple(int(c) for c in x[:3]), set()).add(2 * int(x[3]) + int(x[4]))
    if any(len(s) != 4 for s in hk.values()):
        raise ValueError("plane_wave_hamiltonian: every hole momentum needs all four spin-isospin states")
    n_k = len(hk)
    is_hole = np.zeros(n, bool); is_hole[hole] = True
    loc = np.zeros(n, np.int64); loc[hole] = np.arange(h); loc[part] = np.arange(p)

    shapes = {"pphh": (p, p, h, h), "phph": (p, h, p, h), "phhh": (p, h, h, h), "hhhh": (h, h, h, h)}
    # Closed shells: every hole momentum is full, so t1 vanishes by momentum
    # conservation and t2[a,b,i,j] lives at the total momenta K of hole
    # pairs.  v_pppp and v_ppph rows at any other K only multiply vanishing
    # amplitudes, and are left out (exact: their products are zeros).
    kfull = np.zeros(L ** 3, bool)
    hkeys = list(hk)
    for k1 in hkeys:
        for k2 in hkeys:
            kk = [(k1[d] + k2[d]) % L for d in range(3)]
            kfull[(kk[0] * L + kk[1]) * L + kk[2]] = True
    if not prune:
        kfull[:] = True
    b = _ham._sort_two_body(two_body_rows(vT1, vS1, L, kfull, is_hole), is_hole, loc)
    # normal-ordered three-body part: an SU(4) contact of strength 2 n_k w3 / L^3
    if w3 != 0.0:
        v3 = 2.0 * n_k * w3 / L ** 3
        b3 = _ham._sort_two_body(two_body_rows(v3, v3, L, kfull, is_hole), is_hole, loc)
        # E_3 and the diagonal f_3 from the counts of distinct-label hole tuples
        n_h = 4 * n_k
        e3 = (n_h * (n_h - n_k) * (n_h - 2 * n_k)) / 6.0 * w3 / L ** 6
        f3 = 0.5 * (3 * n_k) * (2 * n_k) * w3 / L ** 6
    else:
        b3, e3, f3 = None, 0.0, 0.0

    kin = kinetic_rows(L)
    T = np.zeros(n)
    T[kin[:, 0].astype(np.int64)] = kin[:, 2]
    two = {k: _ham._canonical_block(shapes[k], *b[k]) for k in shapes}
    coo = {k: (_ham._canonical_block(shapes[k], *b[k], add=b3[k]) if b3 is not None else two[k]) for k in shapes}
    # Fock: kinetic + hole trace of the two-body part (diagonal) + f_3
    f_pp = np.diag(T[part]) + _ham._trace_13(shapes["phph"], *two["phph"], (p, p))
    f_ph = np.zeros((p, h)) + _ham._trace_13(shapes["phhh"], *two["phhh"], (p, h))
    f_hh = np.diag(T[hole]) + _ham._trace_13(shapes["hhhh"], *two["hhhh"], (h, h))
    f_pp[np.diag_indices(p)] += f3
    f_hh[np.diag_indices(h)] += f3
    rows = {}
    for k in ("pppp", "ppph"):
        r = np.concatenate([b[k][0].astype(np.float64), b[k][1][:, None]], 1)
        if b3 is not None and len(b3[k][1]):
            r = np.concatenate([r, np.concatenate([b3[k][0].astype(np.float64), b3[k][1][:, None]], 1)])
        rows[k] = r
    hi, hv = coo["hhhh"]
    diag = (hi[:, 0] == hi[:, 2]) & (hi[:, 1] == hi[:, 3])
    e_ref = float(np.trace(f_hh) - 0.5 * np.sum(hv[diag]) + e3)
    if dense:
        blocks = []
        for k in ("pphh", "phph", "phhh", "hhhh"):
            d = np.zeros(shapes[k])
            idx, val = coo[k]
            if len(val):
                d[tuple(idx.T)] = val
            blocks.append(d)
    else:
        blocks = [_ham.Block(shapes[k], *coo[k]) for k in ("pphh", "phph", "phhh", "hhhh")]
    return e_ref, [f_pp, f_ph, f_hh], [rows["pppp"], rows["ppph"]] + blocks
