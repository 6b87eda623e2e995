"""Lattice Hamiltonian builders and normal ordering (host side, numpy).

These produce the inputs of :func:`nulattice_b200.ccsd.ccsd_solver` in the
reference's conventions, without the reference installed:

* single-particle index ``((x*L + y)*L + z)*4 + 2*tz + sz``
  (``lattice.py:119-151``),
* kinetic energy: dimensionless negative Laplacian, diagonal 6 and ``-1`` for
  each periodic nearest-neighbour hop (``lattice.py:306-418``),
* on-site two-body contact with T=1 / S=1 couplings ``vT1``, ``vS1``
  (``lattice.py:421-627``),
* on-site diagonal three-body contact ``<pqr|W|pqr> = w3`` (``lattice.py:678-752``),
* hole / particle split (``lattice.py:937-954``),
* sorting into the p/h blocks with all antisymmetric permutations
  (``CCM/coupled_cluster.py:99-263``), Fock matrices (``:21-97``), reference
  energy (``:288-317``) and the three-body normal-ordered one- and two-body
  parts (``CCM/three_body_utils.py:6-377``, ``CCM/coupled_cluster.py:752-832``).

Energies are in the reference's unit ``hbar^2 / (2 M a^2)`` (``phys_unit``).
The builders here are vectorised; the sparse blocks are returned as row
arrays ``[k0, k1, k2, k3, val]`` (the reference's sparse-list convention) and
the dense blocks either densely (reference-compatible, ``dense=True``) or as
:class:`Block` COO objects, which :func:`ccsd_solver` also accepts.
"""
from __future__ import annotations

import numpy as np

HBARC = 197.3269804  # MeV fm
MASS = 938.92  # MeV


def phys_unit(a_lat: float) -> float:
    """Energy unit hbar^2/(2 M a^2) in MeV (``lattice.py:57-61``)."""
    return 0.5 * HBARC ** 2 / (MASS * a_lat ** 2)


def state_index(x, y, z, tz, sz, L):
    return ((np.asarray(x) * L + np.asarray(y)) * L + np.asarray(z)) * 4 + 2 * np.asarray(tz) + np.asarray(sz)


def kinetic_rows(L):
    """Rows ``[p, q, T_pq]`` of the lattice kinetic energy (``lattice.py:306-418``).

    Every ordered nearest-neighbour pair appears once per hop direction, so at
    ``L == 2`` the +1 and -1 neighbours coincide and their entries add up.
    """
    n = 4 * L ** 3
    idx = np.arange(n)
    site, loc = idx // 4, idx % 4
    x, y, z = site // (L * L), (site // L) % L, site % L
    rows = [np.stack([idx, idx, np.full(n, 6.0)], 1)]
    for d in range(3):
        c = [x, y, z]
        c[d] = (c[d] + 1) % L
        nb = ((c[0] * L + c[1]) * L + c[2]) * 4 + loc
        rows.append(np.stack([idx, nb, -np.ones(n)], 1))
        rows.append(np.stack([nb, idx, -np.ones(n)], 1))
    return np.concatenate(rows).astype(np.float64)


def _local_contact_channels(vT1, vS1):
    """Antisymmetrised on-site matrix elements <pq||rs> for local states p<q, r<s
    (spin-isospin labels 0..3 = 2*tz + sz), ``lattice.py:555-610``."""
    out = []
    for p in range(4):
        for q in range(p + 1, 4):
            for r in range(4):
                for s in range(r + 1, 4):
                    tp, sp_, tq, sq = p // 2, p % 2, q // 2, q % 2
                    tr, sr, ts, ss = r // 2, r % 2, s // 2, s % 2
                    if tp + tq != tr + ts or sp_ + sq != sr + ss:
                        continue
                    if tp == tq:
                        val = vT1
                    elif sp_ == sq:
                        val = vS1
                    elif p == r:
                        val = 0.5 * (vS1 + vT1)
                    else:
                        val = 0.5 * (vS1 - vT1)
                    out.append((p, q, r, s, val))
    return np.array(out, dtype=np.float64)


def contact_rows(vT1, vS1, L):
    """Rows ``[p, q, r, s, <pq||rs>]`` (p<q, r<s) of the on-site contact."""
    ch = _local_contact_channels(vT1, vS1)
    base = (np.arange(L ** 3) * 4)[:, None]
    cols = [(base + ch[None, :, k]).ravel() for k in range(4)]
    return np.stack(cols + [np.tile(ch[:, 4], L ** 3)], 1)


def three_body_rows(w3, L):
    """Rows ``[p, q, r, p, q, r, w3]`` (p<q<r on one site), ``lattice.py:678-752``."""
    trip = np.array([(a, b, c) for a in range(4) for b in range(a + 1, 4) for c in range(b + 1, 4)])
    base = (np.arange(L ** 3) * 4)[:, None]
    cols = [(base + trip[None, :, k]).ravel() for k in range(3)]
    return np.stack(cols + cols + [np.full(len(cols[0]), float(w3))], 1)


def ph_split(holes, L):
    """Hole indices in the given order and the remaining particle indices
    ascending (``lattice.py:937-954``)."""
    holes = np.asarray(holes, dtype=np.int64).reshape(-1, 5)
    hole = state_index(holes[:, 0], holes[:, 1], holes[:, 2], holes[:, 3], holes[:, 4], L)
    part = np.setdiff1d(np.arange(4 * L ** 3), hole)
    return hole.astype(np.int64), part.astype(np.int64)


class Block:
    """A COO tensor block: ``indices`` (N, rank) int64, ``values`` (N,) float64.

    Repeated keys are summed when the block is densified or uploaded.
    """

    def __init__(self, shape, indices, values):
        self.shape = tuple(int(s) for s in shape)
        self.indices = np.asarray(indices, dtype=np.int64).reshape(-1, len(self.shape))
        self.values = np.asarray(values, dtype=np.float64).reshape(-1)

    def to_dense(self):
        out = np.zeros(self.shape)
        if len(self.values):
            np.add.at(out, tuple(self.indices.T), self.values)
        return out

    def __len__(self):
        return len(self.values)


def _perm_sign(order):
    order = list(order)
    s = 1
    for i in range(len(order)):
        for j in range(i + 1, len(order)):
            if order[i] > order[j]:
                s = -s
    return s


def _sort_two_body(rows, is_hole, loc):
    """Distribute <pq||rs> rows (p<q, r<s) over the six p/h blocks with all the
    antisymmetric permutations (``CCM/coupled_cluster.py:140-260``).

    Returns ``{block: (indices (N,4), values (N,))}`` where the index order of
    each block is the reference's: pppp [a,b,c,d], ppph [a,b,c,k],
    pphh [a,b,i,j], phph [a,i,b,j], phhh [a,i,j,k], hhhh [i,j,k,l].
    """
    i1, i2, i3, i4 = (rows[:, k].astype(np.int64) for k in range(4))
    val = rows[:, 4]
    # put particles first in ket and bra (one swap = one sign flip)
    sk = np.where(is_hole[i1] & ~is_hole[i2], -1.0, 1.0)
    k1 = np.where(sk < 0, i2, i1); k2 = np.where(sk < 0, i1, i2)
    sb = np.where(is_hole[i3] & ~is_hole[i4], -1.0, 1.0)
    b1 = np.where(sb < 0, i4, i3); b2 = np.where(sb < 0, i3, i4)
    nk = is_hole[k1].astype(int) + is_hole[k2].astype(int)
    nb = is_hole[b1].astype(int) + is_hole[b2].astype(int)
    base = val * sk * sb
    L = [loc[k1], loc[k2], loc[b1], loc[b2]]
    out = {}

    def emit(name, mask, perms):
        idx, vals = [], []
        for order, sign in perms:
            idx.append(np.stack([L[o][mask] for o in order], 1))
            vals.append(sign * base[mask])
        out[name] = (np.concatenate(idx) if idx else np.zeros((0, 4), np.int64),
                     np.concatenate(vals) if vals else np.zeros(0))

    four = [((0, 1, 2, 3), 1.0), ((1, 0, 2, 3), -1.0), ((0, 1, 3, 2), -1.0), ((1, 0, 3, 2), 1.0)]
    emit("pppp", (nk == 0) & (nb == 0), four)
    emit("ppph", (nk == 0) & (nb == 1), [((0, 1, 2, 3), 1.0), ((1, 0, 2, 3), -1.0)])
    emit("pphh", (nk == 0) & (nb == 2), four)
    emit("phph", (nk == 1) & (nb == 1), [((0, 1, 2, 3), 1.0)])
    emit("phhh", (nk == 1) & (nb == 2), [((0, 1, 2, 3), 1.0), ((0, 1, 3, 2), -1.0)])
    emit("hhhh", (nk == 2) & (nb == 2), four)
    return out


def _dense_assign(shape, idx, val):
    """Dense block filled by assignment (repeated keys: the last write wins, as
    the reference's ``vint[indx] = ...``)."""
    out = np.zeros(shape)
    if len(val):
        out[tuple(idx.T)] = val
    return out


def _three_body_no2b(rows, is_hole, loc, p, h):
    """Normal-ordered contributions of a diagonal three-body force.

    For ``<xyz|W|xyz>`` rows, the reference's block sorting
    (``CCM/three_body_utils.py:6-156``) followed by ``get_3NF_fock`` (``:248-284``),
    ``get_3NF_tbme`` (``:287-377``) and ``get_3NF_Eref`` (``:229-245``) reduces to
    sums over the hole members of each triple.  Returns
    ``(dE_ref, df_pp, df_hh, {block: (idx, val)})``.
    """
    df_pp = np.zeros((p, p)); df_hh = np.zeros((h, h))
    blocks = {"pppp": [], "phph": [], "hhhh": []}
    de = 0.0
    trip = rows[:, :3].astype(np.int64)
    w = rows[:, 6]
    nh = is_hole[trip].sum(1)
    for n in range(len(w)):
        s = trip[n]
        hs = [q for q in s if is_hole[q]]
        ps = [q for q in s if not is_hole[q]]
        v = w[n]
        if nh[n] == 3:
            de += v  # 36 permutations * v / 6, one sixth per diagonal permutation
            # f_hh[x,x] += 1/2 * sum over the two orderings of the other two holes * 2 perms
            for x in s:
                df_hh[loc[x], loc[x]] += v
            # v_hhhh[m,n,l,k] from pairs with the third hole contracted
            for x in range(3):
                others = [s[y] for y in range(3) if y != x]
                a, b = loc[others[0]], loc[others[1]]
                blocks["hhhh"] += [(a, b, a, b, v), (b, a, a, b, -v), (a, b, b, a, -v), (b, a, b, a, v)]
        elif nh[n] == 2:
            a = loc[ps[0]]
            df_pp[a, a] += v
            for x in hs:
                y = [q for q in hs if q != x][0]
                blocks["phph"].append((a, loc[y], a, loc[y], v))
        elif nh[n] == 1:
            a, b = loc[ps[0]], loc[ps[1]]
            blocks["pppp"] += [(a, b, a, b, v), (b, a, a, b, -v), (a, b, b, a, -v), (b, a, b, a, v)]
    conv = {}
    for k, lst in blocks.items():
        arr = np.array(lst, dtype=np.float64).reshape(-1, 5)
        conv[k] = (arr[:, :4].astype(np.int64), arr[:, 4])
    return de, df_pp, df_hh, conv


def _canonical_block(shape, idx, val, add=None):
    """The non-zero entries, in lexicographic index order, of the dense block
    that ``_dense_assign(shape, idx, val)`` followed by ``np.add.at`` of the
    entries ``add = (idx, val)`` would hold: the last write of a repeated
    two-body key wins, the added entries are summed after it in their order,
    and zeros are dropped.  Built without the dense block (4.4 GB for v_pphh
    at L=6, A=28)."""
    shape = tuple(int(x) for x in shape)
    idx = np.asarray(idx, np.int64).reshape(-1, len(shape))
    val = np.asarray(val, np.float64).reshape(-1)
    key = np.ravel_multi_index(tuple(idx.T), shape) if len(val) else np.zeros(0, np.int64)
    uk, first = np.unique(key[::-1], return_index=True)
    v = val[len(key) - 1 - first] if len(val) else np.zeros(0)
    if add is not None and len(add[1]):
        ak = np.ravel_multi_index(tuple(np.asarray(add[0], np.int64).T), shape)
        allk = np.concatenate([uk, ak])
        allv = np.concatenate([v, np.asarray(add[1], np.float64)])
        order = np.argsort(allk, kind="stable")   # the two-body value first, then the sums in order
        ks, vs = allk[order], allv[order]
        first_of = np.concatenate(([True], ks[1:] != ks[:-1]))
        seg = np.cumsum(first_of) - 1
        v = np.zeros(int(first_of.sum()))
        np.add.at(v, seg, vs)                       # in order, as the dense path's np.add.at
        uk = ks[first_of]
    keep = v != 0
    return np.stack(np.unravel_index(uk[keep], shape), 1).astype(np.int64), v[keep]


def _trace_13(shape, idx, val, out_shape):
    """sum_i X[a, i, b, i] of a COO block (``einsum("aibi->ab")``)."""
    out = np.zeros(out_shape)
    m = idx[:, 1] == idx[:, 3]
    if m.any():
        np.add.at(out, (idx[m, 0], idx[m, 2]), val[m])
    return out


def normal_ordered_hamiltonian(L, holes, vT1, vS1, w3=0.0, dense=True, kinetic=1.0):
    """``get_norm_ordered_ham`` for the lattice contact Hamiltonian
    (``CCM/coupled_cluster.py:752-832`` with ``sparse=True, NO2B=True``).

    Couplings are in the reference's unit hbar^2/(2Ma^2).  Returns
    ``(E_ref, [f_pp, f_ph, f_hh], [v_pppp, v_ppph, v_pphh, v_phph, v_phhh, v_hhhh])``
    where ``v_pppp``/``v_ppph`` are ``(N,5)`` row arrays and the other four blocks
    are dense arrays (``dense=True``) or :class:`Block` objects.
    ``kinetic`` scales the kinetic energy; the Fock traces are still added
    only where a kinetic entry exists, so ``kinetic=0`` gives the derivative
    of every block with respect to the couplings (all blocks are linear in
    vT1, vS1 and w3).
    """
    hole, part = ph_split(holes, L)
    h, p = len(hole), len(part)
    n = 4 * L ** 3
    is_hole = np.zeros(n, bool); is_hole[hole] = True
    loc = np.zeros(n, np.int64); loc[hole] = np.arange(h); loc[part] = np.arange(p)

    b = _sort_two_body(contact_rows(vT1, vS1, L), is_hole, loc)
    shapes = {"pphh": (p, p, h, h), "phph": (p, h, p, h), "phhh": (p, h, h, h), "hhhh": (h, h, h, h)}
    if not dense:
        return _normal_ordered_sparse(L, b, shapes, hole, part, is_hole, loc, p, h, w3, kinetic)
    dense2 = {k: _dense_assign(shapes[k], *b[k]) for k in shapes}

    # Fock matrices: kinetic entry plus the hole trace of the two-body blocks,
    # only where a kinetic entry exists (CCM/coupled_cluster.py:56-95)
    T = np.zeros((n, n)); has_t = np.zeros((n, n), bool)
    kr = kinetic_rows(L)
    ti, tj = kr[:, 0].astype(np.int64), kr[:, 1].astype(np.int64)
    np.add.at(T, (ti, tj), float(kinetic) * kr[:, 2])
    has_t[ti, tj] = True
    f_pp = T[np.ix_(part, part)] + np.einsum("aibi->ab", dense2["phph"])
    f_ph = T[np.ix_(part, hole)] + np.einsum("aibi->ab", dense2["phhh"])
    f_hh = T[np.ix_(hole, hole)] + np.einsum("aibi->ab", dense2["hhhh"])
    f_pp = np.where(has_t[np.ix_(part, part)], f_pp, 0.0)
    f_ph = np.where(has_t[np.ix_(part, hole)], f_ph, 0.0)
    f_hh = np.where(has_t[np.ix_(hole, hole)], f_hh, 0.0)

    sparse_rows = {k: np.concatenate([b[k][0].astype(np.float64), b[k][1][:, None]], 1)
                   for k in ("pppp", "ppph")}
    e3 = 0.0
    if w3 != 0.0:
        e3, dfpp, dfhh, nb = _three_body_no2b(three_body_rows(w3, L), is_hole, loc, p, h)
        f_pp = f_pp + dfpp
        f_hh = f_hh + dfhh
        for k in ("phph", "hhhh"):
            np.add.at(dense2[k], tuple(nb[k][0].T), nb[k][1])
        if len(nb["pppp"][1]):
            sparse_rows["pppp"] = np.concatenate(
                [sparse_rows["pppp"], np.concatenate([nb["pppp"][0].astype(np.float64),
                                                      nb["pppp"][1][:, None]], 1)])
    # reference energy (CCM/coupled_cluster.py:288-317)
    e_ref = float(np.trace(f_hh) - 0.5 * np.einsum("ijij->", dense2["hhhh"]) + e3)
    blocks = [dense2[k] for k in ("pphh", "phph", "phhh", "hhhh")]
    return e_ref, [f_pp, f_ph, f_hh], [sparse_rows["pppp"], sparse_rows["ppph"]] + blocks


def _normal_ordered_sparse(L, b, shapes, hole, part, is_hole, loc, p, h, w3, kinetic):
    """``normal_ordered_hamiltonian(..., dense=False)``: the same numbers with
    the four two-body blocks kept as COO :class:`Block` objects from the
    start (entries and their order as the dense path's non-zeros)."""
    n = 4 * L ** 3
    e3, nb = 0.0, {}
    dfpp = dfhh = None
    if w3 != 0.0:
        e3, dfpp, dfhh, nb = _three_body_no2b(three_body_rows(w3, L), is_hole, loc, p, h)
    # the Fock traces see the two-body entries only; the three-body ones are
    # added to the blocks afterwards (as in the dense path)
    two = {k: _canonical_block(shapes[k], *b[k]) for k in shapes}
    coo = {k: (_canonical_block(shapes[k], *b[k], add=nb[k]) if k in nb else two[k]) for k in shapes}
    T = np.zeros((n, n)); has_t = np.zeros((n, n), bool)
    kr = kinetic_rows(L)
    ti, tj = kr[:, 0].astype(np.int64), kr[:, 1].astype(np.int64)
    np.add.at(T, (ti, tj), float(kinetic) * kr[:, 2])
    has_t[ti, tj] = True
    f_pp = T[np.ix_(part, part)] + _trace_13(shapes["phph"], *two["phph"], (p, p))
    f_ph = T[np.ix_(part, hole)] + _trace_13(shapes["phhh"], *two["phhh"], (p, h))
    f_hh = T[np.ix_(hole, hole)] + _trace_13(shapes["hhhh"], *two["hhhh"], (h, h))
    f_pp = np.where(has_t[np.ix_(part, part)], f_pp, 0.0)
    f_ph = np.where(has_t[np.ix_(part, hole)], f_ph, 0.0)
    f_hh = np.where(has_t[np.ix_(hole, hole)], f_hh, 0.0)
    sparse_rows = {k: np.concatenate([b[k][0].astype(np.float64), b[k][1][:, None]], 1)
                   for k in ("pppp", "ppph")}
    if w3 != 0.0:
        f_pp = f_pp + dfpp
        f_hh = f_hh + dfhh
        if len(nb["pppp"][1]):
            sparse_rows["pppp"] = np.concatenate(
                [sparse_rows["pppp"], np.concatenate([nb["pppp"][0].astype(np.float64),
                                                      nb["pppp"][1][:, None]], 1)])
    hi, hv = coo["hhhh"]
    diag = (hi[:, 0] == hi[:, 2]) & (hi[:, 1] == hi[:, 3])
    e_ref = float(np.trace(f_hh) - 0.5 * np.sum(hv[diag]) + e3)
    blocks = [Block(shapes[k], *coo[k]) for k in ("pphh", "phph", "phhh", "hhhh")]
    return e_ref, [f_pp, f_ph, f_hh], [sparse_rows["pppp"], sparse_rows["ppph"]] + blocks


SEVEN_SITES = [(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)]


def closed_shell_holes(L, A):
    """Fully occupied sites: A=4 occupies site (0,0,0); A=28 occupies (0,0,0)
    and its six nearest neighbours (all four spin-isospin states each)."""
    if A == 4:
        sites = SEVEN_SITES[:1]
    elif A == 28:
        sites = SEVEN_SITES
    else:
        raise ValueError("closed_shell_holes: A must be 4 or 28")
    return [[x % L, y % L, z % L, t, s] for (x, y, z) in sites for t in (0, 1) for s in (0, 1)]


def contact_couplings(C2, C3):
    """Couplings given in units of hbar^2/(M a^2) -> reference units hbar^2/(2 M a^2)."""
    return 2.0 * C2, 2.0 * C3
