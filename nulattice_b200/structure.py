"""Structure detection and the compact channel layout of T2 (host side).

The lattice contact Hamiltonian conserves a label on every single-particle
state: the one-body part (hopping) only connects states of the same
spin-isospin, and an SU(4) on-site contact only scatters a pair into the same
pair of labels.  With every hole site fully occupied (the closed-site
references of the lattice examples) the blocks ``v_pphh``, ``v_phph``,
``v_phhh`` and ``v_ppph`` are identically zero, and the CCSD iteration of
``CCM/coupled_cluster.py:342-545`` collapses to

* T1: ``f_ph``, the Fock term ``f_ck t2_acik`` and the dressed Fock products;
* T2: the particle-particle and hole-hole ladders acting on
  ``tau = t2 + t1 t1`` and the dressed Fock products ``P(ab) X_pp t2`` and
  ``P(ij) X_hh t2`` (``X_pp = f_pp - f_ph t1^T``, ``X_hh = -f_hh - f_ph^T t1``).

Labels are detected from the inputs (connected components of the non-zero
pattern of ``f_pp``, ``f_ph`` and ``f_hh``), then checked against the
two-body blocks.  T2 is stored once per unique amplitude: for each channel
``(g1 < g2)`` a dense block ``B[a', b', i', j']`` with ``a'`` running over the
particles of label g1, ``b'`` over the particles of g2, ``i'`` over the holes
of g1 and ``j'`` over the holes of g2, so that
``t2[a,b,i,j] = B``, ``t2[b,a,i,j] = t2[a,b,j,i] = -B``, ``t2[b,a,j,i] = B``.
Every other entry of the dense T2 is zero for these inputs.  At L=6, A=28
this is 1.28e7 numbers instead of 5.48e8.

If any check fails, :func:`detect` returns ``None`` with the reason and the
solver uses its general dense path instead.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

MAX_LABELS = 64


def _coo(block):
    """(indices (N,k) int64, values (N,)) of a dense array, a :class:`Block`,
    an object with ``.indices``/``.values``, a ``(indices, values)`` pair or an
    (N,5) row list; repeated keys are summed and zeros dropped."""
    if block is None:
        return np.zeros((0, 4), np.int64), np.zeros(0)
    if hasattr(block, "indices") and hasattr(block, "values"):
        idx = np.asarray(_to_np(block.indices), dtype=np.int64)
        val = np.asarray(_to_np(block.values), dtype=np.float64)
    elif isinstance(block, tuple) and len(block) == 2:
        idx = np.asarray(_to_np(block[0]), dtype=np.int64)
        val = np.asarray(_to_np(block[1]), dtype=np.float64)
        if idx.ndim == 2 and idx.shape[0] == 4 and idx.shape[1] != 4:
            idx = idx.T
    else:
        arr = np.asarray(_to_np(block), dtype=np.float64)
        if arr.ndim == 4:
            idx = np.argwhere(arr != 0)
            return idx.astype(np.int64), arr[tuple(idx.T)]
        arr = arr.reshape(-1, 5)
        idx, val = arr[:, :4].astype(np.int64), arr[:, 4]
    idx = idx.reshape(-1, 4)
    if len(val) == 0:
        return idx, val
    dims = idx.max(axis=0) + 1
    if idx.min() < 0 or float(np.prod(dims.astype(np.float64))) >= 2.0 ** 62:
        uniq, inv = np.unique(idx, axis=0, return_inverse=True)
        acc = np.zeros(len(uniq))
        np.add.at(acc, inv.reshape(-1), val)
        keep = acc != 0
        return uniq[keep], acc[keep]
    # rows sorted lexicographically = sorted by the mixed-radix key
    key = ((idx[:, 0] * dims[1] + idx[:, 1]) * dims[2] + idx[:, 2]) * dims[3] + idx[:, 3]
    order = np.argsort(key, kind="stable")
    ks = key[order]
    start = np.flatnonzero(np.concatenate(([True], ks[1:] != ks[:-1])))
    acc = np.add.reduceat(val[order], start)
    uniq = idx[order[start]]
    keep = acc != 0
    return uniq[keep], acc[keep]


def _csr_ptr(rows, n):
    """CSR row pointer (length n + 1, int64) of the sorted or unsorted row
    indices ``rows`` in [0, n): one count and one running sum, written in
    place."""
    ptr = np.empty(n + 1, np.int64)
    ptr[0] = 0
    np.cumsum(np.bincount(rows, minlength=n), out=ptr[1:])
    return ptr


def _nonzero2(a):
    """``np.nonzero`` of a 2-D float array (same indices, same row-major
    order, -0.0 counted as zero and NaN as non-zero), through a flat scan
    of ``a != 0``: a quarter of the time on the dense Fock blocks."""
    k = np.flatnonzero(a != 0)
    n = a.shape[1] if a.ndim == 2 and a.shape[1] else 1
    return k // n, k % n


def _to_np(x):
    if hasattr(x, "detach"):
        return x.detach().cpu().numpy()
    return x


def _components(n, src, dst):
    """Connected-component label (0..k-1, ordered by smallest member) of each
    of n vertices joined by the edges (src[k], dst[k])."""
    from scipy.sparse import coo_matrix
    from scipy.sparse.csgraph import connected_components
    src = np.asarray(src, dtype=np.int64)
    g = coo_matrix((np.ones(len(src)), (src, np.asarray(dst, dtype=np.int64))), shape=(n, n))
    _, lab = connected_components(g, directed=False)
    # relabel by the smallest member, as a union-find with min roots would
    first = np.full(lab.max() + 1 if n else 0, n, dtype=np.int64)
    np.minimum.at(first, lab, np.arange(n))
    _, out = np.unique(first[lab], return_inverse=True)
    return out.astype(np.int64)


def _antisym_ok(idx, val, n0, n1, tol=0.0):
    """True when v[a,b,c,d] = -v[b,a,c,d] = -v[a,b,d,c] entry by entry
    (idx unique; entries absent from the list are zero)."""
    if len(val) == 0:
        return True
    idx = np.asarray(idx, dtype=np.int64)
    val = np.asarray(val, dtype=np.float64)
    dims = idx.max(axis=0) + 1
    size = int(max(dims[0], dims[1])) , int(max(dims[2], dims[3]))
    key = lambda a, b, c, d: ((a * size[0] + b) * size[1] + c) * size[1] + d  # noqa: E731
    k0 = key(idx[:, 0], idx[:, 1], idx[:, 2], idx[:, 3])
    order = np.argsort(k0)
    ks, vs = k0[order], val[order]
    for k in (key(idx[:, 1], idx[:, 0], idx[:, 2], idx[:, 3]), key(idx[:, 0], idx[:, 1], idx[:, 3], idx[:, 2])):
        pos = np.searchsorted(ks, k)
        pos = np.minimum(pos, len(ks) - 1)
        partner = np.where(ks[pos] == k, vs[pos], 0.0)
        if np.any(np.abs(partner + val) > tol * np.abs(val)):
            return False
    return True


@dataclass
class Channel:
    g1: int
    g2: int
    np1: int
    np2: int
    nh1: int
    nh2: int
    offset: int  # element offset of this channel's block in the compact T2

    @property
    def size(self):
        return self.np1 * self.np2 * self.nh1 * self.nh2


@dataclass
class ChannelPlan:
    """Everything the structured kernels need, as host numpy arrays."""
    p: int
    h: int
    n_labels: int
    p_label: np.ndarray   # (p,) label of each particle
    h_label: np.ndarray   # (h,)
    p_loc: np.ndarray     # (p,) index of the particle within its label
    h_loc: np.ndarray     # (h,)
    p_of: list            # per label: particle indices (ascending)
    h_of: list            # per label: hole indices (ascending)
    channels: list
    n_t2: int
    # f_pp restricted to each label, CSR over label-local rows (concatenated
    # over labels; rows of label g start at p_base[g])
    p_base: np.ndarray
    h_base: np.ndarray
    fpp_ptr: np.ndarray
    fpp_col: np.ndarray   # label-local column
    fpp_val: np.ndarray
    # f_ph restricted to each label: per hole (label-ordered) a list of
    # (label-local particle, value)
    fph_ptr: np.ndarray
    fph_col: np.ndarray
    fph_val: np.ndarray
    # per channel: hole-hole ladder as CSR over the output hole pair
    # hp = i'*nh2 + j' (input pair, value), and particle-particle ladder as CSR
    # over the output particle pair ab = a'*np2 + b'
    hh_ptr: list
    hh_col: list
    hh_val: list
    pp_ptr: list
    pp_col: list
    pp_val: list
    info: dict = field(default_factory=dict)

    # -- dense <-> compact ------------------------------------------------
    def pack_t2(self, t2):
        out = np.zeros(self.n_t2)
        for ch in self.channels:
            P1, P2, H1, H2 = self.p_of[ch.g1], self.p_of[ch.g2], self.h_of[ch.g1], self.h_of[ch.g2]
            out[ch.offset:ch.offset + ch.size] = t2[np.ix_(P1, P2, H1, H2)].ravel()
        return out

    def unpack_t2(self, comp, out=None):
        t2 = np.zeros((self.p, self.p, self.h, self.h)) if out is None else out
        for ch in self.channels:
            P1, P2, H1, H2 = self.p_of[ch.g1], self.p_of[ch.g2], self.h_of[ch.g1], self.h_of[ch.g2]
            B = comp[ch.offset:ch.offset + ch.size].reshape(ch.np1, ch.np2, ch.nh1, ch.nh2)
            t2[np.ix_(P1, P2, H1, H2)] = B
            t2[np.ix_(P2, P1, H1, H2)] = -B.transpose(1, 0, 2, 3)
            t2[np.ix_(P1, P2, H2, H1)] = -B.transpose(0, 1, 3, 2)
            t2[np.ix_(P2, P1, H2, H1)] = B.transpose(1, 0, 3, 2)
        return t2

    def t1_mask(self):
        return self.p_label[:, None] == self.h_label[None, :]

    def dense_weight(self):
        """Each stored T2 number appears four times in the dense tensor."""
        return 4.0


def detect(fock_mats, two_body_int, t1initial=None):
    """Return ``(plan, None)`` when the structured path applies, else
    ``(None, reason)``."""
    f_pp, f_ph, f_hh = [np.asarray(_to_np(f), dtype=np.float64) for f in fock_mats]
    p, h = f_ph.shape
    v_pppp, v_ppph, v_pphh, v_phph, v_phhh, v_hhhh = two_body_int
    for name, blk in (("v_pphh", v_pphh), ("v_phph", v_phph), ("v_phhh", v_phhh), ("v_ppph", v_ppph)):
        if len(_coo(blk)[1]):
            return None, f"{name} is non-zero (open-shell site or non-conserving contact)"
    n = p + h
    fpp_r, fpp_c = _nonzero2(f_pp)
    fph_r, fph_c = _nonzero2(f_ph)
    fhh_r, fhh_c = _nonzero2(f_hh)
    lab = _components(n, np.concatenate([fpp_r, fph_r, p + fhh_r]),
                      np.concatenate([fpp_c, p + fph_c, p + fhh_c]))
    G = int(lab.max()) + 1 if n else 0
    if G < 2:
        return None, "one-body part connects every state (no conserved label)"
    if G > MAX_LABELS:
        return None, f"{G} one-body components (more than {MAX_LABELS})"
    p_label, h_label = lab[:p], lab[p:]
    pp_idx, pp_v = _coo(v_pppp)
    hh_idx, hh_v = _coo(v_hhhh)
    for name, idx, lp in (("v_pppp", pp_idx, p_label), ("v_hhhh", hh_idx, h_label)):
        if len(idx):
            la, lb, lc, ld = (lp[idx[:, k]] for k in range(4))
            same = ((la == lc) & (lb == ld)) | ((la == ld) & (lb == lc))
            if not np.all(same):
                return None, f"{name} changes the labels of a pair"
            if np.any(la == lb):
                return None, f"{name} couples a same-label pair"
    if not _antisym_ok(pp_idx, pp_v, p, p) or not _antisym_ok(hh_idx, hh_v, h, h):
        return None, "v_pppp or v_hhhh is not antisymmetric"
    if t1initial is not None:
        t1i = np.asarray(_to_np(t1initial))
        if np.any(t1i[p_label[:, None] != h_label[None, :]] != 0):
            return None, "t1initial couples different labels"
    p_of = [np.flatnonzero(p_label == g) for g in range(G)]
    h_of = [np.flatnonzero(h_label == g) for g in range(G)]
    p_loc = np.zeros(p, np.int64); h_loc = np.zeros(h, np.int64)
    for g in range(G):
        p_loc[p_of[g]] = np.arange(len(p_of[g]))
        h_loc[h_of[g]] = np.arange(len(h_of[g]))
    p_base = np.concatenate([[0], np.cumsum([len(x) for x in p_of])]).astype(np.int64)
    h_base = np.concatenate([[0], np.cumsum([len(x) for x in h_of])]).astype(np.int64)

    channels, off = [], 0
    for g1 in range(G):
        for g2 in range(g1 + 1, G):
            np1, np2, nh1, nh2 = len(p_of[g1]), len(p_of[g2]), len(h_of[g1]), len(h_of[g2])
            if np1 * np2 * nh1 * nh2 == 0:
                continue
            ch = Channel(g1, g2, np1, np2, nh1, nh2, off)
            channels.append(ch)
            off += ch.size

    # f_pp CSR (label-ordered rows, label-local columns).  Every non-zero of
    # f_pp joins two states of one label, so in label order the matrix is
    # block diagonal and a column's local index is its position minus the
    # label's base.
    p_ord = np.concatenate(p_of) if G else np.zeros(0, np.int64)
    h_ord = np.concatenate(h_of) if G else np.zeros(0, np.int64)
    p_pos = np.empty(p, np.int64); p_pos[p_ord] = np.arange(p)
    h_pos = np.empty(h, np.int64); h_pos[h_ord] = np.arange(h)
    r, c = p_pos[fpp_r], p_pos[fpp_c]
    order = np.argsort(r * max(p, 1) + c, kind="stable")
    r, c = r[order], c[order]
    fpp_ptr = _csr_ptr(r, p)
    fpp_col = (c - p_base[p_label[p_ord[c]]]).astype(np.int64)
    fpp_val = np.ascontiguousarray(f_pp[fpp_r[order], fpp_c[order]], dtype=np.float64)
    # f_ph per hole (label-ordered holes, label-local particle rows)
    r, c = h_pos[fph_c], p_pos[fph_r]
    order = np.argsort(r * max(p, 1) + c, kind="stable")
    r, c = r[order], c[order]
    fph_ptr = _csr_ptr(r, h)
    fph_col = (c - p_base[p_label[p_ord[c]]]).astype(np.int64)
    fph_val = np.ascontiguousarray(f_ph[fph_r[order], fph_c[order]], dtype=np.float64)

    # ladders per channel
    hh_ptr, hh_col, hh_val, pp_ptr, pp_col, pp_val = [], [], [], [], [], []
    for ch in channels:
        # hole-hole: output (i,j) in (g1,g2), input (k,l) in (g1,g2), value v[k,l,i,j]
        if len(hh_idx):
            k, l, i, j = hh_idx.T
            m = (h_label[k] == ch.g1) & (h_label[l] == ch.g2) & (h_label[i] == ch.g1) & (h_label[j] == ch.g2)
            out = h_loc[i[m]] * ch.nh2 + h_loc[j[m]]
            inp = h_loc[k[m]] * ch.nh2 + h_loc[l[m]]
            vv = hh_v[m]
        else:
            out = inp = np.zeros(0, np.int64); vv = np.zeros(0)
        order = np.argsort(out, kind="stable")
        hh_ptr.append(_csr_ptr(out, ch.nh1 * ch.nh2))
        hh_col.append(inp[order].astype(np.int64)); hh_val.append(vv[order])
        # particle-particle: output (a,b) in (g1,g2), input (c,d) in (g1,g2)
        if len(pp_idx):
            a, b, c, d = pp_idx.T
            m = (p_label[a] == ch.g1) & (p_label[b] == ch.g2) & (p_label[c] == ch.g1) & (p_label[d] == ch.g2)
            out = p_loc[a[m]] * ch.np2 + p_loc[b[m]]
            inp = p_loc[c[m]] * ch.np2 + p_loc[d[m]]
            vv = pp_v[m]
        else:
            out = inp = np.zeros(0, np.int64); vv = np.zeros(0)
        order = np.argsort(out, kind="stable")
        pp_ptr.append(_csr_ptr(out, ch.np1 * ch.np2))
        pp_col.append(inp[order].astype(np.int64)); pp_val.append(vv[order])

    plan = ChannelPlan(p=p, h=h, n_labels=G, p_label=p_label, h_label=h_label, p_loc=p_loc,
                       h_loc=h_loc, p_of=p_of, h_of=h_of, channels=channels, n_t2=off,
                       p_base=p_base, h_base=h_base, fpp_ptr=fpp_ptr, fpp_col=fpp_col,
                       fpp_val=fpp_val, fph_ptr=fph_ptr, fph_col=fph_col, fph_val=fph_val,
                       hh_ptr=hh_ptr, hh_col=hh_col, hh_val=hh_val, pp_ptr=pp_ptr,
                       pp_col=pp_col, pp_val=pp_val)
    plan.info = dict(labels=G, channels=len(channels), n_t2=off,
                     dense_t2=p * p * h * h, fpp_nnz=len(fpp_val), fph_nnz=len(fph_val),
                     pp_nnz=int(sum(len(x) for x in pp_val)), hh_nnz=int(sum(len(x) for x in hh_val)))
    return plan, None
