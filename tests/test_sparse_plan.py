"""The fixed-order gather plans of the general engine's sparse blocks.

``nlb_ppph_intermediates_f64`` and ``nlb_pppp_ladders_f64`` sum every output
entry over its rows of the v_ppph / v_pppp list in an order fixed on the host
(``dense._SparsePlan``).  Here the kernels' gathers are replayed in numpy from
the plan arrays and compared with a plain scatter of the same list (the
reference's v_ppph_dgrams / v_pppp_dgrams, CCM/ccDgrams.py:13-45, 215-237),
repeated keys included.
"""
import numpy as np
import torch

from nulattice_b200 import dense as D


def _plan_arrays(plan):
    # keep[0:2] are idx/val; the rest follow in the order _SparsePlan uploads them
    return [t.cpu().numpy() for t in plan.keep[2:]]


def _rows(rng, p, last, n):
    idx = np.stack([rng.integers(0, p, n), rng.integers(0, p, n), rng.integers(0, p, n),
                    rng.integers(0, last, n)], axis=1).astype(np.int64)
    idx = np.concatenate([idx, idx[:5]])             # repeated keys must add up
    val = rng.standard_normal(len(idx))
    return idx, val


def test_ppph_gathers_match_scatter():
    rng = np.random.default_rng(3)
    p, h = 7, 3
    idx, val = _rows(rng, p, h, 60)
    t1 = rng.standard_normal((p, h))
    t2 = rng.standard_normal((p, p, h, h))
    plan = D._SparsePlan((torch.as_tensor(idx), torch.as_tensor(val), len(val)), "ppph", torch.device("cpu"))
    perm_adk, perm_ak, perm_cdk, seg_a, seg_ad, seg_adk, seg_ak, seg_cdk = _plan_arrays(plan)
    c, d, a, k = idx.T
    # scatter (reference order of operations does not matter for the check)
    r = [np.zeros(s) for s in ((p, h), (p, p), (p, p, h, h), (p, p), (p, p, h, h), (p, h, h, h), (p, h, h, h))]
    for q in range(len(val)):
        v = val[q]
        r[1][a[q], d[q]] -= v * t1[c[q], k[q]]
        r[3][d[q], a[q]] += v * t1[c[q], k[q]]
        r[0][a[q], :] -= 0.5 * v * t2[c[q], d[q], k[q], :]
        r[2][c[q], d[q], :, k[q]] += v * t1[a[q], :]
        r[4][a[q], d[q], :, k[q]] += v * t1[c[q], :]
        r[5][a[q], :, :, k[q]] += v * t2[c[q], d[q]]
        r[6][a[q], :, :, k[q]] += v * np.outer(t1[c[q]], t1[d[q]])
    g = [np.zeros_like(x) for x in r]
    # replay of the gathers: one output owner per segment, rows in plan order
    for s in range(len(seg_ad) - 1):
        rows = perm_adk[seg_ad[s]:seg_ad[s + 1]]
        acc = sum(val[e] * t1[c[e], k[e]] for e in rows)
        e = rows[-1]
        assert np.all(a[rows] == a[e]) and np.all(d[rows] == d[e])
        g[1][a[e], d[e]] -= acc
        g[3][d[e], a[e]] += acc
    for s in range(len(seg_a) - 1):
        rows = perm_adk[seg_a[s]:seg_a[s + 1]]
        assert np.all(a[rows] == a[rows[0]])
        g[0][a[rows[0]]] -= 0.5 * sum(val[e] * t2[c[e], d[e], k[e], :] for e in rows)
    for s in range(len(seg_adk) - 1):
        rows = perm_adk[seg_adk[s]:seg_adk[s + 1]]
        e = rows[0]
        g[4][a[e], d[e], :, k[e]] += sum(val[q] * t1[c[q], :] for q in rows)
    for s in range(len(seg_cdk) - 1):
        rows = perm_cdk[seg_cdk[s]:seg_cdk[s + 1]]
        e = rows[0]
        assert np.all((c[rows] == c[e]) & (d[rows] == d[e]) & (k[rows] == k[e]))
        g[2][c[e], d[e], :, k[e]] += sum(val[q] * t1[a[q], :] for q in rows)
    for s in range(len(seg_ak) - 1):
        rows = perm_ak[seg_ak[s]:seg_ak[s + 1]]
        e = rows[0]
        assert np.all((a[rows] == a[e]) & (k[rows] == k[e]))
        g[5][a[e], :, :, k[e]] += sum(val[q] * t2[c[q], d[q]] for q in rows)
        g[6][a[e], :, :, k[e]] += sum(val[q] * np.outer(t1[c[q]], t1[d[q]]) for q in rows)
    for x, y in zip(r, g):
        np.testing.assert_allclose(y, x, rtol=1e-12, atol=1e-12)
    # every row sits in exactly one segment of each order, segments in key order
    for perm in (perm_adk, perm_ak, perm_cdk):
        assert sorted(perm.tolist()) == list(range(len(val)))


def test_pppp_gathers_match_scatter():
    rng = np.random.default_rng(4)
    p, h = 6, 3
    idx, val = _rows(rng, p, p, 50)
    t1 = rng.standard_normal((p, h))
    t2 = rng.standard_normal((p, p, h, h))
    plan = D._SparsePlan((torch.as_tensor(idx), torch.as_tensor(val), len(val)), "pppp", torch.device("cpu"))
    perm_ab, seg_ab = _plan_arrays(plan)
    a, b, c, d = idx.T
    l1 = np.zeros((p, p, h, h))
    l2 = np.zeros((p, p, h, h))
    np.add.at(l1, (a, b), val[:, None, None] * t2[c, d])
    np.add.at(l2, (a, b), val[:, None, None] * t1[c][:, :, None] * t1[d][:, None, :])
    g1, g2 = np.zeros_like(l1), np.zeros_like(l2)
    for s in range(len(seg_ab) - 1):
        rows = perm_ab[seg_ab[s]:seg_ab[s + 1]]
        assert np.all((a[rows] == a[rows[0]]) & (b[rows] == b[rows[0]]))
        assert np.all(np.diff(rows) > 0)   # equal keys keep their list order
        g1[a[rows[0]], b[rows[0]]] = sum(val[e] * t2[c[e], d[e]] for e in rows)
        g2[a[rows[0]], b[rows[0]]] = sum(val[e] * np.outer(t1[c[e]], t1[d[e]]) for e in rows)
    np.testing.assert_allclose(g1, l1, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(g2, l2, rtol=1e-12, atol=1e-12)
