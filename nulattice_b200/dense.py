"""General (dense) CCSD engine on the GPU.

Used by :func:`nulattice_b200.ccsd.ccsd_solver` for inputs that the
structured engine does not cover (open-shell sites, non-SU(4) contacts,
Hamiltonians read from files or random test tensors).  It evaluates the
reference's factorised equation set -- ``t1Iter`` / ``t2Iter``
(``CCM/coupled_cluster.py:342-545``) with the diagrams of
``CCM/ccDgrams.py:13-578`` -- on dense FP64 tensors in the reference's
layouts:

* every diagram is an einsum run as a chain of pairwise contractions by the
  strided kernel ``nlb_contract_f64`` (order from ``numpy.einsum_path``);
* ``pAB`` / ``pIJ`` are applied by ``nlb_antisym_acc_f64`` while
  accumulating;
* the sparse ``v_ppph`` / ``v_pppp`` lists go through their scatter kernels;
* Jacobi update with mixing, energy and the torch solver's pulsed DIIS are
  their own kernels.

Diagrams whose two-body block is identically zero are skipped (they add
exact zeros).  The amplitudes live in one vector ``[t1 | t2]`` so that the
DIIS error vectors are the reference's ``torch.cat`` of both.
"""
from __future__ import annotations

import ctypes
import string
import time

import numpy as np
import torch

from . import _lib

_c64 = ctypes.c_int64

# name -> (coefficient, einsum, operands, antisymmetriser); the names are the
# reference's functions in CCM/ccDgrams.py (line of the definition beside it).
TERMS = {
    "dgram_akci_ck": (-1.0, "akci,ck->ai", ("v_phph", "t1"), 0),            # :48
    "dgram_ck_acik": (1.0, "ck,acik->ai", ("f_ph", "t2"), 0),               # :61
    "dgram_cikl_cakl": (-0.5, "cikl,cakl->ai", ("v_phhh", "t2"), 0),        # :74
    "dgram_cdkl_ck_dali": (1.0, "cdkl,ck,dali->ai", ("v_pphh", "t1", "t2"), 0),  # :87
    "dgram_ck_ci": (-0.5, "ck,ci->ki", ("f_ph", "t1"), 0),                  # :102
    "dgram_ck_ak": (-0.5, "ck,ak->ac", ("f_ph", "t1"), 0),                  # :115
    "dgram_bijk_bj": (-1.0, "bijk,bj->ki", ("v_phhh", "t1"), 0),            # :128
    "dgram_cdlk_cdli": (-0.5, "cdlk,cdli->ki", ("v_pphh", "t2"), 0),        # :141
    "dgram_dckl_dakl": (-0.5, "dckl,dakl->ac", ("v_pphh", "t2"), 0),        # :154
    "dgram_cdlk_cl_di": (-0.5, "cdlk,cl,di->ki", ("v_pphh", "t1", "t1"), 0),  # :167
    "dgram_cdkl_dk_al": (0.5, "cdkl,dk,al->ac", ("v_pphh", "t1", "t1"), 0),   # :180
    "dgram_klij_abkl": (0.5, "klij,abkl->abij", ("v_hhhh", "t2"), 0),       # :240
    "dgram_bkcj_acik": (-1.0, "bkcj,acik->abij", ("v_phph", "t2"), 3),      # :253
    "dgram_bkij_ak": (1.0, "bkij,ak->abij", ("v_phhh", "t1"), 1),           # :266
    "dgram_cdkl_acik_dblj": (0.5, "cdkl,acik,dblj->abij", ("v_pphh", "t2", "t2"), 3),  # :279
    "dgram_cdkl_cdij_abkl": (0.25, "cdkl,cdij,abkl->abij", ("v_pphh", "t2", "t2"), 0),  # :292
    "dgram_klij_ak_bl": (0.5, "klij,ak,bl->abij", ("v_hhhh", "t1", "t1"), 1),        # :305
    "dgram_bkci_ak_cj": (-1.0, "bkci,ak,cj->abij", ("v_phph", "t1", "t1"), 3),       # :318
    "dgram_cikl_ck_ablj": (-1.0, "cikl,ck,ablj->abij", ("v_phhh", "t1", "t2"), 2),   # :331
    "dgram_da_dbij": (-1.0, "da,dbij->abij", ("r3", "t2"), 1),                       # :346
    "dgram_acik_bcjk": (1.0, "acik,bcjk->abij", ("r4", "t2"), 3),                    # :359
    "dgram_cikl_al_bcjk": (-1.0, "cikl,al,bcjk->abij", ("v_phhh", "t1", "t2"), 3),   # :372
    "dgram_cjkl_ci_abkl": (0.5, "cjkl,ci,abkl->abij", ("v_phhh", "t1", "t2"), 2),    # :387
    "dgram_bijk_ak1": (0.5, "bijk,ak->abij", ("r5", "t1"), 1),                       # :405
    "dgram_bijk_ak2": (0.5, "bijk,ak->abij", ("r6", "t1"), 3),                       # :418
    "dgram_cjkl_ci_ak_bl": (0.5, "cjkl,ci,ak,bl->abij", ("v_phhh", "t1", "t1", "t1"), 3),  # :431
    "dgram_cdkl_ci_dj_abkl": (0.25, "cdkl,ci,dj,abkl->abij", ("v_pphh", "t1", "t1", "t2"), 2),  # :444
    "dgram_cdkl_ak_bl_cdij": (0.25, "cdkl,ak,bl,cdij->abij", ("v_pphh", "t1", "t1", "t2"), 1),  # :459
    "dgram_cdkl_ci_bl_adkj": (1.0, "cdkl,ci,bl,adkj->abij", ("v_pphh", "t1", "t1", "t2"), 3),   # :474
    "dgram_cdkl_ci_ak_dj_bl": (0.25, "cdkl,ci,ak,dj,bl->abij", ("v_pphh", "t1", "t1", "t1", "t1"), 3),  # :489
    "dgram_cdkl_bdkl": (-0.5, "cdkl,bdkl->bc", ("v_pphh", "t2"), 0),        # :502
    "dgram_cdkl_cdjl": (-0.5, "cdkl,cdjl->kj", ("v_pphh", "t2"), 0),        # :515
    "dgram_ck_bk": (-1.0, "ck,bk->bc", ("f_ph", "t1"), 0),                  # :528
    "dgram_ck_cj": (-1.0, "ck,cj->kj", ("f_ph", "t1"), 0),                  # :541
    "dgram_cdlk_cl_dj": (-1.0, "cdlk,cl,dj->kj", ("v_pphh", "t1", "t1"), 0),  # :554
    "dgram_cdlk_dk_bl": (-1.0, "cdlk,dk,bl->bc", ("v_pphh", "t1", "t1"), 0),  # :567
}


# a 4-D v_pppp with at least this fraction non-zero stays dense (ladders as GEMMs)
DENSE_PPPP_FRACTION = 8

# contractions with at least this many multiply-adds (and no batch index)
# go through gathered panels and one GEMM: the FP64 library GEMM, or in the
# mixed phase the 3xTF32 tcgen05 kernel when both GEMM sides have at least
# TC_MIN_MN rows (its tiles are 128 x 128)
GEMM_MIN_MACS = 1 << 18
TC_MIN_MN = 32


class GpuEinsum:
    """Einsum over CUDA FP64 tensors through ``nlb_contract_f64`` (strided
    tiles) or, for large contractions, ``nlb_contract_gemm_f64``."""

    def __init__(self, stream_ptr):
        self.L = _lib.lib()
        self.sp = ctypes.c_void_p(stream_ptr)
        self._plans = {}
        self._descs = {}
        self._ws = None
        self.launches = 0
        self.gemms = 0
        self.tc_gemms = 0
        self.tensor_cores = False    # mixed phase: GEMM-shaped contractions on the tcgen05 kernel

    def _workspace(self, nbytes, device):
        if self._ws is None or self._ws.numel() * 8 < nbytes:
            self._ws = torch.empty((nbytes + 7) // 8, dtype=torch.float64, device=device)
        return self._ws

    # -- one pairwise contraction ------------------------------------------
    def pair(self, spec, A, B, out, alpha=1.0, beta=0.0):
        # the descriptor and route depend only on the spec, shapes and strides
        key = (spec, tuple(A.shape), A.stride(), tuple(B.shape), B.stride(), tuple(out.shape), out.stride(),
               self.tensor_cores)
        hit = self._descs.get(key)
        if hit is None:
            hit = self._describe(spec, A, B, out)
            self._descs[key] = hit
        d, route, need = hit
        if route == "tc":
            ws = self._workspace(need, out.device)
            _lib.check(self.L.nlb_contract_gemm_tf32x3(ctypes.byref(d), A.data_ptr(), B.data_ptr(), out.data_ptr(),
                                                       alpha, beta, ws.data_ptr(), ws.numel() * 8, self.sp),
                       "contract (tensor cores)")
            self.launches += 4
            self.tc_gemms += 1
        elif route == "gemm":
            ws = self._workspace(need, out.device)
            _lib.check(self.L.nlb_contract_gemm_f64(ctypes.byref(d), A.data_ptr(), B.data_ptr(), out.data_ptr(),
                                                    alpha, beta, ws.data_ptr(), ws.numel() * 8, self.sp),
                       "contract (gemm)")
            self.launches += 4
            self.gemms += 1
        else:
            _lib.check(self.L.nlb_contract_f64(ctypes.byref(d), A.data_ptr(), B.data_ptr(), out.data_ptr(),
                                               alpha, beta, self.sp), "contract")
            self.launches += 1

    def _describe(self, spec, A, B, out):
        """(descriptor, route, workspace bytes) of one pairwise contraction."""
        ins, oz = spec.split("->")
        ia, ib = ins.split(",")
        d = _lib.ContractDesc()
        groups = {"m": [], "n": [], "k": [], "b": []}
        sa = dict(zip(ia, A.stride())); sb = dict(zip(ib, B.stride())); sc = dict(zip(oz, out.stride()))
        ext = {}
        for x, s in zip(ia, A.shape):
            ext[x] = s
        for x, s in zip(ib, B.shape):
            ext[x] = s
        for x in oz:
            if x in ia and x in ib:
                groups["b"].append(x)
            elif x in ia:
                groups["m"].append(x)
            elif x in ib:
                groups["n"].append(x)
            else:
                raise ValueError(f"output index {x} not in inputs of {spec}")
        for x in dict.fromkeys(ia + ib):
            if x not in oz:
                groups["k"].append(x)
        for g in groups.values():
            if len(g) > 4:
                raise ValueError(f"more than four indices in one group of {spec}")
        d.nm, d.nn, d.nk, d.nb = (len(groups[g]) for g in "mnkb")
        for g, (fe, f1, f2, f3) in {"m": ("ext_m", "sa_m", "sc_m", None), "n": ("ext_n", "sb_n", "sc_n", None),
                                    "k": ("ext_k", "sa_k", "sb_k", None),
                                    "b": ("ext_b", "sa_b", "sb_b", "sc_b")}.items():
            for q, x in enumerate(groups[g]):
                getattr(d, fe)[q] = ext[x]
                if g == "m":
                    d.sa_m[q] = sa[x]; d.sc_m[q] = sc[x]
                elif g == "n":
                    d.sb_n[q] = sb[x]; d.sc_n[q] = sc[x]
                elif g == "k":
                    d.sa_k[q] = sa.get(x, 0); d.sb_k[q] = sb.get(x, 0)
                else:
                    d.sa_b[q] = sa[x]; d.sb_b[q] = sb[x]; d.sc_b[q] = sc[x]
        prod = lambda g: int(np.prod([ext[x] for x in groups[g]])) if groups[g] else 1  # noqa: E731
        d.M, d.N, d.K, d.B = prod("m"), prod("n"), prod("k"), prod("b")
        if d.B == 1 and d.K > 0 and d.M * d.N * d.K >= GEMM_MIN_MACS:
            if self.tensor_cores and min(d.M, d.N) >= TC_MIN_MN:
                return d, "tc", int(self.L.nlb_contract_gemm_tc_work(ctypes.byref(d)))
            # large contractions: gathered panels and one library GEMM
            return d, "gemm", int(self.L.nlb_contract_gemm_work(ctypes.byref(d)))
        return d, "tiles", 0

    # -- a chain of pairwise contractions ------------------------------------
    def __call__(self, spec, *ops, out, alpha=1.0, beta=0.0):
        ins, oz = spec.split("->")
        terms = ins.split(",")
        if len(terms) == 1:
            raise ValueError("single-operand einsum is not used here")
        key = (spec, tuple(tuple(o.shape) for o in ops))
        plan = self._plans.get(key)
        if plan is None:
            plan = self._plan(terms, oz, ops)
            self._plans[key] = plan
        cur = list(ops)
        cur_terms = list(terms)
        for n, (i, j, res) in enumerate(plan):
            A, B = cur[i], cur[j]
            last = n == len(plan) - 1
            if last:
                self.pair(f"{cur_terms[i]},{cur_terms[j]}->{res}", A, B, out, alpha, beta)
                return out
            ext = {}
            for t, o in ((cur_terms[i], A), (cur_terms[j], B)):
                for x, s in zip(t, o.shape):
                    ext[x] = s
            tmp = torch.empty([ext[x] for x in res], dtype=torch.float64, device=out.device)
            self.pair(f"{cur_terms[i]},{cur_terms[j]}->{res}", A, B, tmp)
            for q in sorted((i, j), reverse=True):
                del cur[q]; del cur_terms[q]
            cur.append(tmp); cur_terms.append(res)
        return out

    @staticmethod
    def _plan(terms, oz, ops):
        dummies = [np.empty(tuple(o.shape)) for o in ops]
        path = np.einsum_path(",".join(terms) + "->" + oz, *dummies, optimize="greedy")[0][1:]
        cur = list(terms)
        plan = []
        for k, pos in enumerate(path):
            i, j = sorted(pos)
            if k == len(path) - 1:
                res = oz
            else:
                rest = [t for q, t in enumerate(cur) if q not in (i, j)]
                keep = set(oz) | set("".join(rest))
                res = "".join(x for x in dict.fromkeys(cur[i] + cur[j]) if x in keep)
            plan.append((i, j, res))
            cur = [t for q, t in enumerate(cur) if q not in (i, j)] + [res]
        return plan


def _dense_block(x, shape, dev):
    """A C-contiguous FP64 copy on ``dev``: the element-wise kernels (Jacobi,
    antisymmetrisers, energy) index the blocks and every tensor cloned from
    them in row-major order, whatever the strides of the caller's array
    (``np.einsum`` and transposes return permuted strides)."""
    if x is None:
        return torch.zeros(shape, dtype=torch.float64, device=dev)
    if isinstance(x, torch.Tensor):
        return x.to(device=dev, dtype=torch.float64).contiguous()
    if hasattr(x, "to_dense"):
        x = x.to_dense()
    return torch.as_tensor(np.ascontiguousarray(x, dtype=np.float64), device=dev)


def _rows_dev(x, dev):
    from .structure import _coo
    idx, val = _coo(x)
    return (torch.as_tensor(np.ascontiguousarray(idx, dtype=np.int64), device=dev),
            torch.as_tensor(np.ascontiguousarray(val, dtype=np.float64), device=dev), len(val))


def _key_order(*cols):
    """Stable order of the rows by the key columns (first column primary) and
    the starts of the runs of equal keys (with the end appended)."""
    n = len(cols[0])
    order = np.lexsort((np.arange(n),) + tuple(reversed(cols)))
    if n == 0:
        return order.astype(np.int32), np.zeros(1, np.int64)
    srt = np.stack([c[order] for c in cols], axis=1)
    change = np.concatenate([[True], np.any(srt[1:] != srt[:-1], axis=1)])
    starts = np.flatnonzero(change)
    return order.astype(np.int32), np.concatenate([starts, [n]]).astype(np.int64)


def _runs(order, cols):
    """Starts (with the end) of the runs of equal keys of `cols` in `order`."""
    n = len(order)
    if n == 0:
        return np.zeros(1, np.int64)
    srt = np.stack([c[order] for c in cols], axis=1)
    change = np.concatenate([[True], np.any(srt[1:] != srt[:-1], axis=1)])
    return np.concatenate([np.flatnonzero(change), [n]]).astype(np.int64)


class _SparsePlan:
    """A v_ppph / v_pppp row list on the device with the orders its
    contractions gather in (``nlb_ppph_plan`` / ``nlb_pppp_plan``): every
    output entry sums its rows in one fixed order, so results repeat bit for
    bit."""

    def __init__(self, rows, kind, dev):
        idx_d, val_d, nnz = rows
        self.nnz = nnz
        self.keep = [idx_d, val_d]
        idx = idx_d.cpu().numpy().reshape(-1, 4) if nnz else np.zeros((0, 4), np.int64)
        dv = lambda a: self._dev(a, dev)  # noqa: E731
        if kind == "ppph":
            c, d, a, k = idx.T
            perm_adk, seg_adk = _key_order(a, d, k)
            seg_a, seg_ad = _runs(perm_adk, (a,)), _runs(perm_adk, (a, d))
            perm_ak, seg_ak = _key_order(a, k)
            perm_cdk, seg_cdk = _key_order(c, d, k)
            self.c = _lib.PpphPlan(nnz=nnz, idx=idx_d.data_ptr() if nnz else None,
                                   val=val_d.data_ptr() if nnz else None,
                                   perm_adk=dv(perm_adk), perm_ak=dv(perm_ak), perm_cdk=dv(perm_cdk),
                                   n_a=len(seg_a) - 1, n_ad=len(seg_ad) - 1, n_adk=len(seg_adk) - 1,
                                   n_ak=len(seg_ak) - 1, n_cdk=len(seg_cdk) - 1,
                                   seg_a=dv(seg_a), seg_ad=dv(seg_ad), seg_adk=dv(seg_adk), seg_ak=dv(seg_ak),
                                   seg_cdk=dv(seg_cdk))
        else:
            a, b = idx[:, 0], idx[:, 1]
            perm_ab, seg_ab = _key_order(a, b)
            self.c = _lib.PpppPlan(nnz=nnz, idx=idx_d.data_ptr() if nnz else None,
                                   val=val_d.data_ptr() if nnz else None, perm_ab=dv(perm_ab),
                                   n_ab=len(seg_ab) - 1, seg_ab=dv(seg_ab))

    def _dev(self, a, dev):
        t = torch.as_tensor(np.ascontiguousarray(a if len(a) else np.zeros(1, a.dtype)), device=dev)
        self.keep.append(t)
        return t.data_ptr()


class DenseEngine:
    def __init__(self, fock_mats, two_body_int, dev):
        self.dev = dev
        f_pp, f_ph, f_hh = [_dense_block(f, None, dev) for f in fock_mats]
        p, h = f_ph.shape
        self.p, self.h = p, h
        self.T = dict(f_pp=f_pp, f_ph=f_ph, f_hh=f_hh)
        v_pppp, v_ppph, v_pphh, v_phph, v_phhh, v_hhhh = two_body_int
        shapes = {"v_pphh": (p, p, h, h), "v_phph": (p, h, p, h), "v_phhh": (p, h, h, h), "v_hhhh": (h, h, h, h)}
        for name, blk in zip(("v_pphh", "v_phph", "v_phhh", "v_hhhh"), (v_pphh, v_phph, v_phhh, v_hhhh)):
            if blk is not None and not isinstance(blk, torch.Tensor) and hasattr(blk, "indices") \
                    and not hasattr(blk, "to_dense"):
                from .structure import _coo
                idx, val = _coo(blk)
                t = torch.zeros(shapes[name], dtype=torch.float64, device=dev)
                if len(val):
                    t[tuple(torch.as_tensor(idx.T, device=dev))] = torch.as_tensor(val, device=dev)
                self.T[name] = t
            else:
                self.T[name] = _dense_block(blk, shapes[name], dev)
        self.nonzero = {k: bool(torch.count_nonzero(v).item()) for k, v in self.T.items() if k.startswith("v_")}
        # Physical inputs are antisymmetric; there the residual is projected
        # onto antisymmetric tensors (see nlb_antisym_project_f64).
        v = self.T["v_pphh"]
        self.antisym = bool(torch.equal(v, -v.permute(1, 0, 2, 3)) and torch.equal(v, -v.permute(0, 1, 3, 2)))
        # a dense v_pppp (a rotated, e.g. Hartree-Fock, basis) keeps its dense
        # form: both ladders are then GEMM-shaped contractions
        self.pppp_dense = None
        if isinstance(v_pppp, (np.ndarray, torch.Tensor)) and v_pppp.ndim == 4:
            vd = _dense_block(v_pppp, (p, p, p, p), dev)
            if int(torch.count_nonzero(vd).item()) * DENSE_PPPP_FRACTION >= vd.numel():
                self.pppp_dense = vd
        self.pppp = _SparsePlan(self._sparse(v_pppp, (p, p, p, p)) if self.pppp_dense is None else (None, None, 0),
                                "pppp", dev)
        self.ppph = _SparsePlan(self._sparse(v_ppph, (p, p, p, h)), "ppph", dev)
        self.work = torch.zeros(_lib.NLB_DENSE_WORK_DOUBLES, dtype=torch.float64, device=dev)
        self.stream = torch.cuda.current_stream(dev)
        self.E = GpuEinsum(self.stream.cuda_stream)
        self.L = _lib.lib()
        self.sp = ctypes.c_void_p(self.stream.cuda_stream)

    def _sparse(self, x, shape):
        """Row lists stay sparse; a dense 4-D block is converted to rows."""
        if isinstance(x, torch.Tensor) and x.dim() == 4:
            x = x.detach().cpu().numpy()
        if isinstance(x, np.ndarray) and x.ndim == 4:
            idx = np.argwhere(x != 0)
            x = (idx, x[tuple(idx.T)])
        return _rows_dev(x, self.dev)

    def _term(self, name, ops, target, tmp=None):
        coef, spec, names, perm = TERMS[name]
        args = [ops[n] for n in names]
        if perm == 0:
            self.E(spec, *args, out=target, alpha=coef, beta=1.0)
        else:
            self.E(spec, *args, out=tmp, alpha=coef, beta=0.0)
            _lib.check(self.L.nlb_antisym_acc_f64(tmp.data_ptr(), target.data_ptr(), self.p, self.h, perm, 1.0,
                                                  self.sp), "antisym")

    def residuals(self, t1, t2):
        """H1, X_pp, X_hh of t1Iter and H2, X_pp, X_hh of t2Iter at (t1, t2)."""
        p, h, T, nz = self.p, self.h, self.T, self.nonzero
        dev = self.dev
        r = [torch.zeros(s, dtype=torch.float64, device=dev)
             for s in ((p, h), (p, p), (p, p, h, h), (p, p), (p, p, h, h), (p, h, h, h), (p, h, h, h))]
        if self.ppph.nnz:
            ptrs = (ctypes.c_void_p * 7)(*[x.data_ptr() for x in r])
            _lib.check(self.L.nlb_ppph_intermediates_f64(ctypes.byref(self.ppph.c), t1.data_ptr(), t2.data_ptr(),
                                                         p, h, ptrs, self.sp), "ppph")
        ops = dict(T, t1=t1, t2=t2, r3=r[3], r4=r[4], r5=r[5], r6=r[6])
        # T1 equation (coupled_cluster.py:371-408)
        h1 = T["f_ph"].clone()
        xhh1 = -T["f_hh"]
        xpp1 = T["f_pp"].clone()
        self._term("dgram_ck_acik", ops, h1)
        self._term("dgram_ck_ci", ops, xhh1)
        self._term("dgram_ck_ak", ops, xpp1)
        if nz["v_phph"]:
            self._term("dgram_akci_ck", ops, h1)
        if nz["v_phhh"]:
            self._term("dgram_cikl_cakl", ops, h1)
            self._term("dgram_bijk_bj", ops, xhh1)
        if nz["v_pphh"]:
            self._term("dgram_cdkl_ck_dali", ops, h1)
            for n in ("dgram_cdlk_cdli", "dgram_cdlk_cl_di"):
                self._term(n, ops, xhh1)
            for n in ("dgram_dckl_dakl", "dgram_cdkl_dk_al"):
                self._term(n, ops, xpp1)
        h1 += r[0]
        xpp1 += r[1]
        self.E("ac,ci->ai", xpp1, t1, out=h1, beta=1.0)
        self.E("ki,ak->ai", xhh1, t1, out=h1, beta=1.0)
        # T2 equation (coupled_cluster.py:476-536)
        h2 = T["v_pphh"].clone()
        tmp = torch.empty((p, p, h, h), dtype=torch.float64, device=dev)
        self._term("dgram_klij_abkl", ops, h2)
        self._term("dgram_klij_ak_bl", ops, h2, tmp)
        if nz["v_phph"]:
            for n in ("dgram_bkcj_acik", "dgram_bkci_ak_cj"):
                self._term(n, ops, h2, tmp)
        if nz["v_phhh"]:
            for n in ("dgram_bkij_ak", "dgram_cikl_ck_ablj", "dgram_cikl_al_bcjk", "dgram_cjkl_ci_abkl",
                      "dgram_cjkl_ci_ak_bl"):
                self._term(n, ops, h2, tmp)
        if nz["v_pphh"]:
            for n in ("dgram_cdkl_acik_dblj", "dgram_cdkl_cdij_abkl", "dgram_cdkl_ci_dj_abkl",
                      "dgram_cdkl_ak_bl_cdij", "dgram_cdkl_ci_bl_adkj", "dgram_cdkl_ci_ak_dj_bl"):
                self._term(n, ops, h2, tmp)
        xhh2 = -T["f_hh"]
        xpp2 = T["f_pp"].clone()
        self._term("dgram_ck_cj", ops, xhh2)
        self._term("dgram_ck_bk", ops, xpp2)
        if nz["v_pphh"]:
            for n in ("dgram_cdkl_cdjl", "dgram_cdlk_cl_dj"):
                self._term(n, ops, xhh2)
            for n in ("dgram_cdkl_bdkl", "dgram_cdlk_dk_bl"):
                self._term(n, ops, xpp2)
        if self.ppph.nnz:
            _lib.check(self.L.nlb_antisym_acc_f64(r[2].data_ptr(), h2.data_ptr(), p, h, 2, 1.0, self.sp), "pij")
            for n in ("dgram_da_dbij", "dgram_acik_bcjk", "dgram_bijk_ak1", "dgram_bijk_ak2"):
                self._term(n, ops, h2, tmp)
        if self.pppp.nnz or self.pppp_dense is not None:
            l1 = torch.zeros((p, p, h, h), dtype=torch.float64, device=dev)
            l2 = torch.zeros((p, p, h, h), dtype=torch.float64, device=dev)
            if self.pppp_dense is not None:
                # the same sums as the list kernel: l1 = v t2, l2 = v (t1 x t1)
                self.E("abcd,cdij->abij", self.pppp_dense, t2, out=l1)
                self.E("abcd,ci,dj->abij", self.pppp_dense, t1, t1, out=l2)
            else:
                _lib.check(self.L.nlb_pppp_ladders_f64(ctypes.byref(self.pppp.c), t1.data_ptr(), t2.data_ptr(),
                                                       p, h, l1.data_ptr(), l2.data_ptr(), self.sp), "pppp")
            _lib.check(self.L.nlb_antisym_acc_f64(l1.data_ptr(), h2.data_ptr(), p, h, 0, 0.5, self.sp), "l1")
            _lib.check(self.L.nlb_antisym_acc_f64(l2.data_ptr(), h2.data_ptr(), p, h, 2, 0.5, self.sp), "l2")
        self.E("bc,acij->abij", xpp2, t2, out=tmp)
        _lib.check(self.L.nlb_antisym_acc_f64(tmp.data_ptr(), h2.data_ptr(), p, h, 1, 1.0, self.sp), "pab")
        self.E("kj,abik->abij", xhh2, t2, out=tmp)
        _lib.check(self.L.nlb_antisym_acc_f64(tmp.data_ptr(), h2.data_ptr(), p, h, 2, 1.0, self.sp), "pij")
        if self.antisym:
            _lib.check(self.L.nlb_antisym_project_f64(h2.data_ptr(), p, h, self.sp), "project")
        return h1, xpp1, xhh1, h2, xpp2, xhh2

    def energy(self, t1, t2, out):
        v = self.T["v_pphh"] if self.nonzero["v_pphh"] else None
        _lib.check(self.L.nlb_dense_energy_f64(self.T["f_ph"].data_ptr(), t1.data_ptr(),
                                               v.data_ptr() if v is not None else None, t2.data_ptr(), self.p,
                                               self.h, out.data_ptr(), self.work.data_ptr(), self.sp), "energy")


def solve(fock_mats, two_body_int, t1initial=None, eps=1e-8, maxSteps=1000, max_diis=10, delta=0.0, mixing=0.5,
          verbose=False, ccs=False, device=None, criterion="soa", info=None, precision="fp64", mixed_eps=None):
    """The solver loop of ``CCM/soa/coupled_cluster.py:440-575`` (criterion
    ``"soa"``) or ``CCM/coupled_cluster.py:547-687`` (``"numpy"``) on the
    dense GPU engine.  Returns ``(E_corr, t1, t2)`` as CUDA tensors.

    ``precision="mixed"``: the GEMM-shaped contractions run on the tensor
    cores (3xTF32) until the energy test passes at ``mixed_eps`` (default
    ``max(eps, 1e-6)``); the solve then continues from those amplitudes, DIIS
    history included, with FP64 contractions to ``eps``."""
    info = {} if info is None else info
    t0 = time.perf_counter()
    eng = DenseEngine(fock_mats, two_body_int, device)
    mixed = precision == "mixed"
    # 3xTF32 contractions carry about 1e-6 relative error, below which the
    # energy test of the tensor-core phase only sees their noise
    tol = (float(mixed_eps) if mixed_eps is not None else max(float(eps), 1e-6)) if mixed else float(eps)
    eng.E.tensor_cores = mixed
    L, sp, dev = eng.L, eng.sp, device
    p, h = eng.p, eng.h
    n1, n2 = p * h, p * p * h * h
    T = eng.T
    xs = [torch.zeros(n1 + n2, dtype=torch.float64, device=dev) for _ in range(2)]
    cur = 0

    def views(x):
        return x[:n1].view(p, h), x[n1:].view(p, p, h, h)

    t1, t2 = views(xs[cur])
    ep, eh = torch.diagonal(T["f_pp"]), torch.diagonal(T["f_hh"])
    if t1initial is None:
        t1.copy_(T["f_ph"] / (eh[None, :] - ep[:, None] + delta))
    else:
        t1.copy_(torch.as_tensor(np.asarray(t1initial.detach().cpu() if isinstance(t1initial, torch.Tensor)
                                            else t1initial, dtype=np.float64), device=dev))
    if not (ccs or t1initial is not None):
        den = (-ep[:, None, None, None] - ep[None, :, None, None] + eh[None, None, :, None]
               + eh[None, None, None, :] + delta)
        t2.copy_(T["v_pphh"] / den)
    use_diis = criterion == "soa" and max_diis > 0
    if use_diis:
        err = torch.zeros((max_diis, n1 + n2), dtype=torch.float64, device=dev)
        hist = torch.zeros((max_diis, n1 + n2), dtype=torch.float64, device=dev)
        work = torch.zeros(_lib.NLB_DENSE_WORK_DOUBLES, dtype=torch.float64, device=dev)
        nerr = 0
    e_buf = torch.zeros(1, dtype=torch.float64, device=dev)
    eng.energy(t1, t2, e_buf)
    prev = float(e_buf.item())
    if verbose:
        print(f"Step 0: {prev}")
    status, e, it = "max_iter", prev, 0
    for it in range(1, maxSteps + 1):
        t1, t2 = views(xs[cur])
        n1o, n2o = views(xs[cur ^ 1])
        h1, xpp1, xhh1, h2, xpp2, xhh2 = eng.residuals(t1, t2)
        e1 = err[nerr, :n1] if use_diis else None
        e2 = err[nerr, n1:] if use_diis else None
        _lib.check(L.nlb_jacobi_f64(t1.data_ptr(), h1.data_ptr(), None if ccs else t2.data_ptr(),
                                    None if ccs else h2.data_ptr(), xpp1.data_ptr(), xhh1.data_ptr(),
                                    xpp2.data_ptr(), xhh2.data_ptr(), p, h, float(mixing), n1o.data_ptr(),
                                    None if ccs else n2o.data_ptr(),
                                    e1.data_ptr() if e1 is not None else None,
                                    e2.data_ptr() if (e2 is not None and not ccs) else None, sp), "jacobi")
        if ccs:
            n2o.copy_(t2)
            if use_diis:
                e2.zero_()
        cur ^= 1
        t1, t2 = views(xs[cur])
        eng.energy(t1, t2, e_buf)
        e = float(e_buf.item())
        if verbose:
            print(f"Step {it}: {e}", "difference =", abs(e - prev) / abs(e) if e != 0 else float("inf"))
        if criterion == "soa":
            done = abs(e - prev) / max(1.0, abs(e)) < tol
        else:
            done = (e == 0 and prev == 0) or (e != 0 and abs(e - prev) / abs(e) < tol)
        if done and eng.E.tensor_cores:
            # end of the tensor-core phase: FP64 contractions from here on
            eng.E.tensor_cores = False
            info["mixed_iters"] = it
            info["mixed_energy"] = e
            tol = float(eps)
            done = False
        if done:
            status = "converged"
            break
        if use_diis:
            hist[nerr].copy_(xs[cur])
            nerr += 1
            if nerr == max_diis:
                _lib.check(L.nlb_vec_diis_f64(err.data_ptr(), hist.data_ptr(), n1 + n2, max_diis, work.data_ptr(),
                                              xs[cur].data_ptr(), sp), "diis")
                nerr = 0
        if abs(e) > 1e10 or e != e:
            status = "diverged"
            break
        prev = e
    torch.cuda.current_stream(dev).synchronize()
    info.update(status=status, iterations=it, t_iterate=time.perf_counter() - t0,
                launches=eng.E.launches, tc_gemms=eng.E.tc_gemms, gemms=eng.E.gemms)
    t1, t2 = views(xs[cur])
    return e, t1.clone(), t2.clone()
