"""Batched scan: many lattice CCSD instances of uneven size, energies and
coupling derivatives, in one CUDA graph launch.

An instance is a closed-shell nucleus (A = 4 or 28 nucleons) on an L^3
lattice with couplings (C2, C3) in units of hbar^2/(M a^2).  Every
Hamiltonian is linear in the couplings, so the parts (kinetic, unit two-body
contact, unit three-body contact) are built once per (L, A) and combined
per instance.  :class:`BatchScan` allocates each instance's buffers, hands
the whole set to ``nlb_batch_create`` (C-ABI, ``batch.cu``) and launches the
captured graph: mixed-precision forward solve with an FP64 finish, then the
Lambda equations (FP32 with an FP64 finish on lattice instances), then the
coupling derivatives -- all instances at once, one launch.

The reference has no batched driver; each instance is the same problem as
one ``ccsd_solver`` call on the reference's lattice Hamiltonian
(``CCM/coupled_cluster.py:547-687``).
"""
from __future__ import annotations

import ctypes
import time

import numpy as np
import torch

from . import _lib
from . import adjoint as _adj
from . import hamiltonian as ham
from . import structure as _structure
from .ccsd import StructuredEngine, _mp2_t1, ctypes_void, ctypes_sizeof_ctrl


def draw_instances(n=64, seed=0):
    """``n`` instances from ``numpy.random.default_rng(seed)``, drawn in the
    order A ~ U{4, 28}, L ~ U{4, 5, 6}, C2 ~ U[-4, -2], C3 ~ U[0, 2] per
    instance (couplings in units of hbar^2/(M a^2))."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        A = int(rng.choice([4, 28]))
        L = int(rng.choice([4, 5, 6]))
        C2 = float(rng.uniform(-4.0, -2.0))
        C3 = float(rng.uniform(0.0, 2.0))
        out.append((A, L, C2, C3))
    return out


def instance_cost(A, L):
    """Compact T2 length of a closed-shell instance: four labels, A/4 holes and
    L^3 - A/4 particles per label, six label-pair channels."""
    nh = A // 4
    npl = L ** 3 - nh
    return 6 * npl * npl * nh * nh


def shard(instances, rank, world):
    """The instances rank `rank` of `world` GPUs solves: largest first onto the
    least-loaded rank (by compact T2 size), deterministic, disjoint, together
    all of them.  The batch needs no communication between ranks."""
    load = [0] * world
    owner = {}
    order = sorted(range(len(instances)), key=lambda i: (-instance_cost(instances[i][0], instances[i][1]), i))
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        owner[i] = r
        load[r] += instance_cost(instances[i][0], instances[i][1])
    return [instances[i] for i in range(len(instances)) if owner[i] == rank]


def max_over_ranks(x, device=None):
    """The largest value of ``x`` over the ranks of the default process group
    (the job's time is the slowest rank's); ``x`` itself without one.  NCCL
    groups reduce on ``device`` (the rank's GPU), others on the CPU."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    if device is None:
        device = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_results(local):
    """Every rank's list of per-instance results, concatenated in rank order
    (one ``all_gather_object``); ``local`` itself without a process group."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return list(local)
    parts = [None] * dist.get_world_size()
    dist.all_gather_object(parts, list(local))
    return [r for p in parts for r in p]


def combine(parts, coeffs):
    """sum_k c_k H_k of builder outputs (E_ref, fock, two-body blocks); sparse
    blocks are concatenated (repeated keys are summed downstream)."""
    e_ref = sum(c * p[0] for c, p in zip(coeffs, parts))
    fock = [sum(c * p[1][k] for c, p in zip(coeffs, parts)) for k in range(3)]
    two = []
    for k in range(6):
        blocks = [(c, p[2][k]) for c, p in zip(coeffs, parts)]
        first = blocks[0][1]
        if isinstance(first, ham.Block):
            idx = np.concatenate([b.indices for _, b in blocks])
            val = np.concatenate([c * b.values for c, b in blocks])
            two.append(ham.Block(first.shape, idx, val))
        else:
            rows = [np.asarray(b, dtype=np.float64).reshape(-1, 5).copy() for _, b in blocks]
            for (c, _), r in zip(blocks, rows):
                r[:, 4] *= c
            two.append(np.concatenate(rows))
    return e_ref, fock, two


_PARTS = {}


def lattice_parts(L, A):
    """(kinetic, unit contact, unit three-body) builder outputs of (L, A)."""
    key = (int(L), int(A))
    if key not in _PARTS:
        holes = ham.closed_shell_holes(L, A)
        prob = _adj.lattice_problem(L, holes)
        kin = ham.normal_ordered_hamiltonian(L, holes, 0.0, 0.0, 0.0, dense=False, kinetic=1.0)
        _PARTS[key] = (holes, prob, [kin, prob.dv, prob.dw])
    return _PARTS[key]


def instance_hamiltonian(L, A, C2, C3):
    """(E_ref, fock, two) of one instance (reference couplings v = 2 C2, w3 = 2 C3)."""
    _, _, parts = lattice_parts(L, A)
    return combine(parts, [1.0, 2.0 * C2, 2.0 * C3])


class _Instance:
    def __init__(self, A, L, C2, C3, dev, max_diis):
        L_ = _lib.lib()
        self.A, self.L, self.C2, self.C3 = A, L, C2, C3
        holes, prob, _ = lattice_parts(L, A)
        self.prob = prob
        self.e_ref, fock, two = instance_hamiltonian(L, A, C2, C3)
        plan, why = _structure.detect(fock, two)
        if plan is None:
            raise ValueError(f"instance (A={A}, L={L}) needs the structured engine: {why}")
        self.eng = eng = StructuredEngine(plan, fock, dev)
        self.lattice = bool(L_.nlb_lambda_lattice(eng.prob))
        f_pp, f_ph, f_hh = [np.asarray(f) for f in fock]
        t1 = _mp2_t1(f_pp, f_ph, f_hh, 0.0)
        self.e0 = float(np.sum(f_ph * t1))
        self.t1_init = torch.as_tensor(t1.reshape(-1), device=dev)
        pl = plan
        n1, n2 = pl.p * pl.h, max(pl.n_t2, 1)
        self.f32 = eng.buffers(_lib.NLB_F32, max_diis)
        self.f64 = eng.buffers(_lib.NLB_F64, max_diis)
        f64 = dict(dtype=torch.float64, device=dev)
        n_gb = int(L_.nlb_lambda_gb_len(eng.prob))
        prep_len = int(L_.nlb_struct_prep_len(eng.prob))
        acc_len = int(L_.nlb_lambda_acc_len(eng.prob))

        def lam_buffers(tdt, own_t2):
            ft = dict(dtype=tdt, device=dev)
            b = dict(lam1=[torch.zeros(n1, **f64) for _ in range(2)],
                     lam2=[torch.zeros(n2, **ft) for _ in range(2)],
                     t2=torch.zeros(n2, **ft) if own_t2 else None,
                     prep=torch.zeros(prep_len, **f64), ga=torch.zeros(max(eng.n_g, 1), **ft),
                     ha=torch.zeros(max(int(L_.nlb_lambda_ha_len(eng.prob)), 1), **ft),
                     gb=torch.zeros(max(n_gb, 1), **ft),
                     acc=torch.zeros(acc_len, **f64),
                     ctrl=torch.zeros(ctypes_sizeof_ctrl(), dtype=torch.uint8, device=dev))
            return b

        self.l64 = lam_buffers(torch.float64, own_t2=False)
        self.l32 = lam_buffers(torch.float32, own_t2=True) if self.lattice else None
        self.out = torch.zeros(8, **f64)
        solver = _adj.LambdaSolver(eng)
        self.dw_dv = [solver.coefficients(prob.dv[1], prob.dv[2])[:2], solver.coefficients(prob.dw[1], prob.dw[2])[:2]]

    def lambda_state(self, b, dtype, fwd, ring):
        st = _lib.LambdaState()
        st.lam1[0], st.lam1[1] = b["lam1"][0].data_ptr(), b["lam1"][1].data_ptr()
        st.lam2[0], st.lam2[1] = b["lam2"][0].data_ptr(), b["lam2"][1].data_ptr()
        st.t1 = fwd["t1"][0].data_ptr()
        st.t2 = b["t2"].data_ptr() if b["t2"] is not None else fwd["t2"][0].data_ptr()
        st.prep, st.ga, st.ha, st.gb = b["prep"].data_ptr(), b["ga"].data_ptr(), b["ha"].data_ptr(), b["gb"].data_ptr()
        st.acc, st.ctrl = b["acc"].data_ptr(), b["ctrl"].data_ptr()
        st.diis_t1 = ring["diis_t1"].data_ptr() if ring["diis_t1"] is not None else None
        st.diis_t2 = ring["diis_t2"].data_ptr() if ring["diis_t2"] is not None else None
        st.dtype = dtype
        return st

    def item(self):
        it = _lib.BatchItem()
        it.prob = ctypes.pointer(self.eng.prob)
        it.f32 = self.f32["state"]
        it.f64 = self.f64["state"]
        it.l64 = self.lambda_state(self.l64, _lib.NLB_F64, self.f64, self.f64)
        if self.l32 is not None:
            it.l32 = self.lambda_state(self.l32, _lib.NLB_F32, self.f64, self.f32)
        it.t1_init = self.t1_init.data_ptr()
        it.e0 = self.e0
        for d, (dw, dv) in enumerate(self.dw_dv):
            it.dw[d], it.dv[d] = dw.data_ptr(), dv.data_ptr()
        it.out = self.out.data_ptr()
        return it


class BatchScan:
    """The instances of a scan, their buffers and the captured batch graph.

    ``run()`` launches the graph once and returns per-instance results:
    E_CCSD (reference unit hbar^2/(2 M a^2)), dE/dC2, dE/dC3, statuses and
    iteration counts."""

    def __init__(self, instances, device="cuda:0", mixing=0.5, mixed_eps=1e-8, eps=1e-10, lambda_tol_fp32=1e-6,
                 lambda_tol=1e-8, max_steps=500, lambda_max_steps=500, max_diis=8, chunk=8, autotune=True):
        self.dev = torch.device(device)
        self.instances = [_Instance(A, L, C2, C3, self.dev, max_diis) for (A, L, C2, C3) in instances]
        L_ = _lib.lib()
        # launch shapes: tuned once per (L, A) class on its first instance
        self.tuning = {}
        if autotune:
            from . import tune as _tune
            for x in self.instances:
                cls = (x.L, x.A)
                if cls not in self.tuning:
                    info = {}
                    _tune.tune(x.eng, info=info)
                    self.tuning[cls] = (int(x.eng.prob.tune), info)
                x.eng.prob.tune = self.tuning[cls][0]
        items = (_lib.BatchItem * len(self.instances))(*[x.item() for x in self.instances])
        self._items = items
        cfg = _lib.BatchConfig(mixing=mixing, mixed_eps=mixed_eps, eps=eps, lambda_tol_fp32=lambda_tol_fp32,
                               lambda_tol=lambda_tol, max_steps=max_steps, max_diis=max_diis,
                               lambda_max_steps=lambda_max_steps, chunk=chunk,
                               phases=_lib.NLB_PHASE_FWD32 | _lib.NLB_PHASE_FWD64 | _lib.NLB_PHASE_LAMBDA,
                               criterion=_lib.NLB_CRIT_SOA)
        self.cfg = cfg
        handle = ctypes.c_void_p()
        torch.cuda.synchronize(self.dev)
        t0 = time.perf_counter()
        _lib.check(L_.nlb_batch_create(items, len(self.instances), ctypes.byref(cfg), ctypes.byref(handle)),
                   "batch_create")
        self.t_capture = time.perf_counter() - t0
        self.handle = handle

    def launch(self, stream=None):
        stream = torch.cuda.current_stream(self.dev) if stream is None else stream
        _lib.check(_lib.lib().nlb_batch_launch(self.handle, ctypes_void(stream.cuda_stream)), "batch_launch")

    def results(self):
        """Per-instance results after a launch has finished."""
        res = []
        status = {0: "running", 1: "converged", 2: "max_iter", 3: "diverged"}
        for x in self.instances:
            o = x.out.cpu().numpy()
            pl = x.eng.plan
            p, h = pl.p, pl.h
            ut = x.l64["acc"][p * h:p * h + 2 * h * h].cpu().numpy()   # U and T only
            UT = ut[:h * h].reshape(h, h) + ut[h * h:].reshape(h, h)
            grads = []
            ok = int(o[5]) == 1   # the Lambda equations converged (the forward solve did, too)
            for d, part in enumerate((x.prob.dv, x.prob.dw)):
                de_ref, dfock = part[0], part[1]
                g = 2.0 * (float(de_ref) - float(np.sum(UT * np.asarray(dfock[2]))) + float(o[1 + d]))
                grads.append(g if ok else float("nan"))
            res.append(dict(A=x.A, L=x.L, C2=x.C2, C3=x.C3, E=float(o[0]) + x.e_ref, E_corr=float(o[0]),
                            dE_dC2=grads[0], dE_dC3=grads[1], status=status.get(int(o[3]), "?"),
                            lambda_status=status.get(int(o[5]), "?"), iterations=int(o[4]),
                            mixed_iterations=int(o[7]), lambda_iterations=int(o[6]), n_t2=pl.n_t2))
        return res

    def close(self):
        if self.handle:
            _lib.lib().nlb_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # pragma: no cover - interpreter shutdown
            pass
