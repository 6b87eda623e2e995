"""Drop-in CCSD solver: ``ccsd_solver`` with the reference's arguments.

Mirrors ``NuLattice.CCM.soa.coupled_cluster.ccsd_solver``
(``CCM/soa/coupled_cluster.py:440-575``; NumPy twin
``CCM/coupled_cluster.py:547-687``): same positional and keyword arguments,
same return value ``(E_corr, t1, t2)`` with ``t1[a,i]`` and
``t2[a,b,i,j]`` in the reference layout.  The work runs in hand-written
sm_100a kernels (``nulattice_b200/csrc``) reached through the C ABI of
``include/nulattice_b200.h``; there is no CPU path.

Two engines sit behind the entry point:

* the *structured* engine, for inputs that conserve a label on every state
  with closed hole sites (every lattice configuration of the examples): T2 is
  kept in the compact channel layout of :mod:`nulattice_b200.structure`;
* the *general* engine (:mod:`nulattice_b200.dense`), for anything else: the
  full factorised equation set on dense tensors.

Extra keyword-only arguments (not in the reference):

``precision``  ``"fp64"`` (default) or ``"mixed"`` -- the structured engine
               stores T2 in FP32 and computes the elementwise work in FP32
               (T1, energies, norms and DIIS stay FP64), then finishes with
               FP64 steps until ``eps`` is met; the general engine runs its
               GEMM-shaped contractions on the tensor cores (3xTF32, FP32
               accumulation) until ``mixed_eps``, then in FP64 to ``eps``.
``criterion``  ``"soa"`` (default: ``|dE|/max(1,|E|) < eps`` and pulsed DIIS,
               as the torch solver) or ``"numpy"`` (``|dE|/|E| < eps``, no
               DIIS, as the NumPy solver whose DIIS branch never fires).
``t2_format``  ``"dense"`` (default, reference layout) or ``"compact"``.
``info``       a dict to fill with status, iterations, engine and timings.
``engine``     ``"auto"`` (default), ``"structured"`` or ``"general"``.
"""
from __future__ import annotations

import time

import numpy as np
import torch

from . import _lib
from . import structure as _structure

_CRIT = {"soa": _lib.NLB_CRIT_SOA, "numpy": _lib.NLB_CRIT_NUMPY}
_STATUS = {0: "running", 1: "converged", 2: "max_iter", 3: "diverged"}


def _np(x):
    if isinstance(x, torch.Tensor):
        return x.detach().cpu().numpy()
    if hasattr(x, "to_dense") and not isinstance(x, np.ndarray):
        return np.asarray(x.to_dense())
    return np.asarray(x)


def _stream_ptr(dev):
    return ctypes_void(torch.cuda.current_stream(dev).cuda_stream)


def ctypes_void(v):
    import ctypes
    return ctypes.c_void_p(v)


def _resolve_device(device):
    if device is None:
        if not torch.cuda.is_available():
            raise RuntimeError("nulattice_b200.ccsd_solver needs a CUDA device (none available)")
        return torch.device("cuda", torch.cuda.current_device())
    dev = torch.device(device)
    if dev.type != "cuda":
        raise RuntimeError(f"nulattice_b200.ccsd_solver runs on CUDA devices only, got {dev}")
    if dev.index is None:
        dev = torch.device("cuda", torch.cuda.current_device())
    return dev


class StructuredEngine:
    """Device tables and buffers of one structured problem.

    Building it uploads the channel plan once; :meth:`solve` can then be
    called repeatedly (different initial amplitudes, precision, tolerances).
    """

    def __init__(self, plan, fock_mats, device):
        self.plan = plan
        self.dev = device
        f_pp, f_ph, f_hh = [np.asarray(_np(f), dtype=np.float64) for f in fock_mats]
        self.f_ph_np = f_ph
        self.f_pp_np, self.f_hh_np = f_pp, f_hh
        pl = plan
        G = pl.n_labels
        dev = device
        i32 = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.int32), device=dev)  # noqa: E731
        i64 = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.int64), device=dev)  # noqa: E731
        f64 = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=dev)  # noqa: E731
        p_ord = np.concatenate([pl.p_of[g] for g in range(G)]).astype(np.int32)
        h_ord = np.concatenate([pl.h_of[g] for g in range(G)]).astype(np.int32)
        chans = np.zeros(max(len(pl.channels), 1), dtype=_lib.CHANNEL_DTYPE)
        t2_end, g_end, row_end = [], [], []
        hh_ptr, hh_col, hh_val, pp_ptr, pp_col, pp_val = [], [], [], [], [], []
        goff = foff = rows = hp_off = hc_off = pp_off = pc_off = 0
        max_row = 1
        for n, ch in enumerate(pl.channels):
            nhp = ch.nh1 * ch.nh2
            n_ga = ch.nh1 * ch.np2 * nhp
            chans[n] = (ch.g1, ch.g2, ch.np1, ch.np2, ch.nh1, ch.nh2,
                        pl.p_base[ch.g1], pl.p_base[ch.g2], pl.h_base[ch.g1], pl.h_base[ch.g2],
                        ch.offset, goff, foff, hp_off, hc_off, pp_off, pc_off)
            goff += n_ga
            foff += ch.np1 * ch.nh1
            rows += ch.np1
            max_row = max(max_row, ch.np2 * nhp)
            t2_end.append(ch.offset + ch.size)
            g_end.append(goff)
            row_end.append(rows)
            hh_ptr.append(pl.hh_ptr[n]); hh_col.append(pl.hh_col[n]); hh_val.append(pl.hh_val[n])
            pp_ptr.append(pl.pp_ptr[n]); pp_col.append(pl.pp_col[n]); pp_val.append(pl.pp_val[n])
            hp_off += len(pl.hh_ptr[n]); hc_off += len(pl.hh_col[n])
            pp_off += len(pl.pp_ptr[n]); pc_off += len(pl.pp_col[n])
        n_p = np.array([len(x) for x in pl.p_of]); n_h = np.array([len(x) for x in pl.h_of])
        t1c_base = np.concatenate([[0], np.cumsum(n_p * n_h)]).astype(np.int32)
        xc_base = np.concatenate([[0], np.cumsum(n_h * n_h)]).astype(np.int32)
        self.n_f2, self.n_rows, self.max_row = foff, rows, max_row
        self.max_nh = int(max(1, n_h.max() if len(n_h) else 1))
        self.n_t1c, self.n_xc = int(t1c_base[-1]), int(xc_base[-1])
        self.n_g = goff
        cat = lambda xs, dt: np.concatenate(xs).astype(dt) if xs else np.zeros(1, dt)  # noqa: E731
        T = {}
        T["chan"] = torch.as_tensor(chans.view(np.uint8), device=dev)
        T["t2_end"] = i64(t2_end or [0]); T["g_end"] = i64(g_end or [0]); T["row_end"] = i64(row_end or [0])
        T["t1c_base"] = i32(t1c_base); T["xc_base"] = i32(xc_base)
        T["p_ord"] = i32(p_ord); T["h_ord"] = i32(h_ord)
        T["p_label"] = i32(pl.p_label); T["h_label"] = i32(pl.h_label)
        T["p_loc"] = i32(pl.p_loc); T["h_loc"] = i32(pl.h_loc)
        T["p_base"] = i32(pl.p_base); T["h_base"] = i32(pl.h_base)
        T["fpp_ptr"] = i32(pl.fpp_ptr); T["fpp_col"] = i32(pl.fpp_col if len(pl.fpp_col) else [0])
        T["fpp_val"] = f64(pl.fpp_val if len(pl.fpp_val) else [0.0]); T["fpp_diag"] = f64(np.diag(f_pp))
        T["fph_ptr"] = i32(pl.fph_ptr); T["fph_col"] = i32(pl.fph_col if len(pl.fph_col) else [0])
        T["fph_val"] = f64(pl.fph_val if len(pl.fph_val) else [0.0])
        T["f_ph"] = f64(f_ph); T["f_hh"] = f64(f_hh)
        T["hh_ptr"] = i32(cat(hh_ptr, np.int32)); T["hh_col"] = i32(cat(hh_col, np.int32))
        T["hh_val"] = f64(cat(hh_val, np.float64))
        T["pp_ptr"] = i32(cat(pp_ptr, np.int32)); T["pp_col"] = i32(cat(pp_col, np.int32))
        T["pp_val"] = f64(cat(pp_val, np.float64))
        # index tables that spare the step kernels chains of dependent loads
        h_lab = np.asarray(pl.h_label, np.int64)
        T["h_row"] = i32(np.asarray(pl.h_base, np.int64)[h_lab] + np.asarray(pl.h_loc, np.int64))
        fph_rows = np.repeat(np.arange(len(pl.fph_ptr) - 1), np.diff(pl.fph_ptr))
        fph_lab = np.searchsorted(np.asarray(pl.h_base, np.int64), fph_rows, side="right") - 1
        fpp_rows = np.repeat(np.arange(len(pl.fpp_ptr) - 1), np.diff(pl.fpp_ptr))
        fpp_lab = np.searchsorted(np.asarray(pl.p_base, np.int64), fpp_rows, side="right") - 1
        pb = np.asarray(pl.p_base, np.int64)
        T["fph_prow"] = i32(p_ord[pb[fph_lab] + np.asarray(pl.fph_col, np.int64)] if len(fph_rows) else [0])
        T["fpp_prow"] = i32(p_ord[pb[fpp_lab] + np.asarray(pl.fpp_col, np.int64)] if len(fpp_rows) else [0])
        t1c_idx, xc_ki = [], []
        for g in range(G):
            P_, H_ = np.asarray(pl.p_of[g], np.int64), np.asarray(pl.h_of[g], np.int64)
            t1c_idx.append((P_[:, None] * pl.h + H_[None, :]).ravel())
            xc_ki.append((H_[:, None] * pl.h + H_[None, :]).ravel())
        T["t1c_idx"] = i32(cat(t1c_idx, np.int64))
        T["xc_ki"] = i32(cat(xc_ki, np.int64))
        self.tables = T
        prob = _lib.StructProblem()
        prob.p, prob.h, prob.n_labels, prob.n_channels = pl.p, pl.h, G, len(pl.channels)
        prob.n_t2, prob.n_g, prob.n_f2, prob.n_rows = pl.n_t2, self.n_g, self.n_f2, self.n_rows
        prob.n_t1c, prob.n_xc, prob.max_row, prob.max_nh = self.n_t1c, self.n_xc, self.max_row, self.max_nh
        nhs = {(ch.nh1, ch.nh2) for ch in pl.channels}
        uniform = 0
        if len(nhs) == 1:
            n1, n2 = next(iter(nhs))
            uniform = n1 if n1 == n2 else 0
        prob.uniform_nh = uniform
        # diagonal ladders: at most one entry per output pair, and it is the
        # pair itself (with counts of 0 or 1 the rows that hold an entry are
        # the non-zero counts, in order)
        diag = True
        for n in range(len(pl.channels)):
            for ptr, col in ((pl.hh_ptr[n], pl.hh_col[n]), (pl.pp_ptr[n], pl.pp_col[n])):
                cnt = np.diff(ptr)
                if (cnt.size and cnt.max() > 1) or np.any(np.asarray(col) != np.flatnonzero(cnt)):
                    diag = False
                    break
            if not diag:
                break
        prob.diag_ladders = int(diag)
        # off-diagonal f_pp entries per row (rows label-ordered, columns label-local)
        fp = np.asarray(pl.fpp_ptr)
        row_loc = np.concatenate([np.arange(len(x)) for x in pl.p_of]) if G else np.zeros(0, np.int64)
        row_id = np.repeat(np.arange(len(fp) - 1), np.diff(fp))
        offd = np.asarray(pl.fpp_col) != row_loc[row_id]
        prob.max_fpp_offdiag = int(np.bincount(row_id[offd], minlength=1).max()) if offd.any() else 0
        for k, v in T.items():
            setattr(prob, k, v.data_ptr())
        self.prob = prob
        self._bufs = {}
        self.cache = {}
        self.launches = 0

    # -- buffers ---------------------------------------------------------
    def buffers(self, dtype_code, max_diis):
        key = (dtype_code, max_diis)
        if key in self._bufs:
            return self._bufs[key]
        pl, dev = self.plan, self.dev
        tdt = torch.float64 if dtype_code == _lib.NLB_F64 else torch.float32
        L = _lib.lib()
        b = dict(
            t1=[torch.zeros(pl.p * pl.h, dtype=torch.float64, device=dev) for _ in range(2)],
            t2=[torch.zeros(max(pl.n_t2, 1), dtype=tdt, device=dev) for _ in range(2)],
            g=torch.zeros(max(self.n_g, 1), dtype=tdt, device=dev),
            f2=torch.zeros(max(self.n_f2, 1), dtype=tdt, device=dev),
            prep=torch.zeros(int(L.nlb_struct_prep_len(self.prob)), dtype=torch.float64, device=dev),
            ctrl=torch.zeros(ctypes_sizeof_ctrl(), dtype=torch.uint8, device=dev),
            # the DIIS rings: a pulse reads rows 0 .. max_diis - 1 only after the
            # steps since the last reset have written all of them, so they
            # need no zeroing (822 MB of FP64 ring at L=6, A=28)
            diis_t1=torch.empty(max(max_diis, 1) * pl.p * pl.h, dtype=torch.float64, device=dev)
            if max_diis else None,
            diis_t2=torch.empty(max(max_diis, 1) * max(pl.n_t2, 1), dtype=tdt, device=dev)
            if max_diis else None,
        )
        st = _lib.StructState()
        st.t1[0], st.t1[1] = b["t1"][0].data_ptr(), b["t1"][1].data_ptr()
        st.t2[0], st.t2[1] = b["t2"][0].data_ptr(), b["t2"][1].data_ptr()
        st.g, st.f2 = b["g"].data_ptr(), b["f2"].data_ptr()
        st.prep, st.ctrl = b["prep"].data_ptr(), b["ctrl"].data_ptr()
        st.diis_t1 = b["diis_t1"].data_ptr() if max_diis else None
        st.diis_t2 = b["diis_t2"].data_ptr() if max_diis else None
        st.dtype = dtype_code
        b["state"] = st
        self._bufs[key] = b
        return b

    def _graph_for(self, b, chunk, max_diis, issue):
        """CUDA graph of `chunk` steps (+ the DIIS pulse) on buffers `b`.

        Every kernel reads its buffer parity and status from the device, so
        the same graph serves every chunk of every solve on these buffers."""
        key = ("graph", chunk, max_diis, int(self.prob.tune))
        if key in b:
            return b[key]
        dev = self.dev
        side = torch.cuda.Stream(dev)
        side.wait_stream(torch.cuda.current_stream(dev))
        g = torch.cuda.CUDAGraph()
        with torch.cuda.stream(side):
            # the kernels are run once outside capture by the caller's first
            # chunk; here they are only recorded
            with torch.cuda.graph(g, stream=side):
                issue_on = _issue_factory(self, b, max_diis, side)
                issue_on(chunk)
        torch.cuda.current_stream(dev).wait_stream(side)
        b[key] = g
        return g

    def read_ctrl(self, b):
        raw = b["ctrl"].cpu().numpy().tobytes()
        return _lib.Ctrl.from_buffer_copy(raw)

    # -- a whole solve as one graph launch --------------------------------
    def device_loop(self, t1_init, e0, phases, eps, mixed_eps, mixing, max_steps, criterion, max_diis, chunk):
        """Launch the whole forward solve (FP32 and/or FP64 phases) as one CUDA
        graph with device-side loops (the batch machinery with one instance);
        returns (ctrl of the last phase, its buffers, out[8])."""
        import ctypes
        L = _lib.lib()
        # the graph bakes in the launch shapes of the tuning word
        key = ("loop", phases, float(eps), float(mixed_eps), float(mixing), int(max_steps), int(criterion),
               int(max_diis), int(chunk), float(e0), int(self.prob.tune))
        if not hasattr(self, "_loops"):
            self._loops = {}
            self._loop_t1 = torch.zeros(self.plan.p * self.plan.h, dtype=torch.float64, device=self.dev)
            self._loop_out = torch.zeros(8, dtype=torch.float64, device=self.dev)
        b32 = self.buffers(_lib.NLB_F32, max_diis) if phases & _lib.NLB_PHASE_FWD32 else None
        b64 = self.buffers(_lib.NLB_F64, max_diis) if phases & _lib.NLB_PHASE_FWD64 else None
        if key not in self._loops:
            t_build = time.perf_counter()
            it = _lib.BatchItem()
            it.prob = ctypes.pointer(self.prob)
            if b32 is not None:
                it.f32 = b32["state"]
            if b64 is not None:
                it.f64 = b64["state"]
            it.t1_init = self._loop_t1.data_ptr()
            it.e0 = float(e0)
            it.out = self._loop_out.data_ptr()
            items = (_lib.BatchItem * 1)(it)
            cfg = _lib.BatchConfig(mixing=mixing, mixed_eps=mixed_eps, eps=eps, lambda_tol_fp32=0.0, lambda_tol=0.0,
                                   max_steps=max_steps, max_diis=max_diis, lambda_max_steps=0, chunk=chunk,
                                   phases=phases, criterion=criterion)
            handle = ctypes.c_void_p()
            _lib.check(L.nlb_batch_create(items, 1, ctypes.byref(cfg), ctypes.byref(handle)), "loop create")
            self._loops[key] = (handle, items)
            self.cache["t_loop_build"] = time.perf_counter() - t_build
        handle = self._loops[key][0]
        self._loop_t1.copy_(t1_init.reshape(-1))
        stream = torch.cuda.current_stream(self.dev)
        _lib.check(L.nlb_batch_launch(handle, ctypes_void(stream.cuda_stream)), "loop launch")
        b = b64 if b64 is not None else b32
        return b, self._loop_out.cpu().numpy()   # one small read: energy, status, parity, counts

    # -- one phase of iterations ------------------------------------------
    def run(self, b, t1_init, t2c_init, e0, eps, mixing, max_steps, criterion, max_diis, ccs,
            verbose=False, sync_every=16, step_offset=0, t2_events=None, graph=True):
        """Iterate until the device-side test stops the solve.

        ``t2_events``: a list to receive one (start, end) CUDA-event pair per
        T2-update launch (the stages are then launched one by one)."""
        L = _lib.lib()
        dev = self.dev
        stream = torch.cuda.current_stream(dev)
        sp = ctypes_void(stream.cuda_stream)
        b["t1"][0].copy_(t1_init.reshape(-1))
        if t2c_init is None:
            b["t2"][0].zero_()
        elif t2c_init.data_ptr() != b["t2"][0].data_ptr():
            b["t2"][0].copy_(t2c_init)
        b["t2"][1].zero_()
        b["g"].zero_()
        b["f2"].zero_()
        st = b["state"]
        _lib.check(L.nlb_struct_ctrl_init(b["ctrl"].data_ptr(), eps, mixing, max_steps, criterion,
                                          max_diis, int(bool(ccs)), e0, sp), "ctrl_init")
        use_diis = max_diis > 0 and criterion == _lib.NLB_CRIT_SOA
        # a chunk of steps ends on a DIIS pulse, so it is periodic
        chunk = max_diis if use_diis else sync_every
        if use_diis:
            while chunk < 8:
                chunk += max_diis
        use_graph = graph and not verbose and t2_events is None

        def issue(n_steps, done0):
            for k in range(n_steps):
                if t2_events is None:
                    _lib.check(L.nlb_struct_step(self.prob, st, sp), "step")
                else:
                    for stage in range(_lib.NLB_STAGE_PREP, _lib.NLB_STAGE_FINISH + 1):
                        if stage == _lib.NLB_STAGE_T2:
                            ev0 = torch.cuda.Event(enable_timing=True)
                            ev1 = torch.cuda.Event(enable_timing=True)
                            ev0.record(stream)
                        _lib.check(L.nlb_struct_stage(self.prob, st, stage, sp), "stage")
                        if stage == _lib.NLB_STAGE_T2:
                            ev1.record(stream)
                            t2_events.append((ev0, ev1))
                self.launches += 4   # prep+Ga, T2, T1, finish
                if use_diis and (done0 + k + 1) % max_diis == 0:
                    _lib.check(L.nlb_struct_diis(self.prob, st, max_diis, sp), "diis")
                    self.launches += 4

        done = 0
        prev = e0
        while done < max_steps:
            n = 1 if verbose else min(chunk, max_steps - done)
            if use_graph and n == chunk and b.get("warm"):
                g = self._graph_for(b, chunk, max_diis if use_diis else 0, issue)
                g.replay()
                self.launches += (4 * chunk + (4 * (chunk // max_diis) if use_diis else 0))
            else:
                issue(n, done)
                b["warm"] = True
            done += n
            c = self.read_ctrl(b)
            if verbose:
                e = c.e_last
                diff = abs(e - prev) / abs(e) if e != 0 else float("inf")
                print(f"Step {step_offset + c.iter}: {e}", "difference =", diff)
                prev = e
            if c.status != _lib.NLB_RUNNING:
                break
        c = self.read_ctrl(b)
        return c


def _issue_factory(eng, b, max_diis, stream):
    L = _lib.lib()
    sp = ctypes_void(stream.cuda_stream)
    st = b["state"]

    def issue(n):
        for k in range(n):
            _lib.check(L.nlb_struct_step(eng.prob, st, sp), "step")
            if max_diis and (k + 1) % max_diis == 0:
                _lib.check(L.nlb_struct_diis(eng.prob, st, max_diis, sp), "diis")
    return issue


def ctypes_sizeof_ctrl():
    import ctypes
    return ctypes.sizeof(_lib.Ctrl)


class _LoopResult:
    """The parts of the control block a device-loop solve reports back."""

    def __init__(self, parity, e_last, status):
        self.parity, self.e_last, self.status = parity, e_last, status


def _to_host(t):
    """Device tensor -> numpy array.  Large results land in page-locked
    memory from torch's host cache (a copy at PCIe speed, and the block is
    reused by the next call once the array is freed); small ones take the
    plain pageable copy."""
    if t.device.type != "cuda" or t.numel() * t.element_size() < (1 << 20):
        return t.cpu().numpy()
    out = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
    out.copy_(t)
    return out.numpy()


def _mp2_t1(f_pp, f_ph, f_hh, delta):
    """``t1Init`` (``CCM/coupled_cluster.py:319-340``)."""
    den = np.add.outer(-np.diag(f_pp), np.diag(f_hh)) + delta
    with np.errstate(divide="ignore", invalid="ignore"):
        return f_ph / den


def ccsd_solver(fock_mats, two_body_int, t1initial=None, eps=1e-8, maxSteps=1000, max_diis=10,
                delta=0, mixing=0.5, verbose=False, sparse=True, ccs=False, device=None,
                dtype=torch.float64, *, precision="fp64", criterion="soa", t2_format="dense",
                mixed_eps=None, info=None, engine="auto", loop="eager"):
    """Solve the CCSD equations; returns ``(E_corr, t1, t2)``.

    Arguments as ``CCM/soa/coupled_cluster.py:440-454``: ``fock_mats`` =
    ``[f_pp, f_ph, f_hh]``; ``two_body_int`` = ``[v_pppp, v_ppph, v_pphh,
    v_phph, v_phhh, v_hhhh]`` where ``v_pppp``/``v_ppph`` may be dense arrays,
    ``[a,b,c,d,val]`` row lists, ``(indices, values)`` pairs or objects with
    ``.indices``/``.values`` (repeated keys are summed), and the other blocks
    dense arrays or such sparse objects.  ``sparse`` is accepted for
    compatibility; the form of each block is detected.

    Returns torch tensors on ``device`` when ``f_pp`` is a torch tensor, numpy
    arrays otherwise.  On divergence the last amplitudes are returned (the
    NumPy reference returns None there) and ``info["status"]`` says
    ``"diverged"``.

    ``loop``: "eager" (default: every call builds a fresh engine, so a solve
    graph would be built for one use) or "graph" (the whole solve as one
    graph launch with device-side loops).  ``info`` receives the time of each
    phase: ``t_detect``, ``t_engine``, ``t_solve``, ``t_output``.
    """
    t_start = time.perf_counter()
    dev = _resolve_device(device)
    if criterion not in _CRIT:
        raise ValueError("criterion must be 'soa' or 'numpy'")
    if precision not in ("fp64", "mixed"):
        raise ValueError("precision must be 'fp64' or 'mixed'")
    if max_diis > _lib.MAX_DIIS:
        raise ValueError(f"max_diis must be <= {_lib.MAX_DIIS}")
    if not (0.0 <= float(mixing) <= 1.0):
        raise ValueError("mixing must be in [0, 1]")
    want_torch = isinstance(fock_mats[0], torch.Tensor)
    _lib.lib()  # fail loudly before any work when the library is missing
    if engine not in ("auto", "structured", "general"):
        raise ValueError("engine must be 'auto', 'structured' or 'general'")
    if engine == "general":
        plan, why = None, "general engine requested"
    else:
        t_detect = time.perf_counter()
        plan, why = _structure.detect(fock_mats, two_body_int, t1initial)
        t_detect = time.perf_counter() - t_detect
        if plan is None and engine == "structured":
            raise ValueError(f"structured engine does not apply: {why}")
    if info is None:
        info = {}
    info["t_setup_start"] = t_start
    if engine != "general":
        info["t_detect"] = t_detect
    if plan is None:
        from . import dense as _dense
        info["engine"] = "general"
        info["why_general"] = why
        e, t1, t2 = _dense.solve(fock_mats, two_body_int, t1initial=t1initial, eps=eps, maxSteps=maxSteps,
                                 max_diis=max_diis, delta=delta, mixing=mixing, verbose=verbose, ccs=ccs,
                                 device=dev, criterion=criterion, info=info, precision=precision,
                                 mixed_eps=mixed_eps)
    else:
        info["engine"] = "structured"
        t0 = time.perf_counter()
        eng = StructuredEngine(plan, fock_mats, dev)
        from . import tune as _tune
        eng.prob.tune = _tune.known_word(eng)   # cached or default launch shapes, no timing
        info["t_engine"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        e, t1, t2 = solve_structured(eng, t1initial=t1initial, eps=eps, maxSteps=maxSteps,
                                     max_diis=max_diis, delta=delta, mixing=mixing, verbose=verbose,
                                     ccs=ccs, criterion=criterion, precision=precision,
                                     t2_format=t2_format, mixed_eps=mixed_eps, info=info, loop=loop)
        info["t_solve"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    if info.get("status") == "max_iter":
        print("Max iterations reached.")
    elif info.get("status") == "diverged":
        print("Diverged.")
    if want_torch:
        t1 = t1.to(dtype)
        t2 = t2.to(dtype) if t2 is not None else t2
    else:
        t1 = _to_host(t1)
        t2 = _to_host(t2) if t2 is not None else t2
    info["t_output"] = time.perf_counter() - t0
    info["t_total"] = time.perf_counter() - t_start
    return e, t1, t2


def solve_structured(eng, t1initial=None, eps=1e-8, maxSteps=1000, max_diis=10, delta=0.0, mixing=0.5,
                     verbose=False, ccs=False, criterion="soa", precision="fp64", t2_format="dense",
                     mixed_eps=None, info=None, sync_every=16, t2_events=None, refine=True, loop="graph"):
    """Run the structured engine (already built); see :func:`ccsd_solver`.

    ``loop``: "graph" runs the whole solve as one graph launch with
    device-side loops (the graph is built on the first solve of an engine and
    replayed by later ones); "eager" launches the steps chunk by chunk from
    the host, which costs no graph build and suits an engine used once."""
    info = {} if info is None else info
    L = _lib.lib()
    pl, dev = eng.plan, eng.dev
    crit = _CRIT[criterion]
    if t1initial is None:
        # MP2 start, computed once per engine and delta and kept on the device
        key = ("mp2", float(delta))
        if key not in eng.cache:
            t1 = _mp2_t1(eng.f_pp_np, eng.f_ph_np, eng.f_hh_np, float(delta))
            eng.cache[key] = (torch.as_tensor(np.ascontiguousarray(t1), device=dev), float(np.sum(eng.f_ph_np * t1)))
        t1_dev, e0 = eng.cache[key]
    else:
        t1 = np.asarray(_np(t1initial), dtype=np.float64)
        e0 = float(np.sum(eng.f_ph_np * t1))
        t1_dev = torch.as_tensor(np.ascontiguousarray(t1), device=dev)
    diis = int(max_diis) if crit == _lib.NLB_CRIT_SOA else 0
    sp = ctypes_void(torch.cuda.current_stream(dev).cuda_stream)
    iters = 0
    t0 = time.perf_counter()
    if loop not in ("graph", "eager"):
        raise ValueError("loop must be 'graph' or 'eager'")
    if loop == "graph" and t2_events is None and not verbose and not ccs:
        # the whole solve as one graph launch: device-side loops, no host
        # round trip per chunk of steps
        chunk = diis if diis else sync_every
        while diis and chunk < 8:
            chunk += diis
        me = float(mixed_eps) if mixed_eps is not None else max(float(eps), 1e-7)
        if precision == "mixed":
            phases = _lib.NLB_PHASE_FWD32 | (_lib.NLB_PHASE_FWD64 if refine else 0)
        else:
            phases = _lib.NLB_PHASE_FWD64
        eng.cache.pop("t_loop_build", None)
        b, out = eng.device_loop(t1_dev, e0, phases, eps, me, mixing, maxSteps, crit, diis, chunk)
        if "t_loop_build" in eng.cache:
            info["t_loop_build"] = eng.cache["t_loop_build"]
        iters = int(out[4])
        # kernels run: four per step, four per DIIS pulse, the prologue and report
        eng.launches += 4 * iters + (4 * (iters // diis) if diis else 0) + 3
        if precision == "mixed":
            info["mixed_iters"] = int(out[7])
            info["mixed_energy"] = float(out[2])
            if refine and phases & _lib.NLB_PHASE_FWD64:
                info["refine_iters"] = iters - int(out[7])
        c = _LoopResult(int(out[1]), float(out[0]), int(out[3]))
    elif precision == "mixed":
        b32 = eng.buffers(_lib.NLB_F32, diis)
        me = float(mixed_eps) if mixed_eps is not None else max(float(eps), 1e-7)
        c = eng.run(b32, t1_dev, None, e0, me, mixing, maxSteps, crit, diis, ccs, verbose, sync_every,
                    t2_events=t2_events, graph=loop == "graph")
        iters += c.iter
        info["mixed_iters"] = c.iter
        info["mixed_energy"] = c.e_last
        status = _STATUS[c.status]
        if refine and status == "converged" and c.e_last == c.e_last and maxSteps - iters > 0:
            # continue in FP64 from the FP32 amplitudes
            b64 = eng.buffers(_lib.NLB_F64, diis)
            cur = c.parity
            _lib.check(L.nlb_convert(b32["t2"][cur].data_ptr(), _lib.NLB_F32, b64["t2"][0].data_ptr(),
                                     _lib.NLB_F64, pl.n_t2, sp), "convert")
            c = eng.run(b64, b32["t1"][cur].clone(), b64["t2"][0], c.e_last, eps, mixing, maxSteps - iters,
                        crit, diis, ccs, verbose, sync_every, step_offset=iters, graph=loop == "graph")
            eng.launches += 1
            iters += c.iter
            info["refine_iters"] = c.iter
            b = b64
        else:
            b = b32
    else:
        b = eng.buffers(_lib.NLB_F64, diis)
        c = eng.run(b, t1_dev, None, e0, eps, mixing, maxSteps, crit, diis, ccs, verbose, sync_every,
                    t2_events=t2_events, graph=loop == "graph")
        iters += c.iter
    torch.cuda.current_stream(dev).synchronize()
    info["t_iterate"] = time.perf_counter() - t0
    info["status"] = _STATUS[c.status]
    info["iterations"] = iters
    info["n_t2"] = pl.n_t2
    info["plan"] = pl.info
    cur = c.parity
    e = float(c.e_last)
    t1_out = b["t1"][cur].reshape(pl.p, pl.h).clone()
    dcode = b["state"].dtype
    if t2_format == "compact":
        t2_out = b["t2"][cur][:pl.n_t2].clone()
    else:
        t2_out = torch.zeros((pl.p, pl.p, pl.h, pl.h), dtype=torch.float64, device=dev)
        _lib.check(L.nlb_struct_unpack_t2(eng.prob, b["t2"][cur].data_ptr(), dcode, t2_out.data_ptr(), sp),
                   "unpack")
    return e, t1_out, t2_out
