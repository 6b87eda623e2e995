"""Coupling derivatives of the CCSD energy through the Lambda equations.

The reference has no gradients.  Here, at converged amplitudes t, the
derivative of E_CCSD = E_ref + E_corr with respect to a coupling c is

    dE/dc = dE_ref/dc + <lam1, R1(t; dH)> + <Lam, R2(t; dH)>

where dH = dH/dc is the Hamiltonian built with unit coupling and no kinetic
energy (every block is linear in the couplings, and so is the residual R of
``t1Iter`` / ``t2Iter``), and (lam1, Lam) solve the Lambda equations
``dE/dt + (dR/dt)^T lam = 0`` (CUDA kernels ``nlb_lambda_*``).  Only the
amplitudes at convergence are kept; nothing is taped per iteration.

:func:`lattice_ccsd_energy` wraps a lattice solve in a
``torch.autograd.Function``: ``E.backward()`` fills ``C2.grad`` and
``C3.grad`` (couplings in units of hbar^2/(M a^2); energies in the
reference's unit hbar^2/(2 M a^2)).
"""
from __future__ import annotations

import ctypes
import time

import numpy as np
import torch

from . import _lib
from . import hamiltonian as ham
from . import structure as _structure
from .ccsd import StructuredEngine, ctypes_void, solve_structured


def diag_coefficients(eng, dtwo):
    """Map a derivative Hamiltonian's v_hhhh / v_pppp onto the engine's
    channels as diagonal ladder coefficients (dw, dv), laid out like the
    hole-hole / particle-particle CSR pointer arrays."""
    pl = eng.plan
    hh_idx, hh_val = _structure._coo(dtwo[5])
    pp_idx, pp_val = _structure._coo(dtwo[0])
    dw = np.zeros(max(sum(len(x) for x in pl.hh_ptr), 1))
    dv = np.zeros(max(sum(len(x) for x in pl.pp_ptr), 1))
    hh_off = pp_off = 0
    for n, ch in enumerate(pl.channels):
        if len(hh_val):
            k, l, i, j = hh_idx.T
            m = (pl.h_label[k] == ch.g1) & (pl.h_label[l] == ch.g2) & (pl.h_label[i] == ch.g1) & \
                (pl.h_label[j] == ch.g2)
            if np.any(m & ((k != i) | (l != j))):
                raise ValueError("derivative hole-hole ladder is not diagonal")
            np.add.at(dw, hh_off + pl.h_loc[i[m]] * ch.nh2 + pl.h_loc[j[m]], hh_val[m])
        if len(pp_val):
            a, b, c, d = pp_idx.T
            m = (pl.p_label[a] == ch.g1) & (pl.p_label[b] == ch.g2) & (pl.p_label[c] == ch.g1) & \
                (pl.p_label[d] == ch.g2)
            if np.any(m & ((a != c) | (b != d))):
                raise ValueError("derivative particle-particle ladder is not diagonal")
            np.add.at(dv, pp_off + pl.p_loc[a[m]] * ch.np2 + pl.p_loc[b[m]], pp_val[m])
        hh_off += len(pl.hh_ptr[n])
        pp_off += len(pl.pp_ptr[n])
    return dw, dv


class LambdaSolver:
    """Buffers and captured step graphs of the Lambda iteration for one
    engine (kept on the engine, so repeated gradients reuse them)."""

    def __init__(self, eng):
        L = _lib.lib()
        self.eng = eng
        self.lattice = bool(L.nlb_lambda_lattice(eng.prob))
        self.n_gb = int(L.nlb_lambda_gb_len(eng.prob))
        self._bufs = {}
        self._coef = {}

    def coefficients(self, dfock, dtwo):
        """Device (dw, dv) and the host f_hh block of a derivative
        Hamiltonian, mapped and checked once (its f_pp and f_ph must vanish)."""
        key = (id(dfock), id(dtwo))
        if key not in self._coef:
            df_pp, df_ph, df_hh = [np.asarray(f) for f in dfock]
            if np.any(df_pp) or np.any(df_ph):
                raise ValueError("derivative Fock blocks f_pp/f_ph must vanish (closed-site inputs)")
            dw, dv = diag_coefficients(self.eng, dtwo)
            dev = self.eng.dev
            self._coef[key] = (dfock, dtwo, torch.as_tensor(dw, dtype=torch.float64, device=dev),
                               torch.as_tensor(dv, dtype=torch.float64, device=dev), np.array(df_hh, dtype=np.float64))
        return self._coef[key][2:]

    def buffers(self, dtype_code, max_diis):
        key = (dtype_code, max_diis)
        if key in self._bufs:
            return self._bufs[key]
        L = _lib.lib()
        eng, pl, dev = self.eng, self.eng.plan, self.eng.dev
        tdt = torch.float64 if dtype_code == _lib.NLB_F64 else torch.float32
        f64 = dict(dtype=torch.float64, device=dev)
        ft = dict(dtype=tdt, device=dev)
        b = dict(
            lam1=[torch.zeros(pl.p * pl.h, **f64) for _ in range(2)],
            lam2=[torch.zeros(max(pl.n_t2, 1), **ft) for _ in range(2)],
            t1=torch.zeros(pl.p * pl.h, **f64),
            t2=torch.zeros(max(pl.n_t2, 1), **ft),
            prep=torch.zeros(int(L.nlb_struct_prep_len(eng.prob)), **f64),
            ga=torch.zeros(max(eng.n_g, 1), **ft),
            ha=torch.zeros(max(int(L.nlb_lambda_ha_len(eng.prob)), 1), **ft),
            gb=torch.zeros(max(self.n_gb, 1), **ft),
            acc=torch.zeros(int(L.nlb_lambda_acc_len(eng.prob)), **f64),
            ctrl=torch.zeros(ctypes.sizeof(_lib.Ctrl), dtype=torch.uint8, device=dev),
            diis_t1=torch.zeros(max(max_diis, 1) * pl.p * pl.h, **f64) if max_diis else None,
            diis_t2=torch.zeros(max(max_diis, 1) * max(pl.n_t2, 1), **ft) if max_diis else None,
        )
        st = _lib.LambdaState()
        st.lam1[0], st.lam1[1] = b["lam1"][0].data_ptr(), b["lam1"][1].data_ptr()
        st.lam2[0], st.lam2[1] = b["lam2"][0].data_ptr(), b["lam2"][1].data_ptr()
        st.t1, st.t2, st.prep = b["t1"].data_ptr(), b["t2"].data_ptr(), b["prep"].data_ptr()
        st.ga, st.ha, st.gb = b["ga"].data_ptr(), b["ha"].data_ptr(), b["gb"].data_ptr()
        st.acc, st.ctrl = b["acc"].data_ptr(), b["ctrl"].data_ptr()
        st.diis_t1 = b["diis_t1"].data_ptr() if max_diis else None
        st.diis_t2 = b["diis_t2"].data_ptr() if max_diis else None
        st.dtype = dtype_code
        b["state"] = st
        self._bufs[key] = b
        return b

    def _issue(self, b, n, max_diis, stream):
        L = _lib.lib()
        sp = ctypes_void(stream.cuda_stream)
        for k in range(n):
            _lib.check(L.nlb_lambda_step(self.eng.prob, b["state"], sp), "lambda_step")
            if max_diis and (k + 1) % max_diis == 0:
                _lib.check(L.nlb_lambda_diis(self.eng.prob, b["state"], max_diis, sp), "lambda_diis")

    def _graph(self, b, chunk, max_diis):
        key = ("graph", chunk, max_diis, int(self.eng.prob.tune))   # shapes of the tuning word
        if key not in b:
            dev = self.eng.dev
            side = torch.cuda.Stream(dev)
            side.wait_stream(torch.cuda.current_stream(dev))
            g = torch.cuda.CUDAGraph()
            with torch.cuda.stream(side):
                with torch.cuda.graph(g, stream=side):
                    self._issue(b, chunk, max_diis, side)
            torch.cuda.current_stream(dev).wait_stream(side)
            b[key] = g
        return b[key]

    def run(self, b, tol, mixing, max_steps, max_diis, keep):
        """Iterate to the relative step tol; returns the final ctrl block."""
        L = _lib.lib()
        dev = self.eng.dev
        stream = torch.cuda.current_stream(dev)
        sp = ctypes_void(stream.cuda_stream)
        _lib.check(L.nlb_lambda_init(self.eng.prob, b["state"], tol, mixing, max_steps, max_diis,
                                     _lib.NLB_LAMBDA_KEEP if keep else 0, sp), "lambda_init")
        chunk = max_diis if max_diis else 16
        while chunk < 8:
            chunk += max_diis
        done, launches = 0, 2
        while done < max_steps:
            n = min(chunk, max_steps - done)
            if n == chunk and b.get("warm"):
                self._graph(b, chunk, max_diis).replay()
            else:
                self._issue(b, n, max_diis, stream)
                b["warm"] = True
            launches += 6 * n + (4 * (n // max_diis) if max_diis else 0)
            done += n
            c = _lib.Ctrl.from_buffer_copy(b["ctrl"].cpu().numpy().tobytes())
            if c.status != _lib.NLB_RUNNING:
                break
        self.launches = launches
        return c


def lambda_gradient(eng, t1_dev, t2c_dev, derivs, tol=1e-9, mixing=0.5, max_steps=5000, max_diis=8,
                    precision="mixed", tol_fp32=1e-6, info=None):
    """Solve the Lambda equations at (t1, compact t2) and return dE/dc for each
    derivative Hamiltonian in ``derivs`` (a list of ``(dE_ref, dfock, dtwo)``).

    ``precision="mixed"`` (lattice inputs) iterates the multipliers in FP32
    to the relative step ``tol_fp32`` and continues in FP64 to ``tol``;
    ``"fp64"`` iterates in FP64 throughout.  ``max_diis`` is the pulsed DIIS
    subspace (0: plain Jacobi with mixing)."""
    info = {} if info is None else info
    L = _lib.lib()
    pl, dev = eng.plan, eng.dev
    sp = ctypes_void(torch.cuda.current_stream(dev).cuda_stream)
    if not eng.prob.diag_ladders:
        raise ValueError("the adjoint needs diagonal ladders (SU(4) closed-site inputs)")
    solver = getattr(eng, "_lambda_solver", None)
    if solver is None:
        solver = eng._lambda_solver = LambdaSolver(eng)
    if not solver.lattice:
        precision, max_diis = "fp64", max_diis   # the general path iterates in FP64
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    iters = 0
    launches = 0
    b64 = solver.buffers(_lib.NLB_F64, max_diis)
    b64["t1"].copy_(t1_dev.reshape(-1))
    b64["t2"].copy_(t2c_dev.reshape(-1).to(torch.float64))
    keep = False
    if precision == "mixed":
        b32 = solver.buffers(_lib.NLB_F32, max_diis)
        b32["t1"].copy_(t1_dev.reshape(-1))
        b32["t2"].copy_(t2c_dev.reshape(-1).to(torch.float32))
        c = solver.run(b32, max(tol, tol_fp32), mixing, max_steps, max_diis, keep=False)
        iters += c.iter
        launches += solver.launches
        info["lambda_iters_fp32"] = c.iter
        info["t_lambda_fp32"] = time.perf_counter() - t0   # run() ends on a read of the control block
        if c.status == _lib.NLB_CONVERGED:
            b64["lam1"][0].copy_(b32["lam1"][c.parity])
            _lib.check(L.nlb_convert(b32["lam2"][c.parity].data_ptr(), _lib.NLB_F32, b64["lam2"][0].data_ptr(),
                                     _lib.NLB_F64, pl.n_t2, sp), "convert")
            keep = True
    # continuing from converged FP32 multipliers, the FP64 phase has about two
    # decades left: a DIIS pulse every four steps reaches them in one pulse
    # instead of eight steps (the equations are linear)
    diis64 = min(max_diis, 4) if keep else max_diis
    t1 = time.perf_counter()
    c = solver.run(b64, tol, mixing, max(max_steps - iters, 1), diis64, keep=keep)
    iters += c.iter
    launches += solver.launches
    info["t_lambda_fp64"] = time.perf_counter() - t1
    status = {1: "converged", 2: "max_iter", 3: "diverged"}.get(c.status, "running")
    # After the last step that ran, acc holds U = t1^T lam1 and T for the
    # multipliers that step started from; at convergence they differ from the
    # final ones by less than the tolerance.
    p, h = pl.p, pl.h
    ut = b64["acc"][p * h:p * h + 2 * h * h].cpu().numpy()   # U and T only
    U = ut[:h * h].reshape(h, h)
    T = ut[h * h:].reshape(h, h)
    out = torch.zeros(max(len(derivs), 1), dtype=torch.float64, device=dev)
    coefs = [solver.coefficients(dfock, dtwo) for _, dfock, dtwo in derivs]
    for n, (dw_d, dv_d, _) in enumerate(coefs):
        _lib.check(L.nlb_lambda_coupling(eng.prob, b64["state"], dw_d.data_ptr(), dv_d.data_ptr(),
                                         out[n:].data_ptr(), sp), "lambda_coupling")
        launches += 1
    outn = out.cpu().numpy()
    grads = [float(de_ref) - float(np.sum((U + T) * df_hh)) + float(outn[n])
             for n, ((de_ref, _, _), (_, _, df_hh)) in enumerate(zip(derivs, coefs))]
    torch.cuda.current_stream(dev).synchronize()
    info.update(lambda_status=status, lambda_iters=iters, t_lambda=time.perf_counter() - t0,
                lambda_launches=launches, lambda_precision=precision, lambda_path="lattice" if solver.lattice
                else "general")
    if status != "converged":
        raise RuntimeError(f"Lambda equations did not converge: {status}")
    return grads


_PROBLEMS = {}


def lattice_problem(L, holes):
    """The :class:`LatticeProblem` of (L, holes), built once per process."""
    key = (int(L), repr(np.asarray(holes).tolist()))
    if key not in _PROBLEMS:
        _PROBLEMS[key] = LatticeProblem(L, holes)
    return _PROBLEMS[key]


class LatticeProblem:
    """A closed-shell lattice nucleus: Hamiltonian parts linear in (v, w3)."""

    def __init__(self, L, holes):
        self.L, self.holes = L, holes
        self.dv = ham.normal_ordered_hamiltonian(L, holes, 1.0, 1.0, 0.0, dense=False, kinetic=0.0)
        self.dw = ham.normal_ordered_hamiltonian(L, holes, 0.0, 0.0, 1.0, dense=False, kinetic=0.0)

    def hamiltonian(self, v, w):
        return ham.normal_ordered_hamiltonian(self.L, self.holes, v, v, w, dense=False)


def ccsd_energy_and_gradient(L, holes, C2, C3, device="cuda:0", precision="fp64", eps=1e-12, max_diis=8,
                             maxSteps=5000, lambda_tol=1e-11, mixed_eps=None, info=None, engine=None):
    """E_CCSD and (dE/dC2, dE/dC3) for couplings in units of hbar^2/(M a^2).

    Energies are in the reference unit hbar^2/(2 M a^2); v = 2 C2 and
    w3 = 2 C3 are the reference couplings.  ``engine``: a StructuredEngine
    built earlier for the same (L, holes, C2, C3) (``info["engine"]`` of a
    previous call), reused with its buffers and captured graphs."""
    info = {} if info is None else info
    dev = torch.device(device)
    prob = lattice_problem(L, holes)
    v, w = 2.0 * float(C2), 2.0 * float(C3)
    e_ref, fock, two = prob.hamiltonian(v, w)
    if engine is None:
        plan, why = _structure.detect(fock, two)
        if plan is None:
            raise ValueError(f"the adjoint needs the structured engine: {why}")
        engine = StructuredEngine(plan, fock, dev)
        from . import tune as _tune
        engine.prob.tune = _tune.known_word(engine)
    eng = info["engine"] = engine
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    e, t1, t2c = solve_structured(eng, eps=eps, maxSteps=maxSteps, max_diis=max_diis, precision=precision,
                                  mixed_eps=mixed_eps, t2_format="compact", info=info)
    torch.cuda.synchronize(dev)
    info["t_forward"] = time.perf_counter() - t0
    if info.get("status") != "converged":
        raise RuntimeError(f"CCSD did not converge: {info.get('status')}")
    gv, gw = lambda_gradient(eng, t1, t2c, [prob.dv, prob.dw], tol=lambda_tol, info=info,
                             precision="mixed" if precision == "mixed" else "fp64")
    return e + e_ref, 2.0 * gv, 2.0 * gw


class _CCSDEnergy(torch.autograd.Function):
    @staticmethod
    def forward(ctx, C2, C3, L, holes, device, precision):
        info = {}
        E, g2, g3 = ccsd_energy_and_gradient(L, holes, float(C2), float(C3), device=device, precision=precision,
                                             info=info)
        ctx.grads = (g2, g3)
        ctx.info = info
        return torch.tensor(E, dtype=torch.float64)

    @staticmethod
    def backward(ctx, grad_out):
        g2, g3 = ctx.grads
        return (grad_out * g2, grad_out * g3, None, None, None, None)


def lattice_ccsd_energy(C2, C3, L, holes, device="cuda:0", precision="fp64"):
    """E_CCSD(C2, C3) as a differentiable torch scalar (CPU, FP64).

    ``C2`` and ``C3`` are 0-d float64 tensors (``requires_grad`` as wanted)
    in units of hbar^2/(M a^2).  The forward pass solves CCSD on ``device``
    and, in the same call, the Lambda equations, so ``backward`` only scales
    the stored derivatives."""
    return _CCSDEnergy.apply(C2, C3, L, holes, device, precision)
