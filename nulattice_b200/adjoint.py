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


def lambda_gradient(eng, t1_dev, t2c_dev, derivs, tol=1e-11, mixing=0.5, max_steps=5000, sync_every=16,
                    info=None):
    """Solve the Lambda equations at (t1, compact t2) and return dE/dc for each
    derivative Hamiltonian in ``derivs`` (a list of ``(dE_ref, dfock, dtwo)``)."""
    info = {} if info is None else info
    L = _lib.lib()
    pl, dev = eng.plan, eng.dev
    sp = ctypes_void(torch.cuda.current_stream(dev).cuda_stream)
    if not eng.prob.diag_ladders:
        raise ValueError("the adjoint needs diagonal ladders (SU(4) closed-site inputs)")
    f64 = dict(dtype=torch.float64, device=dev)
    lam1 = [torch.zeros(pl.p * pl.h, **f64) for _ in range(2)]
    lam2 = [torch.zeros(max(pl.n_t2, 1), **f64) for _ in range(2)]
    prep = torch.zeros(int(L.nlb_struct_prep_len(eng.prob)), **f64)
    ga = torch.zeros(max(eng.n_g, 1), **f64)
    ha = torch.zeros(max(eng.n_g, 1), **f64)
    acc = torch.zeros(int(L.nlb_lambda_acc_len(eng.prob)), **f64)
    ctrl = torch.zeros(ctypes.sizeof(_lib.Ctrl), dtype=torch.uint8, device=dev)
    t1c = t1_dev.reshape(-1).to(torch.float64).contiguous()
    t2c = t2c_dev.to(torch.float64).contiguous()
    st = _lib.LambdaState()
    st.lam1[0], st.lam1[1] = lam1[0].data_ptr(), lam1[1].data_ptr()
    st.lam2[0], st.lam2[1] = lam2[0].data_ptr(), lam2[1].data_ptr()
    st.t1, st.t2, st.prep, st.ga, st.ha = t1c.data_ptr(), t2c.data_ptr(), prep.data_ptr(), ga.data_ptr(), ha.data_ptr()
    st.acc, st.ctrl = acc.data_ptr(), ctrl.data_ptr()
    t0 = time.perf_counter()
    _lib.check(L.nlb_lambda_init(eng.prob, st, tol, mixing, max_steps, sp), "lambda_init")
    done, launches = 0, 2
    while done < max_steps:
        for _ in range(min(sync_every, max_steps - done)):
            _lib.check(L.nlb_lambda_step(eng.prob, st, sp), "lambda_step")
            done += 1
            launches += 5
        c = _lib.Ctrl.from_buffer_copy(ctrl.cpu().numpy().tobytes())
        if c.status != _lib.NLB_RUNNING:
            break
    status = {1: "converged", 2: "max_iter", 3: "diverged"}.get(c.status, "running")
    # After the last step that ran, acc holds U = t1^T lam1 and T for the
    # multipliers that step started from; at convergence they differ from the
    # final ones by less than the tolerance.
    p, h = pl.p, pl.h
    accn = acc.cpu().numpy()
    U = accn[p * h:p * h + h * h].reshape(h, h)
    T = accn[p * h + h * h:p * h + 2 * h * h].reshape(h, h)
    out = torch.zeros(1, **f64)
    grads = []
    for de_ref, dfock, dtwo in derivs:
        df_pp, df_ph, df_hh = [np.asarray(f) for f in dfock]
        if np.any(df_pp) or np.any(df_ph):
            raise ValueError("derivative Fock blocks f_pp/f_ph must vanish (closed-site inputs)")
        dw, dv = diag_coefficients(eng, dtwo)
        dw_d, dv_d = torch.as_tensor(dw, **f64), torch.as_tensor(dv, **f64)
        _lib.check(L.nlb_lambda_coupling(eng.prob, st, dw_d.data_ptr(), dv_d.data_ptr(), out.data_ptr(), sp),
                   "lambda_coupling")
        launches += 1
        grads.append(float(de_ref) - float(np.sum((U + T) * df_hh)) + float(out.item()))
    torch.cuda.current_stream(dev).synchronize()
    info.update(lambda_status=status, lambda_iters=c.iter, t_lambda=time.perf_counter() - t0,
                lambda_launches=launches)
    if status != "converged":
        raise RuntimeError(f"Lambda equations did not converge: {status}")
    return grads


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
    w3 = 2 C3 are the reference couplings."""
    info = {} if info is None else info
    dev = torch.device(device)
    prob = LatticeProblem(L, holes)
    v, w = 2.0 * float(C2), 2.0 * float(C3)
    e_ref, fock, two = prob.hamiltonian(v, w)
    plan, why = _structure.detect(fock, two)
    if plan is None:
        raise ValueError(f"the adjoint needs the structured engine: {why}")
    eng = StructuredEngine(plan, fock, dev)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    e, t1, t2c = solve_structured(eng, eps=eps, maxSteps=maxSteps, max_diis=max_diis, precision=precision,
                                  mixed_eps=mixed_eps, t2_format="compact", info=info)
    torch.cuda.synchronize(dev)
    info["t_forward"] = time.perf_counter() - t0
    if info.get("status") != "converged":
        raise RuntimeError(f"CCSD did not converge: {info.get('status')}")
    gv, gw = lambda_gradient(eng, t1, t2c, [prob.dv, prob.dw], tol=lambda_tol, info=info)
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
