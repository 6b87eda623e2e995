"""dE_CCSD/dC2 and dE_CCSD/dC3 from the CUDA Lambda kernels."""
import numpy as np
import pytest
import torch

import golden_io as G
import struct_model as M
import torch_ccsd as TC
from nulattice_b200 import adjoint as A
from nulattice_b200 import hamiltonian as ham
from nulattice_b200 import structure as S
from nulattice_b200.ccsd import StructuredEngine, solve_structured

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def _energy(L, holes, C2, C3):
    v, w = ham.contact_couplings(C2, C3)
    e_ref, fock, two = ham.normal_ordered_hamiltonian(L, holes, v, v, w, dense=False)
    plan, _ = S.detect(fock, two)
    eng = StructuredEngine(plan, fock, torch.device(DEV))
    info = {}
    e, _, _ = solve_structured(eng, eps=1e-14, maxSteps=6000, max_diis=8, t2_format="compact", info=info)
    assert info["status"] == "converged"
    return e + e_ref


@pytest.mark.parametrize("L,A_", [(3, 4), (4, 28)])
def test_gradient_matches_central_differences(L, A_):
    holes = ham.closed_shell_holes(L, A_)
    C2, C3, h = -3.0, 1.0, 1e-4
    info = {}
    E, g2, g3 = A.ccsd_energy_and_gradient(L, holes, C2, C3, device=DEV, info=info)
    fd2 = (_energy(L, holes, C2 + h, C3) - _energy(L, holes, C2 - h, C3)) / (2 * h)
    fd3 = (_energy(L, holes, C2, C3 + h) - _energy(L, holes, C2, C3 - h)) / (2 * h)
    assert abs(g2 - fd2) <= 1e-5 * abs(fd2), (g2, fd2)
    assert abs(g3 - fd3) <= 1e-5 * abs(fd3), (g3, fd3)
    assert info["lambda_status"] == "converged"


def test_gradient_matches_autograd_through_plain_fp64_torch_ccsd():
    L, holes = 3, ham.closed_shell_holes(3, 4)
    C2, C3 = -3.0, 1.0
    E, g2, g3 = A.ccsd_energy_and_gradient(L, holes, C2, C3, device=DEV)
    parts = [ham.normal_ordered_hamiltonian(L, holes, 0, 0, 0, kinetic=1.0),
             ham.normal_ordered_hamiltonian(L, holes, 1, 1, 0, kinetic=0.0),
             ham.normal_ordered_hamiltonian(L, holes, 0, 0, 1, kinetic=0.0)]
    c2 = torch.tensor(C2, dtype=torch.float64, device=DEV, requires_grad=True)
    c3 = torch.tensor(C3, dtype=torch.float64, device=DEV, requires_grad=True)
    H = TC.TorchHam(parts, 2 * c2, 2 * c3, device=DEV)
    e, _, _, _ = TC.solve(H, eps=1e-14, max_steps=4000)
    d2, d3 = torch.autograd.grad(e + H.e_ref, (c2, c3))
    assert float(e + H.e_ref) == pytest.approx(E, rel=1e-11)
    assert g2 == pytest.approx(float(d2), rel=1e-8)
    assert g3 == pytest.approx(float(d3), rel=1e-8)


def test_gpu_lambda_matches_cpu_model_on_o16():
    L, holes = 2, G.load("o16_L2")["holes"]
    E, g2, g3 = A.ccsd_energy_and_gradient(L, holes, -4.5, 3.0, device=DEV, lambda_tol=1e-13)
    prob = A.LatticeProblem(L, holes)
    e_ref, fock, two = ham.normal_ordered_hamiltonian(L, holes, -9.0, -9.0, 6.0)
    plan, _ = S.detect(fock, two)
    from oracle import ccsd_oracle as O
    e, t1, t2, _, _ = O.solve(fock, two, eps=1e-15, maxSteps=6000, max_diis=0, criterion="numpy")
    B = plan.pack_t2(t2)
    lam1, Lam, _ = M.lambda_solve(plan, fock, t1, B, tol=1e-13)
    gv = M.coupling_gradient(plan, prob.dv[1], prob.dv[2], prob.dv[0], t1, B, lam1, Lam)
    gw = M.coupling_gradient(plan, prob.dw[1], prob.dw[2], prob.dw[0], t1, B, lam1, Lam)
    assert g2 == pytest.approx(2 * gv, rel=1e-9)
    assert g3 == pytest.approx(2 * gw, rel=1e-9)


def test_autograd_function_backward():
    L, holes = 3, ham.closed_shell_holes(3, 4)
    C2 = torch.tensor(-3.0, dtype=torch.float64, requires_grad=True)
    C3 = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
    E = A.lattice_ccsd_energy(C2, C3, L, holes, device=DEV)
    (2.0 * E).backward()
    _, g2, g3 = A.ccsd_energy_and_gradient(L, holes, -3.0, 1.0, device=DEV)
    assert float(C2.grad) == pytest.approx(2 * g2, rel=1e-12)
    assert float(C3.grad) == pytest.approx(2 * g3, rel=1e-12)


def test_mixed_precision_forward_with_adjoint():
    L, holes = 4, ham.closed_shell_holes(4, 28)
    _, g2, g3 = A.ccsd_energy_and_gradient(L, holes, -3.0, 1.0, device=DEV)
    _, m2, m3 = A.ccsd_energy_and_gradient(L, holes, -3.0, 1.0, device=DEV, precision="mixed")
    assert m2 == pytest.approx(g2, rel=1e-6)
    assert m3 == pytest.approx(g3, rel=1e-6)


def _converged(L, A_, general=False):
    v, w = ham.contact_couplings(-3.0, 1.0)
    e_ref, fock, two = ham.normal_ordered_hamiltonian(L, ham.closed_shell_holes(L, A_), v, v, w, dense=False)
    plan, _ = S.detect(fock, two)
    eng = StructuredEngine(plan, fock, torch.device(DEV))
    if general:
        eng.prob.max_fpp_offdiag = 99   # neither lattice kernel applies
    info = {}
    e, t1, t2c = solve_structured(eng, eps=1e-14, maxSteps=6000, max_diis=8, t2_format="compact", info=info)
    assert info["status"] == "converged"
    return eng, t1, t2c


@pytest.mark.parametrize("L", [3, 4])
def test_lattice_lambda_steps_match_general_kernels(L):
    """Three Jacobi steps of the Lambda equations from zero: the lattice
    kernels (column + row pass) against the general row kernel, FP64 to
    1e-12 and FP32 to 1e-5, multipliers and the U / T accumulators (the
    lattice path keeps its Z1 contributions in per-writer slots instead of
    the general path's Y1 accumulator; they enter lam1, compared here)."""
    from nulattice_b200 import _lib
    out = {}
    for kind in ("lattice64", "lattice32", "general"):
        eng, t1, t2c = _converged(L, 28, general=(kind == "general"))
        solver = A.LambdaSolver(eng)
        assert solver.lattice == (kind != "general")
        code = _lib.NLB_F32 if kind == "lattice32" else _lib.NLB_F64
        b = solver.buffers(code, 0)
        b["t1"].copy_(t1.reshape(-1))
        b["t2"].copy_(t2c.to(b["t2"].dtype))
        c = solver.run(b, 0.0, 0.5, 3, 0, keep=False)
        assert c.iter == 3
        ph, hh = eng.plan.p * eng.plan.h, eng.plan.h * eng.plan.h
        out[kind] = (b["lam1"][c.parity].cpu().numpy(), b["lam2"][c.parity].double().cpu().numpy(),
                     b["acc"][ph:ph + 2 * hh].cpu().numpy())
    ref = out["general"]
    for kind, tol in (("lattice64", 1e-12), ("lattice32", 2e-5)):
        for got, want in zip(out[kind], ref):
            scale = max(np.abs(want).max(), 1e-30)
            assert np.abs(got - want).max() <= tol * scale, (kind, np.abs(got - want).max() / scale)


def test_lambda_diis_and_mixed_match_jacobi_gradient():
    """The coupling derivatives do not depend on how the Lambda equations are
    iterated: Jacobi, pulsed DIIS, and FP32 DIIS with an FP64 finish."""
    L, A_ = 4, 28
    eng, t1, t2c = _converged(L, A_)
    prob = A.lattice_problem(L, ham.closed_shell_holes(L, A_))
    res = {}
    for name, kw in (("jacobi", dict(max_diis=0, precision="fp64")), ("diis", dict(max_diis=8, precision="fp64")),
                     ("mixed", dict(max_diis=8, precision="mixed"))):
        info = {}
        res[name] = A.lambda_gradient(eng, t1, t2c, [prob.dv, prob.dw], tol=1e-11, info=info, **kw)
        assert info["lambda_status"] == "converged" and info["lambda_path"] == "lattice"
        res[name + "_iters"] = info["lambda_iters"]
    assert res["diis_iters"] < res["jacobi_iters"]
    for name in ("diis", "mixed"):
        np.testing.assert_allclose(res[name], res["jacobi"], rtol=1e-8)
