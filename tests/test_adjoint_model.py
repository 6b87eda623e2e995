"""The hand-derived Lambda (adjoint) equations on the compact layout, on CPU.

Checked against torch autograd of the Lagrangian (exact J^T lambda), against
central finite differences of the oracle's tight solves, and against autograd
through the unrolled plain FP64 torch CCSD (O-16 at L=2, the reference's own
test fixture)."""
import numpy as np
import pytest
import torch

import golden_io as G
import struct_model as M
import torch_ccsd as TC
from nulattice_b200 import hamiltonian as ham
from nulattice_b200 import structure as S
from oracle import ccsd_oracle as O

V0, W0 = -9.0, 6.0


@pytest.fixture(scope="module")
def o16():
    L, holes = 2, G.load("o16_L2")["holes"]
    parts = [ham.normal_ordered_hamiltonian(L, holes, 0, 0, 0, kinetic=1.0),
             ham.normal_ordered_hamiltonian(L, holes, 1, 1, 0, kinetic=0.0),
             ham.normal_ordered_hamiltonian(L, holes, 0, 0, 1, kinetic=0.0)]
    e_ref, fock, two = ham.normal_ordered_hamiltonian(L, holes, V0, V0, W0)
    plan, _ = S.detect(fock, two)
    e, t1, t2, _, st = O.solve(fock, two, eps=1e-15, maxSteps=5000, max_diis=0, criterion="numpy")
    assert st == "converged"
    return dict(L=L, holes=holes, parts=parts, fock=fock, two=two, plan=plan, t1=t1, B=plan.pack_t2(t2),
                E=e + e_ref)


def test_builder_is_linear_in_the_couplings(o16):
    (ek, fk, tk), (ev, fv, tv), (ew, fw, tw) = o16["parts"]
    e_ref, fock, two = ham.normal_ordered_hamiltonian(o16["L"], o16["holes"], V0, V0, W0)
    assert e_ref == pytest.approx(ek + V0 * ev + W0 * ew, abs=1e-12)
    for f, a, b, c in zip(fock, fk, fv, fw):
        np.testing.assert_allclose(f, a + V0 * b + W0 * c, atol=1e-12)


def _torch_unpack(plan, Bv):
    t2 = torch.zeros((plan.p, plan.p, plan.h, plan.h), dtype=torch.float64)
    for ch in plan.channels:
        P1, P2, H1, H2 = [torch.as_tensor(x) for x in (plan.p_of[ch.g1], plan.p_of[ch.g2], plan.h_of[ch.g1],
                                                       plan.h_of[ch.g2])]
        blk = Bv[ch.offset:ch.offset + ch.size].reshape(ch.np1, ch.np2, ch.nh1, ch.nh2)
        ix = lambda a, b, c, d: (a[:, None, None, None], b[None, :, None, None],  # noqa: E731
                                 c[None, None, :, None], d[None, None, None, :])
        t2 = t2.index_put(ix(P1, P2, H1, H2), blk)
        t2 = t2.index_put(ix(P2, P1, H1, H2), -blk.permute(1, 0, 2, 3))
        t2 = t2.index_put(ix(P1, P2, H2, H1), -blk.permute(0, 1, 3, 2))
        t2 = t2.index_put(ix(P2, P1, H2, H1), blk.permute(1, 0, 3, 2))
    return t2


def _torch_pack(plan, R2):
    out = []
    for ch in plan.channels:
        P1, P2, H1, H2 = [torch.as_tensor(x) for x in (plan.p_of[ch.g1], plan.p_of[ch.g2], plan.h_of[ch.g1],
                                                       plan.h_of[ch.g2])]
        out.append(R2[P1][:, P2][:, :, H1][:, :, :, H2].reshape(-1))
    return torch.cat(out)


def test_lambda_residual_is_the_lagrangian_gradient(o16):
    plan, t1, B = o16["plan"], o16["t1"], o16["B"]
    rng = np.random.default_rng(1)
    lam1 = np.where(plan.t1_mask(), rng.standard_normal(t1.shape), 0.0)
    Lam = rng.standard_normal(plan.n_t2)
    Z1, Z2, _, _ = M.lambda_residual(plan, o16["fock"], t1, B, lam1, Lam)
    H = TC.TorchHam(o16["parts"], torch.tensor(V0, dtype=torch.float64), torch.tensor(W0, dtype=torch.float64))
    t1v = torch.tensor(t1, requires_grad=True)
    Bv = torch.tensor(B, requires_grad=True)
    t2v = _torch_unpack(plan, Bv)
    r1, r2, *_ = TC.residuals(H, t1v, t2v)
    lag = TC.energy(H, t1v, t2v) + torch.sum(torch.tensor(lam1) * r1) + torch.sum(torch.tensor(Lam) * _torch_pack(plan, r2))
    g1, gB = torch.autograd.grad(lag, (t1v, Bv))
    np.testing.assert_allclose(np.where(plan.t1_mask(), g1.numpy(), 0.0), Z1, atol=1e-12)
    np.testing.assert_allclose(gB.numpy(), Z2, atol=1e-12)


def test_coupling_gradient_matches_finite_differences_and_autograd(o16):
    plan, t1, B = o16["plan"], o16["t1"], o16["B"]
    lam1, Lam, it = M.lambda_solve(plan, o16["fock"], t1, B)
    grads = [M.coupling_gradient(plan, d[1], d[2], d[0], t1, B, lam1, Lam) for d in o16["parts"][1:]]

    def etot(v, w):
        e_ref, fock, two = ham.normal_ordered_hamiltonian(o16["L"], o16["holes"], v, v, w)
        e, *_ = O.solve(fock, two, eps=1e-15, maxSteps=8000, max_diis=0, criterion="numpy")
        return e + e_ref

    h = 1e-4
    fd = [(etot(V0 + h, W0) - etot(V0 - h, W0)) / (2 * h), (etot(V0, W0 + h) - etot(V0, W0 - h)) / (2 * h)]
    for g, f in zip(grads, fd):
        assert abs(g - f) <= 1e-7 * abs(f), (g, f)
    v = torch.tensor(V0, dtype=torch.float64, requires_grad=True)
    w = torch.tensor(W0, dtype=torch.float64, requires_grad=True)
    H = TC.TorchHam(o16["parts"], v, w)
    e, _, _, _ = TC.solve(H, eps=1e-15, max_steps=8000)
    dv, dw = torch.autograd.grad(e + H.e_ref, (v, w))
    assert grads[0] == pytest.approx(float(dv), rel=1e-9)
    assert grads[1] == pytest.approx(float(dw), rel=1e-9)
