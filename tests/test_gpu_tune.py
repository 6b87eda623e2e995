"""Every launch shape the autotuner can pick computes the same steps."""
import numpy as np
import pytest
import torch

from nulattice_b200 import adjoint as A
from nulattice_b200 import hamiltonian as ham
from nulattice_b200 import structure as S
from nulattice_b200 import tune as T
from nulattice_b200.ccsd import StructuredEngine, solve_structured

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def _engine(L=4, A_=28):
    v2, w3 = ham.contact_couplings(-3.0, 1.0)
    e_ref, fock, two = ham.normal_ordered_hamiltonian(L, ham.closed_shell_holes(L, A_), v2, v2, w3, dense=False)
    plan, _ = S.detect(fock, two)
    return StructuredEngine(plan, fock, torch.device(DEV))


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-13), ("mixed", 1e-5)])
def test_forward_launch_shapes_agree(precision, tol):
    out = []
    words = [T.word(fwd32=v) for v in T.FWD_F32] if precision == "mixed" else [T.word(fwd64=v) for v in T.FWD_F64]
    for w in words:
        eng = _engine()
        eng.prob.tune = w
        e, t1, t2 = solve_structured(eng, eps=0.0, maxSteps=9, max_diis=4, precision=precision, mixed_eps=0.0,
                                     refine=False, t2_format="compact")
        out.append((e, t1.cpu().numpy(), t2.double().cpu().numpy()))
    for e, t1, t2 in out[1:]:
        assert e == pytest.approx(out[0][0], rel=tol)
        np.testing.assert_allclose(t2, out[0][2], atol=tol * np.abs(out[0][2]).max())


def test_lambda_launch_shapes_agree():
    eng = _engine()
    e, t1, t2c = solve_structured(eng, eps=1e-12, maxSteps=2000, max_diis=8, t2_format="compact")
    prob = A.lattice_problem(4, ham.closed_shell_holes(4, 28))
    ref = None
    for w in (T.word(), T.word(lam32=1), T.word(chunks=2), T.word(lam32=1, chunks=4)):
        eng.prob.tune = w
        g = A.lambda_gradient(eng, t1, t2c, [prob.dv, prob.dw], tol=1e-10, precision="mixed")
        if ref is None:
            ref = g
        np.testing.assert_allclose(g, ref, rtol=1e-8)


def test_tuner_picks_a_valid_word(tmp_path, monkeypatch):
    monkeypatch.setenv("NLB_TUNE_CACHE", str(tmp_path / "tune.json"))
    eng = _engine()
    info = {}
    w = T.tune(eng, info=info)
    d = T.describe(w)
    assert d["t2_fp32"] in T.FWD_F32.values() and d["t2_fp64"] in T.FWD_F64.values()
    assert d["lambda_fp32"] in T.LAM_F32.values() and not info["cached"]
    eng2 = _engine()
    info2 = {}
    assert T.tune(eng2, info=info2) == w and info2["cached"]
