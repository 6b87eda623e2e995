"""Momentum-block CUDA path vs the oracle, the reference's plane-wave
energies and the general engine."""
import numpy as np
import pytest
import torch

from nulattice_b200 import ccsd_solver
from nulattice_b200 import momentum as MB
from nulattice_b200 import planewave as PW
from oracle import ccsd_oracle as O

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda", 0)


def _engine(L, A, v, vs, w):
    plan = MB.MomentumPlan(L, PW.momentum_holes(L, A))
    V = MB.contact_tensor(L, plan.n_k, v, vs, w)
    fpp, fhh, e_ref = MB.fock_blocks(L, plan.n_k, plan.hmom, plan.pmom, v, vs, w)
    return plan, MB.MomentumEngine(plan, V, fpp, fhh, DEV), (V, fpp, fhh)


@pytest.mark.parametrize("L,A,w,steps", [(2, 4, 0.7, 6), (3, 4, 0.7, 6), (3, 28, 0.7, 3)])
def test_steps_match_the_oracle(L, A, w, steps):
    """Jacobi steps from the MP2 start (the reference's NumPy loop, no DIIS):
    amplitudes in the reference's layout and the energy, against the oracle
    on the dense plane-wave blocks."""
    e_ref, fock, two = PW.plane_wave_hamiltonian(L, PW.momentum_holes(L, A), -6.0, -5.0, w, dense=True)
    plan, eng, (V, fpp, fhh) = _engine(L, A, -6.0, -5.0, w)
    e, t2 = MB.solve(plan, V, fpp, fhh, eps=0.0, maxSteps=steps, max_diis=0, criterion="numpy", engine=eng)
    eo, t1o, t2o, _, _ = O.solve(fock, two, eps=0.0, maxSteps=steps, max_diis=0, criterion="numpy")
    assert not np.any(t1o)
    assert e == pytest.approx(eo, rel=1e-12)
    np.testing.assert_allclose(plan.to_dense(t2), t2o, rtol=0, atol=1e-12 * np.abs(t2o).max())


@pytest.mark.parametrize("key", [(2, -3.0, 1.0), (3, -3.0, 1.0), (3, -6.0, 2.0)])
def test_reference_plane_wave_energies(key):
    """E_ref and E_corr of the reference's plane-wave runs (A=4)."""
    from test_planewave import REF
    L, v, w = key
    info = {}
    e, e_ref, t2, plan = MB.ccsd_plane_wave(L, PW.momentum_holes(L, 4), v, v, w, eps=1e-13, maxSteps=3000,
                                            max_diis=10, device=DEV, info=info)
    assert info["status"] == "converged" and info["engine"] == "momentum"
    assert e_ref == pytest.approx(REF[key][0], abs=1e-11)
    assert e == pytest.approx(REF[key][1], rel=1e-9)


@pytest.mark.parametrize("L,A,w", [(4, 4, 1.0), (3, 28, 0.5)])
def test_matches_the_general_engine(L, A, w):
    """The same solve (pulsed DIIS, soa test) on the dense general engine:
    same energy and amplitudes.  The two engines add their sums in different
    orders, so near the stopping threshold one may take another DIIS cycle
    than the other; the iteration counts are not compared."""
    e_ref, fock, two = PW.plane_wave_hamiltonian(L, PW.momentum_holes(L, A), -4.0, -4.0, w, dense=False)
    i0, i1 = {}, {}
    e0, t1, t2g = ccsd_solver(fock, two, eps=1e-12, maxSteps=2000, max_diis=8, device=DEV, info=i0)
    e1, e_ref1, t2m, plan = MB.ccsd_plane_wave(L, PW.momentum_holes(L, A), -4.0, -4.0, w, eps=1e-12,
                                               maxSteps=2000, max_diis=8, device=DEV, info=i1)
    assert i0["engine"] == "general" and i0["status"] == i1["status"] == "converged"
    assert e_ref1 == pytest.approx(e_ref, rel=1e-13)
    assert e1 == pytest.approx(e0, rel=1e-10)
    np.testing.assert_allclose(plan.to_dense(t2m), t2g, rtol=0, atol=1e-8 * np.abs(t2g).max())


def test_large_closed_shell_reaches_the_fixed_point():
    """L=6, A=28 (4.4 GB as a dense t2, 20 MB blocked): the solve converges,
    an unmixed Jacobi step at the result moves nothing beyond the tolerance,
    and the blocked amplitudes stay exactly antisymmetric."""
    L, A = 6, 28
    plan, eng, (V, fpp, fhh) = _engine(L, A, -4.0, -4.0, 1.0)
    info = {}
    e, t2 = MB.solve(plan, V, fpp, fhh, eps=1e-12, maxSteps=1000, max_diis=8, engine=eng, info=info)
    assert info["status"] == "converged" and np.isfinite(e) and e < 0
    assert MB.jacobi_gap(eng, t2) < 1e-8
    # antisymmetry: t2[b,a,i,j] = -t2[a,b,i,j] through the block tables
    a, b, i, j = plan._index_grid()
    key = ((a * plan.p + b) * plan.h + i) * plan.h + j
    swap = ((b * plan.p + a) * plan.h + i) * plan.h + j
    order = np.argsort(key)
    pos = order[np.searchsorted(key[order], swap)]
    t = t2.cpu().numpy()
    np.testing.assert_array_equal(t[pos], -t)


@pytest.mark.parametrize("L,A,w", [(3, 4, 0.7), (3, 28, 0.5), (6, 28, 1.0)])
def test_mixed_precision_reaches_the_fp64_fixed_point(L, A, w):
    """FP32 amplitudes and intermediates to |dE|/|E| < 1e-8, then FP64 from
    the converted amplitudes: the FP64 solve's energy within 1e-10 and its
    amplitudes within 1e-8 of their largest; the FP32 phase alone within
    1e-6."""
    plan, eng, (V, fpp, fhh) = _engine(L, A, -4.0, -4.0, w)
    i64, imx = {}, {}
    e64, t64 = MB.solve(plan, V, fpp, fhh, eps=1e-12, maxSteps=2000, max_diis=8, engine=eng, info=i64)
    t64 = t64.clone()
    emx, tmx = MB.solve(plan, V, fpp, fhh, eps=1e-12, maxSteps=2000, max_diis=8, engine=eng, info=imx,
                        precision="mixed", mixed_eps=1e-8)
    assert i64["status"] == imx["status"] == "converged", (i64, imx)
    assert imx["mixed_iters"] > 0 and imx["mixed_status"] == "converged"
    assert abs(imx["mixed_energy"] - e64) <= 1e-6 * abs(e64)
    assert emx == pytest.approx(e64, rel=1e-10)
    assert tmx.dtype == torch.float64
    np.testing.assert_allclose(tmx.cpu().numpy(), t64.cpu().numpy(), rtol=0,
                               atol=1e-8 * float(t64.abs().max()))


def test_fp32_step_tracks_the_fp64_step():
    """One FP32 step from the same amplitudes as an FP64 step: the same
    update to FP32 rounding (the kernels are one template)."""
    plan, eng, (V, fpp, fhh) = _engine(4, 28, -4.0, -4.0, 0.5)
    e32 = MB.MomentumEngine(plan, V, fpp, fhh, DEV, dtype=torch.float32, tables=eng)
    x64, y64 = eng.zeros(), eng.zeros()
    eng.init(x64)
    x32, y32 = e32.zeros(), e32.zeros()
    x32.copy_(x64)
    E64, E32 = float(eng.energy(x64).item()), float(e32.energy(x32).item())
    eng.step(x64, y64)
    e32.step(x32, y32)
    torch.cuda.synchronize()
    assert E32 == pytest.approx(E64, rel=1e-6)
    scale = float(y64.abs().max())
    assert float((y32.double() - y64).abs().max()) <= 1e-5 * scale
