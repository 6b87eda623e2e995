"""Host side of the momentum-block path: plan tables, closed-form Fock blocks
and E_ref against the plane-wave builder, and the blocked layout."""
import numpy as np
import pytest

from nulattice_b200 import hamiltonian as ham
from nulattice_b200 import momentum as MB
from nulattice_b200 import planewave as PW


@pytest.mark.parametrize("L,A,w3", [(3, 4, 0.0), (3, 4, 0.7), (3, 28, 0.7), (4, 28, 1.3)])
def test_fock_blocks_and_reference_energy_match_the_builder(L, A, w3):
    holes = PW.momentum_holes(L, A)
    e_ref, fock, _ = PW.plane_wave_hamiltonian(L, holes, -6.0, -5.0, w3, dense=True)
    plan = MB.MomentumPlan(L, holes)
    fpp, fhh, e2 = MB.fock_blocks(L, plan.n_k, plan.hmom, plan.pmom, -6.0, -5.0, w3)
    assert e2 == pytest.approx(e_ref, rel=1e-13, abs=1e-13)
    pidx = {int(x): q for q, x in enumerate(plan.part)}
    hidx = {int(x): q for q, x in enumerate(plan.hole)}
    f_pp, f_ph, f_hh = fock
    assert not np.any(f_ph)
    for q, m in enumerate(plan.pmom):
        ix = [pidx[int(m) * 4 + s] for s in range(4)]
        np.testing.assert_allclose(fpp[q], f_pp[np.ix_(ix, ix)], atol=1e-13)
    for q, m in enumerate(plan.hmom):
        ix = [hidx[int(m) * 4 + s] for s in range(4)]
        np.testing.assert_allclose(fhh[q], f_hh[np.ix_(ix, ix)], atol=1e-13)
    # the Fock matrices are block-diagonal in momentum: nothing outside the blocks
    blk = np.zeros_like(f_pp, bool)
    for m in plan.pmom:
        ix = [pidx[int(m) * 4 + s] for s in range(4)]
        blk[np.ix_(ix, ix)] = True
    assert not np.any(f_pp[~blk])


@pytest.mark.parametrize("L,A", [(2, 4), (3, 4), (3, 28)])
def test_blocked_layout_covers_every_momentum_allowed_amplitude(L, A):
    holes = PW.momentum_holes(L, A)
    plan = MB.MomentumPlan(L, holes)
    a, b, i, j = plan._index_grid()
    assert len(a) == plan.n_t2 == plan.blk_off[-1]
    # distinct entries, all momentum-conserving, and all such entries present
    key = ((a * plan.p + b) * plan.h + i) * plan.h + j
    assert len(np.unique(key)) == plan.n_t2
    ka, kb = plan.part[a] // 4, plan.part[b] // 4
    ki, kj = plan.hole[i] // 4, plan.hole[j] // 4
    np.testing.assert_array_equal(MB._madd(L, ka, kb), MB._madd(L, ki, kj))
    kp = plan.part // 4
    kh = plan.hole // 4
    allowed = MB._madd(L, kp[:, None, None, None], kp[None, :, None, None]) == \
        MB._madd(L, kh[None, None, :, None], kh[None, None, None, :])
    assert int(allowed.sum()) == plan.n_t2
    rng = np.random.default_rng(1)
    x = rng.standard_normal(plan.n_t2)
    np.testing.assert_array_equal(plan.from_dense(plan.to_dense(x)), x)


def test_plan_sizes_at_the_largest_shells():
    plan = MB.MomentumPlan(6, PW.momentum_holes(6, 28))
    assert len(plan.Ks) == 25 and plan.n_t2 == 2_566_400
    assert plan.p == 836 and plan.h == 28
    plan4 = MB.MomentumPlan(6, PW.momentum_holes(6, 4))
    assert len(plan4.Ks) == 1 and plan4.n_t2 == 55_040
    # tiles cover every block: 64-row x 16-column tiles
    for q in range(len(plan.Ks)):
        t = plan.tiles[plan.tiles[:, 0] == q]
        assert len(t) == -(-int(plan.nr[q]) // MB.TILE_ROWS) * (int(plan.nc[q]) // MB.TILE_COLS)


def test_open_shell_holes_are_rejected():
    holes = PW.momentum_holes(3, 4)[:3]
    with pytest.raises(ValueError):
        MB.MomentumPlan(3, holes)


def test_contact_tensor_is_antisymmetric_and_the_builder_value():
    L, nk = 3, 7
    v = MB.contact_tensor(L, nk, -6.0, -5.0, 0.7)
    np.testing.assert_array_equal(v, -v.transpose(1, 0, 2, 3))
    np.testing.assert_array_equal(v, -v.transpose(0, 1, 3, 2))
    v3 = 2.0 * nk * 0.7 / L ** 3
    np.testing.assert_allclose(v, (PW._vloc_tensor(-6.0, -5.0) + PW._vloc_tensor(v3, v3)) / L ** 3, rtol=1e-15)
    assert ham.contact_couplings(-3.0, 1.0) == (-6.0, 2.0)


@pytest.mark.parametrize("L,A,w3", [(3, 4, 0.7), (3, 28, 0.7)])
def test_blocked_residual_model_matches_the_oracle(L, A, w3):
    """The blocked algebra of the momentum-block kernels (CPU model in
    momentum_model.py) against the oracle's dense T2 residual and dressed
    Fock blocks, at random antisymmetric momentum-conserving amplitudes."""
    import momentum_model as MM
    from oracle import ccsd_oracle as O
    holes = PW.momentum_holes(L, A)
    e_ref, fock, two = PW.plane_wave_hamiltonian(L, holes, -6.0, -5.0, w3, dense=True)
    plan = MB.MomentumPlan(L, holes)
    V = MB.contact_tensor(L, plan.n_k, -6.0, -5.0, w3)
    fpp, fhh, _ = MB.fock_blocks(L, plan.n_k, plan.hmom, plan.pmom, -6.0, -5.0, w3)
    t2 = plan.to_dense(np.random.default_rng(3).standard_normal(plan.n_t2) * 1e-2)
    t2 = 0.25 * ((t2 - t2.transpose(1, 0, 2, 3)) - (t2.transpose(0, 1, 3, 2) - t2.transpose(1, 0, 3, 2)))
    H, Xpp, Xhh = MM.residual(plan, V, fpp, fhh, plan.from_dense(t2))
    h2o, xppo, xhho = O.t2_residual(O.Hamiltonian(fock, two), np.zeros((plan.p, plan.h)), t2)
    # the oracle's residual vanishes outside the momentum blocks
    assert np.abs(h2o).sum() == pytest.approx(np.abs(plan.from_dense(h2o)).sum(), rel=1e-14)
    np.testing.assert_allclose(H, plan.from_dense(h2o), rtol=0, atol=1e-13 * np.abs(h2o).max())
    pidx = {int(x): q for q, x in enumerate(plan.part)}
    hidx = {int(x): q for q, x in enumerate(plan.hole)}
    for q, m in enumerate(plan.pmom):
        ix = [pidx[int(m) * 4 + s] for s in range(4)]
        np.testing.assert_allclose(Xpp[q], xppo[np.ix_(ix, ix)], rtol=0, atol=1e-13)
    for q, m in enumerate(plan.hmom):
        ix = [hidx[int(m) * 4 + s] for s in range(4)]
        np.testing.assert_allclose(Xhh[q], xhho[np.ix_(ix, ix)], rtol=0, atol=1e-13)


def test_blocked_jacobi_step_model_matches_the_oracle():
    """One mixed Jacobi step of the blocked model from the MP2 start against
    the oracle's solver loop (one step, no DIIS) on the dense blocks."""
    import momentum_model as MM
    from oracle import ccsd_oracle as O
    L, A, w3 = 3, 4, 0.7
    holes = PW.momentum_holes(L, A)
    e_ref, fock, two = PW.plane_wave_hamiltonian(L, holes, -6.0, -5.0, w3, dense=True)
    plan = MB.MomentumPlan(L, holes)
    V = MB.contact_tensor(L, plan.n_k, -6.0, -5.0, w3)
    fpp, fhh, _ = MB.fock_blocks(L, plan.n_k, plan.hmom, plan.pmom, -6.0, -5.0, w3)
    _, _, t0, _, _ = O.solve(fock, two, eps=0.0, maxSteps=0, max_diis=0, criterion="numpy")
    _, t1o, t2o, _, _ = O.solve(fock, two, eps=0.0, maxSteps=1, max_diis=0, criterion="numpy")
    assert not np.any(t1o)
    t1 = MM.step(plan, V, fpp, fhh, plan.from_dense(t0), 0.5)
    np.testing.assert_allclose(t1, plan.from_dense(t2o), rtol=0, atol=1e-13 * np.abs(t2o).max())


def test_c_abi_rejects_incomplete_problems_before_any_launch():
    """The momentum-block entry points check their descriptors on the host
    and return NLB_ERR_ARG with a message (no CUDA call is made)."""
    import ctypes
    from nulattice_b200 import _lib
    L = _lib.lib()
    P, S = _lib.PwProblem(), _lib.PwState()
    assert L.nlb_pw_init(None, None, 0.0, None) == _lib.NLB_ERR_ARG
    assert b"nlb_pw_init" in L.nlb_last_error()
    assert L.nlb_pw_energy(ctypes.byref(P), None, ctypes.byref(S), None) == _lib.NLB_ERR_ARG
    assert b"nlb_pw_energy" in L.nlb_last_error()
    assert L.nlb_pw_step(ctypes.byref(P), None, None, None, 0.5, ctypes.byref(S), None) == _lib.NLB_ERR_ARG
    assert b"nlb_pw_step" in L.nlb_last_error()
