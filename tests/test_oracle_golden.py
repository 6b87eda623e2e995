"""The CPU oracle against golden vectors produced by the reference itself."""
import numpy as np
import pytest

import golden_io as G
from oracle import ccsd_oracle as O


@pytest.fixture(scope="module")
def rnd():
    return G.load("dgrams_random")


@pytest.mark.parametrize("name", sorted(O.DIAGRAMS))
def test_diagram(rnd, name):
    coef, spec, names, perm = O.DIAGRAMS[name]
    out = O.diagram(name, **{k: rnd[k] for k in names})
    np.testing.assert_allclose(out, rnd["out_" + name], rtol=1e-10, atol=1e-10)


def test_ppph_intermediates_with_repeated_keys(rnd):
    rows = G.rows(rnd, "v_ppph")
    r = O.ppph_intermediates(rows[:, :4].astype(int), rows[:, 4], rnd["t1"], rnd["t2"])
    for n in range(7):
        np.testing.assert_allclose(r[n], rnd[f"out_v_ppph_dgrams_{n}"], rtol=1e-12, atol=1e-12)


def test_pppp_ladders_with_repeated_keys(rnd):
    rows = G.rows(rnd, "v_pppp")
    l1, l2 = O.pppp_ladders(rows[:, :4].astype(int), rows[:, 4], rnd["t1"], rnd["t2"])
    np.testing.assert_allclose(l1, rnd["out_v_pppp_dgrams_0"], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(l2, rnd["out_v_pppp_dgrams_1"], rtol=1e-12, atol=1e-12)


def test_full_steps_all_blocks(rnd):
    H = O.Hamiltonian([rnd["f_pp"], rnd["f_ph"], rnd["f_hh"]],
                      [G.rows(rnd, "v_pppp"), G.rows(rnd, "v_ppph"), rnd["v_pphh"], rnd["v_phph"],
                       rnd["v_phhh"], rnd["v_hhhh"]])
    np.testing.assert_allclose(O.t1_step(H, rnd["t1"], rnd["t2"]), rnd["out_t1Iter"], rtol=1e-11, atol=1e-11)
    np.testing.assert_allclose(O.t2_step(H, rnd["t1"], rnd["t2"]), rnd["out_t2Iter"], rtol=1e-11, atol=1e-10)
    assert O.energy(H, rnd["t1"], rnd["t2"]) == pytest.approx(float(rnd["out_energy"]), rel=1e-13)


@pytest.mark.parametrize("tag", ["o16_L2", "he4_L3_c1", "he4_L3_t5", "he3_L3", "li6x_L3", "he4_L4_c2",
                                 "he4_L5_c3"])
def test_trajectory(tag):
    g = G.load(tag)
    fock, two = G.hamiltonian(g)
    e, t1, t2, _, _ = O.solve(fock, two, eps=0.0, maxSteps=int(g["traj_steps"]), max_diis=0, criterion="numpy")
    assert e == pytest.approx(float(g["traj_e"]), rel=1e-12)
    np.testing.assert_allclose(t1, g["traj_t1"], atol=1e-13)
    if "traj_t2_idx" in g:
        np.testing.assert_allclose(t2, G.dense(g, "traj_t2"), atol=1e-13)
    assert np.linalg.norm(t2) == pytest.approx(float(g["traj_t2_norm"]), rel=1e-12)


@pytest.mark.parametrize("tag", ["o16_L2", "he4_L3_c1", "he4_L3_t5", "he3_L3"])
def test_tight_fixed_point(tag):
    g = G.load(tag)
    fock, two = G.hamiltonian(g)
    e, t1, t2, it, st = O.solve(fock, two, eps=float(g["tight_eps"]), maxSteps=5000, max_diis=0,
                                criterion="numpy")
    assert st == "converged"
    assert abs(e - float(g["tight_e"])) <= 1e-10 * abs(float(g["tight_e"]))
    np.testing.assert_allclose(t1, g["tight_t1"], atol=1e-10)


def test_unmixed_ten_steps():
    g = G.load("o16_L2")
    fock, two = G.hamiltonian(g)
    e, t1, _, _, _ = O.solve(fock, two, eps=0.0, maxSteps=10, max_diis=0, mixing=0.0, criterion="numpy")
    assert e == pytest.approx(float(g["m0_e"]), rel=1e-12)
    np.testing.assert_allclose(t1, g["m0_t1"], atol=1e-12)


def test_pulsed_diis_matches_torch_solver():
    g = G.load("he4_L3_t5")
    d = G.load("soa_diis_he4_L3")
    fock, two = G.hamiltonian(g)
    for steps in (4, 9, 13):
        e, t1, t2, _, _ = O.solve(fock, two, eps=0.0, maxSteps=steps, max_diis=4, criterion="soa")
        assert e == pytest.approx(float(d[f"diis_e_{steps}"]), rel=1e-11)
        np.testing.assert_allclose(t1, d[f"diis_t1_{steps}"], atol=1e-11)
        assert np.linalg.norm(t2) == pytest.approx(float(d[f"diis_t2norm_{steps}"]), rel=1e-10)


@pytest.mark.parametrize("tag", ["he4_L3_c1", "he4_L5_c3"])
def test_fixed_point_gap_small_at_golden(tag):
    """The reference's tight runs stop at a true fixed point: one more unmixed
    Jacobi step of the reference moves t1 and t2 by less than 1e-12."""
    g = G.load(tag)
    assert max(g["tight_gap"]) < 1e-12


HE3 = [[0, 0, 0, 0, 0], [0, 0, 0, 1, 0], [0, 0, 0, 0, 1]]


@pytest.mark.parametrize("holes", ["he4"])
def test_rotation_invariance_of_the_oracle(holes):
    """Rotating particles and holes separately makes every non-zero block
    dense but leaves the CCSD correlation energy unchanged (the premise of
    the GPU test of dense, rotated-basis inputs)."""
    import rotation
    from nulattice_b200 import hamiltonian as ham
    hl = ham.closed_shell_holes(2, 4) if holes == "he4" else HE3
    e_ref, fock, two = ham.normal_ordered_hamiltonian(2, hl, -6.0, -6.0, 2.0)
    fr, tr = rotation.rotate(fock, two, 3)
    assert np.count_nonzero(tr[0]) > 0.5 * tr[0].size and np.count_nonzero(fr[0]) > 0.5 * fr[0].size
    e0 = O.solve(fock, two, eps=1e-13, maxSteps=3000, max_diis=8)[0]
    e1 = O.solve(fr, [rotation.rows_of(tr[0]), rotation.rows_of(tr[1])] + tr[2:], eps=1e-13, maxSteps=3000,
                 max_diis=8)[0]
    assert e1 == pytest.approx(e0, rel=1e-9)
