"""Plane-wave inputs: the builder and the solver against energies the
reference itself produced on these inputs (its get_norm_ordered_ham and
ccsd_solver, run on the plane-wave matrix elements of the lattice contact
Hamiltonian, closed n=0 shell of four nucleons, couplings as contact values
vT1 = vS1 and w3; recorded with the reference run at eps 1e-13)."""
import numpy as np
import pytest

from nulattice_b200 import planewave as PW

# (L, v, w3): (E_ref, E_corr) from the reference
REF = {(2, -3.0, 1.0): (-2.1875, -0.58364681184630),
       (3, -3.0, 1.0): (-0.661179698217, -0.23907614672081),
       (3, -6.0, 2.0): (-1.322359396433, -1.32858694500718)}


@pytest.mark.parametrize("key", list(REF))
def test_reference_energy(key):
    L, v, w = key
    e, f, two = PW.plane_wave_hamiltonian(L, PW.momentum_holes(L, 4), v, v, w)
    assert e == pytest.approx(REF[key][0], abs=1e-11)
    # closed form: half the 12 ordered label-distinct hole pairs, a sixth of
    # the 24 label-distinct hole triples
    assert e == pytest.approx(0.5 * 12 * v / L ** 3 + 24 * w / (6 * L ** 6), abs=1e-14)


def test_structure_of_the_blocks():
    L = 3
    e, f, two = PW.plane_wave_hamiltonian(L, PW.momentum_holes(L, 4), -3.0, -3.0, 1.0)
    f_pp, f_ph, f_hh = f
    # diagonal one-body part, kinetic energy plus traces
    assert np.count_nonzero(f_pp - np.diag(np.diag(f_pp))) == 0
    assert np.count_nonzero(f_ph) == 0
    # antisymmetry of the dense blocks
    v_pphh, v_phph, v_phhh, v_hhhh = two[2:]
    np.testing.assert_array_equal(v_pphh, -v_pphh.transpose(1, 0, 2, 3))
    np.testing.assert_array_equal(v_pphh, -v_pphh.transpose(0, 1, 3, 2))
    np.testing.assert_array_equal(v_hhhh, -v_hhhh.transpose(1, 0, 2, 3))
    assert np.count_nonzero(v_pphh) > 0          # unlike the closed-site position basis
    # momentum conservation in v_pphh: k_a + k_b = k_i + k_j (mod L)
    from nulattice_b200 import hamiltonian as ham
    hole, part = ham.ph_split(PW.momentum_holes(L, 4), L)

    def kv(s):
        k = s // 4
        return np.stack([k // (L * L), (k // L) % L, k % L], -1)
    a, b, i, j = np.nonzero(v_pphh)
    tot = (kv(part[a]) + kv(part[b]) - kv(hole[i]) - kv(hole[j])) % L
    assert np.all(tot == 0)


def test_sparse_and_dense_agree():
    L = 3
    e1, f1, t1 = PW.plane_wave_hamiltonian(L, PW.momentum_holes(L, 4), -6.0, -6.0, 2.0, dense=True)
    e2, f2, t2 = PW.plane_wave_hamiltonian(L, PW.momentum_holes(L, 4), -6.0, -6.0, 2.0, dense=False)
    assert e1 == e2
    for a, b in zip(t1[2:], t2[2:]):
        np.testing.assert_array_equal(a, b.to_dense())


def test_a28_shell_and_bad_holes():
    h = PW.momentum_holes(4, 28)
    assert len(h) == 28
    e, f, two = PW.plane_wave_hamiltonian(4, h, -3.0, -3.0, 0.0, dense=False)
    # closed A=28 shell at L=4: kinetic 2 - 2 cos(pi/2) = 2 for each of the
    # 24 unit-momentum holes, plus half the two-body trace over the 28 * 21
    # ordered hole pairs with distinct labels
    assert e == pytest.approx(24 * 2.0 + 0.5 * (28 * 21) * -3.0 / 4 ** 3, abs=1e-12)
    with pytest.raises(ValueError):
        PW.plane_wave_hamiltonian(3, PW.momentum_holes(3, 4)[:3], -3.0, -3.0, 0.0)


def test_oracle_reproduces_reference_L2():
    """The CPU oracle on the plane-wave inputs gives the reference's
    correlation energy (tight convergence)."""
    from oracle import ccsd_oracle as O
    L, v, w = 2, -3.0, 1.0
    e, f, two = PW.plane_wave_hamiltonian(L, PW.momentum_holes(L, 4), v, v, w)
    res = O.solve(f, two, eps=1e-13, maxSteps=3000, max_diis=10)
    assert res[4] == "converged"
    assert res[0] == pytest.approx(REF[(L, v, w)][1], rel=1e-10)


@pytest.mark.parametrize("L,A,w,steps", [(2, 4, 1.0, 4), (3, 4, 1.0, 4), (3, 28, 0.5, 1)])
def test_pruned_rows_change_nothing(L, A, w, steps):
    """Leaving out the v_pppp / v_ppph rows at total momenta no hole pair
    has gives bit for bit the same solve (they only meet zero amplitudes)."""
    from oracle import ccsd_oracle as O
    out = []
    for prune in (True, False):
        e, f, two = PW.plane_wave_hamiltonian(L, PW.momentum_holes(L, A), -3.0, -3.0, w, prune=prune)
        r = O.solve(f, two, eps=0.0, maxSteps=steps, max_diis=0)
        out.append((e, r[0], r[2], len(two[0])))
    assert out[0][0] == out[1][0] and out[0][1] == out[1][1]
    np.testing.assert_array_equal(out[0][2], out[1][2])
    assert out[0][3] < out[1][3]
