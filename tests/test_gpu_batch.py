"""The batched scan (one graph launch for many instances) against the
single-instance pipeline on the same instances."""
import numpy as np
import pytest
import torch

from nulattice_b200 import adjoint as A
from nulattice_b200 import batch as B
from nulattice_b200 import hamiltonian as ham

pytestmark = pytest.mark.gpu
DEV = "cuda:0"

# uneven sizes: one hole per label (general kernels) and seven (lattice kernels)
INSTANCES = [(4, 3, -3.0, 1.0), (28, 3, -2.5, 0.5), (28, 4, -3.5, 1.5), (4, 4, -2.2, 0.3), (28, 4, -3.0, 1.0)]


def test_batch_matches_single_instance_pipeline():
    """Same kernels and schedule, but the batch's graph and the pipeline run
    different phase boundaries -- agreement is to what the stopping criteria
    fix (|dE|/|E| < 1e-10 forward, relative step 1e-8 for Lambda)."""
    scan = B.BatchScan(INSTANCES, device=DEV)
    scan.launch()
    torch.cuda.synchronize()
    res = scan.results()
    scan.close()
    for r, (A_, L, C2, C3) in zip(res, INSTANCES):
        assert r["status"] == "converged" and r["lambda_status"] == "converged", r
        info = {}
        E, g2, g3 = A.ccsd_energy_and_gradient(L, ham.closed_shell_holes(L, A_), C2, C3, device=DEV,
                                               precision="mixed", eps=1e-10, mixed_eps=1e-8, lambda_tol=1e-8,
                                               info=info)
        assert r["E"] == pytest.approx(E, rel=1e-8), (r, E)
        assert r["dE_dC2"] == pytest.approx(g2, rel=1e-6), (r, g2)
        assert r["dE_dC3"] == pytest.approx(g3, rel=1e-6), (r, g3)
        # the FP32 phase stops near its noise floor (1e-8), so its length can
        # differ between runs; both pipelines end converged in FP64
        assert r["iterations"] > 0 and info["iterations"] > 0


def test_batch_relaunch_is_reproducible():
    """The graph resets every instance itself: a second launch gives the
    same numbers bit for bit, for seven holes per label (lattice kernels)
    and for one (the general FP64 Lambda path): every reduction adds its
    partial sums in a fixed order."""
    scan = B.BatchScan(INSTANCES[:3], device=DEV)
    scan.launch()
    torch.cuda.synchronize()
    a = scan.results()
    scan.launch()
    torch.cuda.synchronize()
    b = scan.results()
    scan.close()
    for x, y in zip(a, b):
        assert x == y


def _oracle_energy(L, A_, C2, C3):
    """E_CCSD (E_ref + E_corr) of the CPU oracle: the reference's algorithm
    with the torch solver's pulsed DIIS, converged to 1e-12."""
    from oracle import ccsd_oracle as O
    e_ref, fock, two = ham.normal_ordered_hamiltonian(L, ham.closed_shell_holes(L, A_), 2 * C2, 2 * C2, 2 * C3)
    e, t1, t2, it, st = O.solve(fock, two, eps=1e-12, maxSteps=3000, max_diis=8, criterion="soa")
    assert st == "converged"
    return e_ref + e, e


def test_batch_matches_the_oracle():
    """Instances of the scan against the CPU oracle, not only against the
    single-instance pipeline: energies of an A=4 and an A=28 instance at L=3
    within 1e-9, and the A=4 instance's dE/dC2, dE/dC3 against central
    differences (step 1e-4) of the oracle's energies within 1e-6."""
    inst = [(4, 3, -3.2, 1.1), (28, 3, -2.7, 0.6)]
    scan = B.BatchScan(inst, device=DEV)
    scan.launch()
    torch.cuda.synchronize()
    res = scan.results()
    scan.close()
    for r, (A_, L, C2, C3) in zip(res, inst):
        assert r["status"] == "converged" and r["lambda_status"] == "converged", r
        E, e_corr = _oracle_energy(L, A_, C2, C3)
        assert r["E_corr"] == pytest.approx(e_corr, rel=1e-9), (r, e_corr)
        assert r["E"] == pytest.approx(E, rel=1e-9)
    A_, L, C2, C3 = inst[0]
    h = 1e-4
    d2 = (_oracle_energy(L, A_, C2 + h, C3)[0] - _oracle_energy(L, A_, C2 - h, C3)[0]) / (2 * h)
    d3 = (_oracle_energy(L, A_, C2, C3 + h)[0] - _oracle_energy(L, A_, C2, C3 - h)[0]) / (2 * h)
    assert res[0]["dE_dC2"] == pytest.approx(d2, rel=1e-6)
    assert res[0]["dE_dC3"] == pytest.approx(d3, rel=1e-6)
