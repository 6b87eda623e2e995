"""Every engine repeats a solve bit for bit.

No kernel adds floating-point numbers with atomics: each reducing launch
writes one partial sum per block and the consumer adds them in block order,
and the general engine gathers its sparse v_ppph / v_pppp terms in a fixed
row order.  Two identical solves therefore give identical energies,
amplitudes and iteration counts, so the stopping step of a solve does not
depend on how the GPU schedules its blocks.
"""
import numpy as np
import pytest
import torch

from nulattice_b200 import ccsd_solver, hamiltonian as ham
from nulattice_b200 import momentum as MB
from nulattice_b200 import planewave as PW

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda", 0)


def _twice(fn):
    out = []
    for _ in range(2):
        info = {}
        res = fn(info)
        torch.cuda.synchronize()
        out.append((res, info))
    return out


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_structured_engine_repeats(precision):
    """A=28 seven-site cluster at L=4 with pulsed DIIS (soa test)."""
    v2, w3 = ham.contact_couplings(-3.0, 1.0)
    e_ref, fock, two = ham.normal_ordered_hamiltonian(4, ham.closed_shell_holes(4, 28), v2, v2, w3, dense=False)
    runs = _twice(lambda info: ccsd_solver(fock, two, eps=1e-11, maxSteps=400, max_diis=8, device=DEV,
                                           precision=precision, t2_format="compact", info=info))
    (r0, i0), (r1, i1) = runs
    assert i0["engine"] == "structured" and i0["status"] == "converged"
    assert i0["iterations"] == i1["iterations"]
    assert r0[0] == r1[0]
    np.testing.assert_array_equal(np.asarray(r0[1]), np.asarray(r1[1]))
    np.testing.assert_array_equal(np.asarray(r0[2]), np.asarray(r1[2]))


def test_general_engine_repeats():
    """Plane-wave A=28 shell at L=3 (v_pppp and v_ppph rows, three-body term):
    the input on which the iteration count used to vary between runs."""
    e_ref, fock, two = PW.plane_wave_hamiltonian(3, PW.momentum_holes(3, 28), -4.0, -4.0, 0.5, dense=False)
    runs = _twice(lambda info: ccsd_solver(fock, two, eps=1e-12, maxSteps=2000, max_diis=8, device=DEV, info=info))
    (r0, i0), (r1, i1) = runs
    assert i0["engine"] == "general" and i0["status"] == "converged"
    assert i0["iterations"] == i1["iterations"]
    assert r0[0] == r1[0]
    assert torch.equal(torch.as_tensor(r0[2]), torch.as_tensor(r1[2]))


def test_momentum_engine_repeats():
    runs = _twice(lambda info: MB.ccsd_plane_wave(3, PW.momentum_holes(3, 28), -4.0, -4.0, 0.5, eps=1e-12,
                                                  maxSteps=2000, max_diis=8, device=DEV, info=info))
    (r0, i0), (r1, i1) = runs
    assert i0["status"] == "converged" and i0["iterations"] == i1["iterations"]
    assert r0[0] == r1[0]
    assert torch.equal(r0[2], r1[2])


def test_lambda_lattice_path_repeats():
    """The coupling derivatives through the lattice Lambda kernels: the Z1
    contributions, Ha and the X_hh contractions sit in per-writer slots that
    are added in a fixed order, so two gradient solves agree bit for bit."""
    from nulattice_b200 import adjoint as A
    holes = ham.closed_shell_holes(4, 28)
    runs = []
    for _ in range(2):
        info = {}
        E, g2, g3 = A.ccsd_energy_and_gradient(4, holes, -3.0, 1.0, device=DEV, precision="mixed", eps=1e-10,
                                               mixed_eps=1e-8, lambda_tol=1e-9, info=info)
        torch.cuda.synchronize()
        runs.append((E, g2, g3, info["lambda_iters"], info.get("lambda_path")))
    assert runs[0][4] == "lattice"
    assert runs[0] == runs[1]


def test_lambda_general_path_repeats():
    """One hole per label (A=4, L=4) takes the general FP64 Lambda kernels:
    the row kernel's Z1 and X_hh contributions sit in per-row slots added in
    a fixed order by k_l_rows_reduce, so two gradient solves agree bit for
    bit."""
    from nulattice_b200 import adjoint as A
    holes = ham.closed_shell_holes(4, 4)
    runs = []
    for _ in range(2):
        info = {}
        E, g2, g3 = A.ccsd_energy_and_gradient(4, holes, -3.0, 1.0, device=DEV, precision="fp64", eps=1e-11,
                                               lambda_tol=1e-10, info=info)
        torch.cuda.synchronize()
        runs.append((E, g2, g3, info["lambda_iters"], info.get("lambda_path")))
    assert runs[0][4] == "general"
    assert runs[0] == runs[1]
