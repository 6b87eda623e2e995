"""Structured CUDA engine vs the reference (golden vectors) and the oracle."""
import numpy as np
import pytest
import torch

import golden_io as G
from nulattice_b200 import ccsd_solver
from nulattice_b200 import hamiltonian as ham
from oracle import ccsd_oracle as O

pytestmark = pytest.mark.gpu

DEV = "cuda:0"


def _solve(tag, **kw):
    g = G.load(tag)
    fock, two = G.hamiltonian(g)
    info = {}
    out = ccsd_solver(fock, two, device=DEV, info=info, **kw)
    assert info["engine"] == "structured", info
    return g, out, info


@pytest.mark.parametrize("tag", ["o16_L2", "he4_L3_c1", "he4_L3_t5", "he4_L4_c2", "he4_L5_c3"])
def test_tight_energy_matches_reference(tag):
    """Fixed point of the reference's own NumPy solver, 1e-10 relative."""
    g, (e, t1, t2), info = _solve(tag, eps=float(g_eps(tag)), maxSteps=5000, max_diis=0,
                                  criterion="numpy")
    ref = float(g["tight_e"])
    assert info["status"] == "converged"
    assert abs(e - ref) <= 1e-10 * abs(ref), (e, ref)
    np.testing.assert_allclose(t1, g["tight_t1"], atol=1e-10)
    assert np.linalg.norm(t2) == pytest.approx(float(g["tight_t2_norm"]), rel=1e-9)


def g_eps(tag):
    return float(G.load(tag)["tight_eps"])


@pytest.mark.parametrize("tag", ["o16_L2", "he4_L3_c1", "he4_L3_t5", "he4_L4_c2", "he4_L5_c3"])
def test_trajectory_matches_reference(tag):
    g = G.load(tag)
    _, (e, t1, t2), info = _solve(tag, eps=0.0, maxSteps=int(g["traj_steps"]), max_diis=0,
                                  criterion="numpy")
    assert e == pytest.approx(float(g["traj_e"]), rel=1e-12)
    np.testing.assert_allclose(t1, g["traj_t1"], atol=1e-13)
    if "traj_t2_idx" in g:
        np.testing.assert_allclose(t2, G.dense(g, "traj_t2"), atol=1e-13)
    assert np.linalg.norm(t2) == pytest.approx(float(g["traj_t2_norm"]), rel=1e-11)


def test_unmixed_ten_steps():
    g = G.load("o16_L2")
    _, (e, t1, _), _ = _solve("o16_L2", eps=0.0, maxSteps=10, max_diis=0, mixing=0.0, criterion="numpy")
    assert e == pytest.approx(float(g["m0_e"]), rel=1e-12)
    np.testing.assert_allclose(t1, g["m0_t1"], atol=1e-12)


def test_pulsed_diis_matches_torch_solver():
    d = G.load("soa_diis_he4_L3")
    for steps in (4, 9, 13):
        _, (e, t1, t2), _ = _solve("he4_L3_t5", eps=0.0, maxSteps=steps, max_diis=4)
        assert e == pytest.approx(float(d[f"diis_e_{steps}"]), rel=1e-11)
        np.testing.assert_allclose(t1, d[f"diis_t1_{steps}"], atol=1e-11)
        assert np.linalg.norm(t2) == pytest.approx(float(d[f"diis_t2norm_{steps}"]), rel=1e-10)


def test_diis_converges_to_reference_fixed_point():
    g = G.load("he4_L3_t5")
    _, (e, _, _), info = _solve("he4_L3_t5", eps=1e-13, maxSteps=2000, max_diis=8)
    assert info["status"] == "converged"
    assert abs(e - float(g["tight_e"])) <= 1e-10 * abs(float(g["tight_e"]))
    assert info["iterations"] < int(g["tight_iters"])


def test_a28_two_steps_match_reference():
    g = G.load("a28_L4")
    e_ref, fock, two = ham.normal_ordered_hamiltonian(4, g["holes"], -6.0, -6.0, 2.0, dense=False)
    info = {}
    e, t1, t2 = ccsd_solver(fock, two, eps=0.0, maxSteps=int(g["traj_steps"]), max_diis=0, device=DEV,
                            criterion="numpy", info=info)
    assert info["engine"] == "structured"
    assert e == pytest.approx(float(g["traj_e"]), rel=1e-12)
    np.testing.assert_allclose(t1, g["traj_t1"], atol=1e-13)
    assert np.linalg.norm(t2) == pytest.approx(float(g["traj_t2_norm"]), rel=1e-11)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_a28_tight_fixed_point_matches_reference(precision):
    """A=28 (seven closed sites), L=4: the fixed point of the reference's own
    NumPy solver (eps 1e-13, 141 Jacobi steps, Jacobi gap 1e-12).  The
    structured engine with pulsed DIIS, FP64 throughout or FP32 T2 to 1e-8
    and then FP64, reaches it within 1e-10 (the FP32 phase alone within
    1e-6)."""
    g = G.load("a28_L4_tight")
    fock, two = G.hamiltonian(g)
    ref = float(g["tight_e"])
    info = {}
    kw = dict(precision="mixed", mixed_eps=1e-8) if precision == "mixed" else {}
    e, t1, t2 = ccsd_solver(fock, two, eps=1e-13, maxSteps=3000, max_diis=8, device=DEV, info=info, **kw)
    assert info["engine"] == "structured" and info["status"] == "converged", info
    if precision == "mixed":
        assert abs(info["mixed_energy"] - ref) <= 1e-6 * abs(ref), (info, ref)
    assert abs(e - ref) <= 1e-10 * abs(ref), (e, ref)
    np.testing.assert_allclose(t1, g["tight_t1"], atol=1e-9)
    assert np.linalg.norm(t2) == pytest.approx(float(g["tight_t2_norm"]), rel=1e-9)


@pytest.mark.parametrize("tag", ["he4_L3_c1", "he4_L4_c2", "he4_L5_c3"])
def test_mixed_precision_energy(tag):
    g = G.load(tag)
    ref = float(g["tight_e"])
    _, (e, _, _), info = _solve(tag, eps=1e-12, maxSteps=3000, max_diis=8, precision="mixed",
                                mixed_eps=1e-7)
    assert info["status"] == "converged", info
    assert abs(info["mixed_energy"] - ref) <= 1e-6 * abs(ref), (info, ref)
    assert abs(e - ref) <= 1e-10 * abs(ref), (e, ref, info)


def test_compact_output_and_torch_inputs():
    g = G.load("he4_L3_c1")
    fock, two = G.hamiltonian(g)
    ft = [torch.as_tensor(f, device=DEV) for f in fock]
    e, t1, t2c = ccsd_solver(ft, two, eps=0.0, maxSteps=3, max_diis=0, device=DEV, criterion="numpy",
                             t2_format="compact")
    assert isinstance(t1, torch.Tensor) and t1.device.type == "cuda"
    from nulattice_b200 import structure as S
    plan, _ = S.detect(fock, two)
    np.testing.assert_allclose(plan.unpack_t2(t2c.cpu().numpy()), G.dense(g, "traj_t2"), atol=1e-13)


def test_ccs_and_t1initial_match_oracle():
    g = G.load("he4_L3_c1")
    fock, two = G.hamiltonian(g)
    for kw in (dict(ccs=True), dict(t1initial=g["traj_t1"])):
        e, t1, t2 = ccsd_solver(fock, two, eps=0.0, maxSteps=5, max_diis=0, device=DEV, criterion="numpy", **kw)
        eo, t1o, t2o, _, _ = O.solve(fock, two, eps=0.0, maxSteps=5, max_diis=0, criterion="numpy", **kw)
        assert e == pytest.approx(eo, rel=1e-12)
        np.testing.assert_allclose(t1, t1o, atol=1e-13)
        np.testing.assert_allclose(t2, t2o, atol=1e-13)


def test_max_iter_status():
    info = {}
    g = G.load("he4_L3_c1")
    fock, two = G.hamiltonian(g)
    ccsd_solver(fock, two, eps=1e-15, maxSteps=7, max_diis=0, device=DEV, info=info)
    assert info["status"] == "max_iter" and info["iterations"] == 7


def test_nan_input_reports_divergence():
    """A NaN injected on the host into f_pp ends the solve with status diverged."""
    g = G.load("he4_L3_c1")
    fock, two = G.hamiltonian(g)
    fock = [f.copy() for f in fock]
    fock[0][5, 5] = np.nan
    info = {}
    ccsd_solver(fock, two, eps=1e-12, maxSteps=50, max_diis=0, device=DEV, info=info)
    assert info["status"] == "diverged"


def _lattice_engine(L, A, general=False):
    from nulattice_b200 import structure as S
    from nulattice_b200.ccsd import StructuredEngine
    v2, w3 = ham.contact_couplings(-3.0, 1.0)
    e_ref, fock, two = ham.normal_ordered_hamiltonian(L, ham.closed_shell_holes(L, A), v2, v2, w3, dense=False)
    plan, why = S.detect(fock, two)
    assert plan is not None, why
    eng = StructuredEngine(plan, fock, torch.device(DEV))
    assert eng.prob.uniform_nh == 7 and eng.prob.diag_ladders and eng.prob.max_fpp_offdiag == 6
    if general:
        eng.prob.max_fpp_offdiag = 99   # the one-hole-pair-per-thread lattice kernel no longer applies
    return eng


@pytest.mark.parametrize("L", [3, 4, 5])
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-13), ("mixed", 1e-5)])
def test_lattice_t2_kernel_matches_general_kernel(L, precision, tol):
    """Seven-hole lattice T2 kernel vs the general row kernel: same steps,
    DIIS pulses included, on rows of 20, 63 and 118 particles per label."""
    _lattice_vs_general(L, precision, tol, 0)


@pytest.mark.parametrize("L", [3, 4, 5, 6])
@pytest.mark.parametrize("shape", [1, 2, 3, 4, 5, 6, 7, 8])
def test_fp32_lattice_launch_shapes_match_general_kernel(L, shape):
    """Every other FP32 launch shape of the lattice T2 update (512 and 384
    threads, scalar and packed FP32x2 sums, and the two-rows-per-pass kernel
    at 256 to 512 threads, whose blocks also meet single rows at channel
    ends) against the general row kernel, up to rows of 209 particles per
    label."""
    _lattice_vs_general(L, "mixed", 1e-5, shape)


def _lattice_vs_general(L, precision, tol, shape):
    from nulattice_b200.ccsd import solve_structured
    out = []
    for general in (False, True):
        eng = _lattice_engine(L, 28, general)
        eng.prob.tune = shape
        info = {}
        e, t1, t2 = solve_structured(eng, eps=0.0, maxSteps=11, max_diis=4, precision=precision,
                                     mixed_eps=0.0, refine=False, t2_format="compact", info=info)
        out.append((e, t1.cpu().numpy(), t2.double().cpu().numpy()))
    (ea, t1a, t2a), (eb, t1b, t2b) = out
    assert np.abs(t2a).max() > 1e-4
    assert ea == pytest.approx(eb, rel=tol)
    np.testing.assert_allclose(t1a, t1b, atol=tol * np.abs(t1b).max())
    np.testing.assert_allclose(t2a, t2b, atol=tol * np.abs(t2b).max())


def test_index_tables_are_optional():
    """The step kernels' index tables (hole rows, particle of each f_ph /
    f_pp entry, flat t1 index, X_hh hole pair) only shorten load chains:
    without them the same steps come out."""
    from nulattice_b200.ccsd import solve_structured
    out = []
    for tables in (True, False):
        eng = _lattice_engine(4, 28)
        if not tables:
            for name in ("h_row", "fph_prow", "fpp_prow", "t1c_idx", "xc_ki"):
                setattr(eng.prob, name, None)
        e, t1, t2 = solve_structured(eng, eps=0.0, maxSteps=10, max_diis=4, t2_format="compact")
        out.append((e, t1.cpu().numpy(), t2.cpu().numpy()))
    (ea, t1a, t2a), (eb, t1b, t2b) = out
    # the two index paths may contract different products into FMAs: a few
    # ulp per step, amplified by the ten steps and the DIIS pulse
    assert ea == pytest.approx(eb, rel=1e-12)
    np.testing.assert_allclose(t1a, t1b, rtol=0, atol=1e-10 * np.abs(t1b).max())
    np.testing.assert_allclose(t2a, t2b, rtol=0, atol=1e-10 * np.abs(t2b).max())


@pytest.mark.parametrize("key", [(2, -3.0, 1.0), (3, -3.0, 1.0)])
def test_plane_wave_inputs_match_reference(key):
    """Plane-wave inputs (diagonal one-body part, non-zero v_pphh / v_phph /
    v_phhh) go to the general engine and give the reference's correlation
    energy."""
    from nulattice_b200 import planewave as PW
    from test_planewave import REF
    L, v, w = key
    e_ref, fock, two = PW.plane_wave_hamiltonian(L, PW.momentum_holes(L, 4), v, v, w, dense=False)
    info = {}
    e, t1, t2 = ccsd_solver(fock, two, eps=1e-13, maxSteps=3000, max_diis=10, device=DEV, info=info)
    assert info["engine"] == "general" and info["status"] == "converged"
    assert e_ref == pytest.approx(REF[key][0], abs=1e-11)
    assert e == pytest.approx(REF[key][1], rel=1e-9)


def test_plane_wave_L4_steps_match_oracle():
    """Plane waves at L=4 (beyond what the reference solves in minutes):
    five Jacobi steps of the general engine against the oracle."""
    from nulattice_b200 import planewave as PW
    e_ref, fock, two = PW.plane_wave_hamiltonian(4, PW.momentum_holes(4, 4), -3.0, -3.0, 1.0, dense=False)
    e, t1, t2 = ccsd_solver(fock, two, eps=0.0, maxSteps=5, max_diis=0, device=DEV, criterion="numpy")
    dense_two = [two[0], two[1]] + [b.to_dense() for b in two[2:]]
    eo, t1o, t2o, it, st = O.solve(fock, dense_two, eps=0.0, maxSteps=5, max_diis=0, criterion="numpy")
    assert e == pytest.approx(eo, rel=1e-12)
    np.testing.assert_allclose(t2, t2o, rtol=0, atol=1e-12 * np.abs(t2o).max())
