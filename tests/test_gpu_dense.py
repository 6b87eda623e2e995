"""General (dense) CUDA engine vs the reference's golden vectors."""
import numpy as np
import pytest
import torch

import golden_io as G
from nulattice_b200 import ccsd_solver
from nulattice_b200 import dense as D

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda", 0)


@pytest.fixture(scope="module")
def rnd():
    return G.load("dgrams_random")


def _perm(x, perm):
    if perm in (1, 3):
        x = x - x.permute(1, 0, 2, 3)
    if perm in (2, 3):
        x = x - x.permute(0, 1, 3, 2)
    return x


@pytest.mark.parametrize("name", sorted(D.TERMS))
def test_each_diagram(rnd, name):
    coef, spec, names, perm = D.TERMS[name]
    alias = {"r3": "x_pp", "r4": "x_pphh", "r5": "x_phhh", "r6": "x_phhh"}
    ops = [torch.as_tensor(rnd[alias.get(n, n)], device=DEV) for n in names]
    oz = spec.split("->")[1]
    sizes = {}
    for t, o in zip(spec.split("->")[0].split(","), ops):
        for x, s in zip(t, o.shape):
            sizes[x] = s
    out = torch.empty([sizes[x] for x in oz], dtype=torch.float64, device=DEV)
    E = D.GpuEinsum(torch.cuda.current_stream(DEV).cuda_stream)
    E(spec, *ops, out=out, alpha=coef)
    got = _perm(out, perm).cpu().numpy() if perm else out.cpu().numpy()
    np.testing.assert_allclose(got, rnd["out_" + name], rtol=1e-10, atol=1e-10)


def test_full_step_all_blocks(rnd):
    fock = [rnd["f_pp"], rnd["f_ph"], rnd["f_hh"]]
    two = [G.rows(rnd, "v_pppp"), G.rows(rnd, "v_ppph"), rnd["v_pphh"], rnd["v_phph"], rnd["v_phhh"], rnd["v_hhhh"]]
    eng = D.DenseEngine(fock, two, DEV)
    t1 = torch.as_tensor(rnd["t1"], device=DEV)
    t2 = torch.as_tensor(rnd["t2"], device=DEV)
    h1, xpp1, xhh1, h2, xpp2, xhh2 = eng.residuals(t1, t2)
    n1 = t1 + h1 / -(torch.diagonal(xpp1)[:, None] + torch.diagonal(xhh1)[None, :])
    dp, dh = torch.diagonal(xpp2), torch.diagonal(xhh2)
    den = -(dp[:, None, None, None] + dp[None, :, None, None] + dh[None, None, :, None] + dh[None, None, None, :])
    n2 = t2 + h2 / den
    np.testing.assert_allclose(n1.cpu().numpy(), rnd["out_t1Iter"], rtol=1e-11, atol=1e-11)
    np.testing.assert_allclose(n2.cpu().numpy(), rnd["out_t2Iter"], rtol=1e-11, atol=1e-10)
    e = torch.zeros(1, dtype=torch.float64, device=DEV)
    eng.energy(t1, t2, e)
    assert float(e.item()) == pytest.approx(float(rnd["out_energy"]), rel=1e-12)


@pytest.mark.parametrize("tag", ["he3_L3", "li6x_L3", "he4_L3_c1"])
def test_trajectory_general_engine(tag):
    g = G.load(tag)
    fock, two = G.hamiltonian(g)
    info = {}
    e, t1, t2 = ccsd_solver(fock, two, eps=0.0, maxSteps=int(g["traj_steps"]), max_diis=0, device=DEV,
                            criterion="numpy", engine="general", info=info)
    assert info["engine"] == "general"
    assert e == pytest.approx(float(g["traj_e"]), rel=1e-12)
    np.testing.assert_allclose(t1, g["traj_t1"], atol=1e-13)
    np.testing.assert_allclose(t2, G.dense(g, "traj_t2"), atol=1e-13)


@pytest.mark.parametrize("tag", ["he3_L3", "li6x_L3"])
def test_tight_energy_general_engine(tag):
    g = G.load(tag)
    fock, two = G.hamiltonian(g)
    info = {}
    e, t1, t2 = ccsd_solver(fock, two, eps=float(g["tight_eps"]), maxSteps=5000, max_diis=0, device=DEV,
                            criterion="numpy", info=info)
    assert info["engine"] == "general" and info["status"] == "converged"
    ref = float(g["tight_e"])
    assert abs(e - ref) <= 1e-10 * abs(ref), (e, ref)
    np.testing.assert_allclose(t1, g["tight_t1"], atol=1e-10)


def test_pulsed_diis_general_engine():
    d = G.load("soa_diis_he4_L3")
    g = G.load("he4_L3_t5")
    fock, two = G.hamiltonian(g)
    for steps in (4, 9, 13):
        e, t1, t2 = ccsd_solver(fock, two, eps=0.0, maxSteps=steps, max_diis=4, device=DEV, engine="general")
        assert e == pytest.approx(float(d[f"diis_e_{steps}"]), rel=1e-11)
        np.testing.assert_allclose(t1, d[f"diis_t1_{steps}"], atol=1e-11)


@pytest.mark.parametrize("spec,shapes", [
    ("bkcj,acik->abij", {"a": 40, "b": 40, "c": 40, "i": 6, "j": 6, "k": 6}),     # ring term
    ("klcd,cdij->klij", {"c": 48, "d": 48, "i": 5, "j": 5, "k": 5, "l": 5}),      # pp-ladder shape
    ("aick,bjck->abij", {"a": 33, "b": 31, "c": 29, "i": 4, "j": 4, "k": 4}),     # ragged extents
])
@pytest.mark.parametrize("beta", [0.0, 0.7])
def test_gemm_path_matches_strided_kernel(monkeypatch, spec, shapes, beta):
    """The gathered-panel library GEMM gives the strided contraction kernel's
    result (alpha, beta and permuted operand strides included)."""
    g = torch.Generator().manual_seed(5)
    ins, oz = spec.split("->")
    ta, tb = ins.split(",")
    A = torch.randn([shapes[x] for x in ta], generator=g, dtype=torch.float64).to(DEV)
    B = torch.randn([shapes[x] for x in tb], generator=g, dtype=torch.float64).to(DEV)
    B = B.transpose(0, 2).contiguous().transpose(0, 2)          # non-contiguous strides
    C0 = torch.randn([shapes[x] for x in oz], generator=g, dtype=torch.float64).to(DEV)
    outs = []
    for min_macs in (1 << 62, 1):
        monkeypatch.setattr(D, "GEMM_MIN_MACS", min_macs)
        E = D.GpuEinsum(torch.cuda.current_stream(DEV).cuda_stream)
        C = C0.clone()
        E.pair(spec, A, B, C, alpha=-0.5, beta=beta)
        outs.append((C.cpu().numpy(), E.gemms))
    (c_tile, n0), (c_gemm, n1) = outs
    assert n0 == 0 and n1 == 1
    ref = -0.5 * np.einsum(spec, A.cpu().numpy(), B.cpu().numpy()) + beta * C0.cpu().numpy()
    np.testing.assert_allclose(c_tile, ref, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(c_gemm, ref, rtol=1e-12, atol=1e-12)


# CCSD energies (MeV, two decimals) the reference's reproduction script for
# arXiv:2509.08771 table 5 prints at L=3 (examples/reproduction_arxiv_2509.08771
# /table_5_output_without_imsrg2.txt): (a_lat, vT1 = vS1, w3) -> (3He, 4He)
TABLE5 = {(2.5, -9.0, 6.0): (-15.7, -30.09), (2.0, -8.0, 5.5): (-13.23, -29.83), (1.7, -7.0, 4.4): (-6.68, -29.37)}
HE3 = [[0, 0, 0, 0, 0], [0, 0, 0, 1, 0], [0, 0, 0, 0, 1]]
HE4 = HE3 + [[0, 0, 0, 1, 1]]


@pytest.mark.parametrize("key", list(TABLE5))
def test_reproduces_reference_table5(key):
    """The reference's published L=3 CCSD energies of 3He (open-shell site:
    the general engine) and 4He (closed site: the structured engine), with
    the script's solver settings (NumPy convergence test, eps 1e-8, at most
    100 steps)."""
    from nulattice_b200 import hamiltonian as ham
    a_lat, v, w = key
    for holes, want, engine in ((HE3, TABLE5[key][0], "general"), (HE4, TABLE5[key][1], "structured")):
        e_ref, fock, two = ham.normal_ordered_hamiltonian(3, holes, v, v, w, dense=False)
        info = {}
        e, t1, t2 = ccsd_solver(fock, two, eps=1e-8, maxSteps=100, max_diis=10, device=DEV, criterion="numpy",
                                info=info, t2_format="compact" if engine == "structured" else "dense")
        assert info["engine"] == engine
        mev = (e + e_ref) * ham.phys_unit(a_lat)
        assert abs(mev - want) <= 0.005 + 1e-9, (key, holes == HE3, mev, want)


@pytest.mark.parametrize("holes", ["he4", "he3"])
def test_rotated_dense_inputs(holes):
    """A basis rotated within the particles and within the holes (as after
    Hartree-Fock): every non-zero block dense, v_pppp as a dense 4-D array
    (its ladders as library GEMMs).  The correlation energy equals the one
    of the unrotated input -- for the closed-site 4He that one comes from the
    structured engine, so the two engines check each other."""
    import rotation
    from nulattice_b200 import hamiltonian as ham
    hl = ham.closed_shell_holes(2, 4) if holes == "he4" else HE3
    e_ref, fock, two = ham.normal_ordered_hamiltonian(2, hl, -6.0, -6.0, 2.0)
    fr, tr = rotation.rotate(fock, two, 3)
    i0, i1 = {}, {}
    e0, _, _ = ccsd_solver(fock, two, eps=1e-12, maxSteps=3000, max_diis=8, device=DEV, info=i0)
    e1, _, _ = ccsd_solver(fr, tr, eps=1e-12, maxSteps=3000, max_diis=8, device=DEV, info=i1)
    assert i1["engine"] == "general"
    assert i0["engine"] == ("structured" if holes == "he4" else "general")
    assert i0["status"] == "converged" and i1["status"] == "converged"
    assert e1 == pytest.approx(e0, rel=1e-9)
