"""Generate the golden vectors that pin the CCSD oracle to the reference.

Run where a checkout of the reference NuLattice tree is available, with
``NULATTICE_REF`` naming its root (the directory holding ``src/NuLattice``):

    NULATTICE_REF=<reference root> python tests/golden/make_goldens.py [case ...]

Everything here calls the reference's own code (``CCM/coupled_cluster.py``,
``CCM/ccDgrams.py``, ``CCM/soa/coupled_cluster.py``, ``lattice.py``) and
stores its inputs and outputs as compressed ``.npz`` fixtures next to this
script.  The tests read only the fixtures, so they also run where the
reference is absent.  ``opt_einsum`` is not installed here; the stand-in in
``_standin/`` maps ``contract`` onto ``numpy.einsum`` (same sums, FP64
summation order may differ in the last bits).
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("NULATTICE_REF")
if not REF or not os.path.isdir(os.path.join(REF, "src", "NuLattice")):
    sys.exit("set NULATTICE_REF to the root of a NuLattice checkout (the directory holding src/NuLattice)")
sys.path.insert(0, os.path.join(HERE, "_standin"))
sys.path.insert(0, os.path.join(REF, "src"))

import NuLattice.lattice as lat  # noqa: E402
import NuLattice.references as refs  # noqa: E402
import NuLattice.CCM.coupled_cluster as ccm  # noqa: E402
import NuLattice.CCM.ccDgrams as dg  # noqa: E402


def coo(arr):
    arr = np.asarray(arr)
    idx = np.argwhere(arr != 0).astype(np.int32)
    return idx, arr[tuple(idx.T)] if len(idx) else np.zeros(0)


def put_block(out, name, arr):
    idx, val = coo(arr)
    out[name + "_shape"] = np.array(np.shape(arr), dtype=np.int64)
    out[name + "_idx"] = idx
    out[name + "_val"] = val


def put_list(out, name, lst):
    a = np.array(lst, dtype=np.float64).reshape(-1, 5)
    out[name + "_idx"] = a[:, :4].astype(np.int32)
    out[name + "_val"] = a[:, 4].copy()


# ---------------------------------------------------------------------------
# per-diagram goldens on random tensors (mirrors tests/CCM/test_t1iter_dgrams.py)
# ---------------------------------------------------------------------------
DGRAMS = [
    ("dgram_akci_ck", ("v_phph", "t1")),
    ("dgram_ck_acik", ("f_ph", "t2")),
    ("dgram_cikl_cakl", ("v_phhh", "t2")),
    ("dgram_cdkl_ck_dali", ("v_pphh", "t1", "t2")),
    ("dgram_ck_ci", ("f_ph", "t1")),
    ("dgram_ck_ak", ("f_ph", "t1")),
    ("dgram_bijk_bj", ("v_phhh", "t1")),
    ("dgram_cdlk_cdli", ("v_pphh", "t2")),
    ("dgram_dckl_dakl", ("v_pphh", "t2")),
    ("dgram_cdlk_cl_di", ("v_pphh", "t1")),
    ("dgram_cdkl_dk_al", ("v_pphh", "t1")),
    ("dgram_klij_abkl", ("v_hhhh", "t2")),
    ("dgram_bkcj_acik", ("v_phph", "t2")),
    ("dgram_bkij_ak", ("v_phhh", "t1")),
    ("dgram_cdkl_acik_dblj", ("v_pphh", "t2")),
    ("dgram_cdkl_cdij_abkl", ("v_pphh", "t2")),
    ("dgram_klij_ak_bl", ("v_hhhh", "t1")),
    ("dgram_bkci_ak_cj", ("v_phph", "t1")),
    ("dgram_cikl_ck_ablj", ("v_phhh", "t1", "t2")),
    ("dgram_da_dbij", ("x_pp", "t2")),
    ("dgram_acik_bcjk", ("x_pphh", "t2")),
    ("dgram_cikl_al_bcjk", ("v_phhh", "t1", "t2")),
    ("dgram_cjkl_ci_abkl", ("v_phhh", "t1", "t2")),
    ("dgram_bijk_ak1", ("x_phhh", "t1")),
    ("dgram_bijk_ak2", ("x_phhh", "t1")),
    ("dgram_cjkl_ci_ak_bl", ("v_phhh", "t1")),
    ("dgram_cdkl_ci_dj_abkl", ("v_pphh", "t1", "t2")),
    ("dgram_cdkl_ak_bl_cdij", ("v_pphh", "t1", "t2")),
    ("dgram_cdkl_ci_bl_adkj", ("v_pphh", "t1", "t2")),
    ("dgram_cdkl_ci_ak_dj_bl", ("v_pphh", "t1")),
    ("dgram_cdkl_bdkl", ("v_pphh", "t2")),
    ("dgram_cdkl_cdjl", ("v_pphh", "t2")),
    ("dgram_ck_bk", ("f_ph", "t1")),
    ("dgram_ck_cj", ("f_ph", "t1")),
    ("dgram_cdlk_cl_dj", ("v_pphh", "t1")),
    ("dgram_cdlk_dk_bl", ("v_pphh", "t1")),
    ("pAB", ("t2",)),
    ("pIJ", ("t2",)),
]


def random_sparse_list(rng, p, n, last):
    """Random [a,b,c,d,val] list with some repeated keys (they must be summed)."""
    rows = []
    for _ in range(n):
        a, b, c = rng.integers(0, p, size=3)
        d = rng.integers(0, last)
        rows.append([int(a), int(b), int(c), int(d), float(rng.standard_normal())])
    rows += [list(r[:4]) + [0.5] for r in rows[:3]]  # duplicates of the first keys
    return rows


def case_dgrams():
    p, h = 6, 4
    np.random.seed(42)
    d = {
        "t1": np.random.randn(p, h),
        "t2": np.random.randn(p, p, h, h),
        "f_ph": np.random.randn(p, h),
        "f_pp": np.random.randn(p, p),
        "f_hh": np.random.randn(h, h),
        "v_phph": np.random.randn(p, h, p, h),
        "v_phhh": np.random.randn(p, h, h, h),
        "v_pphh": np.random.randn(p, p, h, h),
        "v_hhhh": np.random.randn(h, h, h, h),
        "x_pp": np.random.randn(p, p),
        "x_pphh": np.random.randn(p, p, h, h),
        "x_phhh": np.random.randn(p, h, h, h),
    }
    out = {k: v for k, v in d.items()}
    for name, args in DGRAMS:
        out["out_" + name] = getattr(dg, name)(*[d[a] for a in args])
    rng = np.random.default_rng(7)
    v_pppp = random_sparse_list(rng, p, 40, p)
    v_ppph = random_sparse_list(rng, p, 40, h)
    put_list(out, "v_pppp", v_pppp)
    put_list(out, "v_ppph", v_ppph)
    r_ppph = dg.v_ppph_dgrams(v_ppph, d["t1"], d["t2"])
    for n, r in enumerate(r_ppph):
        out[f"out_v_ppph_dgrams_{n}"] = r
    r_pppp = dg.v_pppp_dgrams(v_pppp, d["t1"], d["t2"])
    out["out_v_pppp_dgrams_0"], out["out_v_pppp_dgrams_1"] = r_pppp
    # full t1Iter / t2Iter with every block populated (sparse lists)
    out["out_t1Iter"] = ccm.t1Iter(d["t1"], d["t2"], d["f_ph"], d["f_pp"], d["f_hh"],
                                   d["v_phph"], d["v_phhh"], d["v_pphh"], r_ppph, sparse=True)
    out["out_t2Iter"] = ccm.t2Iter(d["t1"], d["t2"], d["f_ph"], d["f_hh"], d["f_pp"],
                                   v_pppp, d["v_phph"], d["v_phhh"], d["v_pphh"], r_ppph,
                                   d["v_hhhh"], sparse=True)
    out["out_energy"] = np.array(ccm.ccsd_energy(d["f_ph"], d["v_pphh"], d["t2"], d["t1"]))
    np.savez_compressed(os.path.join(HERE, "dgrams_random.npz"), **out)


# ---------------------------------------------------------------------------
# physical lattice systems through the reference's own builders + solver
# ---------------------------------------------------------------------------
SEVEN = [(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)]


def holes_for(name, L):
    if name == "he4":
        return refs.ref_4He_gs
    if name == "he3":
        return refs.ref_3He_gs
    if name == "o16":
        return refs.ref_16O_gs
    if name == "a28":
        return [[x % L, y % L, z % L, t, s] for (x, y, z) in SEVEN for t in (0, 1) for s in (0, 1)]
    if name == "li6x":
        # a full site plus a half-filled site whose two holes (tz,sz)=(0,0),(1,1)
        # share total Tz and Sz with its two particle states: with vT1 != vS1
        # this populates v_pphh, v_phph and v_phhh
        return [[0, 0, 0, t, s] for t in (0, 1) for s in (0, 1)] + \
               [[1, 0, 0, 0, 0], [1, 0, 0, 1, 1]]
    raise KeyError(name)


class Counter:
    def __init__(self):
        self.n = 0
        self._orig = ccm.t2Iter

    def __enter__(self):
        def wrapped(*a, **k):
            self.n += 1
            return self._orig(*a, **k)
        ccm.t2Iter = wrapped
        return self

    def __exit__(self, *exc):
        ccm.t2Iter = self._orig


def build(L, name, v2, w3, vs1=None):
    lattice = lat.get_lattice(L)
    holes = holes_for(name, L)
    vs1 = v2 if vs1 is None else vs1
    res = ccm.get_norm_ordered_ham(L, holes, lat.Tkin(lattice, L), lat.contacts(v2, vs1, lattice, L),
                                   lat.NNNcontact(w3, lattice, L), sparse=True, NO2B=True)
    e_ref, fock, two = res
    # input-side cast of the 3NF NO2B list entries (they arrive as floats)
    two[0] = [[int(a), int(b), int(c), int(d), v] for a, b, c, d, v in two[0]]
    two[1] = [[int(a), int(b), int(c), int(d), v] for a, b, c, d, v in two[1]]
    return holes, e_ref, fock, two


def jacobi_gap(fock, two, t1, t2):
    """Size of one unmixed reference Jacobi step at (t1, t2): 0 at the fixed point."""
    f_pp, f_ph, f_hh = fock
    v_pppp, v_ppph, v_pphh, v_phph, v_phhh, v_hhhh = two
    r = dg.v_ppph_dgrams(v_ppph, t1, t2)
    n1 = ccm.t1Iter(t1, t2, f_ph, f_pp, f_hh, v_phph, v_phhh, v_pphh, r, sparse=True)
    n2 = ccm.t2Iter(t1, t2, f_ph, f_hh, f_pp, v_pppp, v_phph, v_phhh, v_pphh, r, v_hhhh, sparse=True)
    return float(np.linalg.norm(n1 - t1)), float(np.linalg.norm(n2 - t2))


def case_system(tag, L, name, v2, w3, tight=True, store_t2=True, traj_steps=3, eps=1e-14, vs1=None):
    t0 = time.perf_counter()
    holes, e_ref, fock, two = build(L, name, v2, w3, vs1)
    f_pp, f_ph, f_hh = fock
    out = {"L": np.array(L), "v2": np.array(v2), "w3": np.array(w3),
           "vs1": np.array(v2 if vs1 is None else vs1),
           "holes": np.array(holes, dtype=np.int64), "e_ref": np.array(float(e_ref))}
    out["f_pp"], out["f_ph"], out["f_hh"] = f_pp, f_ph, f_hh
    put_list(out, "v_pppp", two[0])
    put_list(out, "v_ppph", two[1])
    for nm, arr in zip(("v_pphh", "v_phph", "v_phhh", "v_hhhh"), two[2:]):
        put_block(out, nm, arr)
    print(f"[{tag}] setup {time.perf_counter() - t0:.1f}s p={f_ph.shape[0]} h={f_ph.shape[1]}", flush=True)

    # short trajectory from the MP2 start: default mixing, no DIIS
    e, t1, t2 = ccm.ccsd_solver(fock, two, eps=0.0, maxSteps=traj_steps, max_diis=0, mixing=0.5, sparse=True)
    out["traj_steps"] = np.array(traj_steps)
    out["traj_e"] = np.array(float(e))
    out["traj_t1"] = t1
    if store_t2:
        put_block(out, "traj_t2", t2)
    out["traj_t2_norm"] = np.array(float(np.linalg.norm(t2)))
    out["traj_t2_sum_abs"] = np.array(float(np.abs(t2).sum()))
    print(f"[{tag}] trajectory {time.perf_counter() - t0:.1f}s", flush=True)

    # unmixed ten steps (reference test_ccsd.py::test_debug_solver_path_consistency settings)
    if tight:
        e10, t1_10, t2_10 = ccm.ccsd_solver(fock, two, eps=0.0, maxSteps=10, max_diis=0, mixing=0.0,
                                            sparse=True)
        out["m0_e"] = np.array(float(e10))
        out["m0_t1"] = t1_10
        out["m0_t2_norm"] = np.array(float(np.linalg.norm(t2_10)))

    if tight:
        with Counter() as c:
            e, t1, t2 = ccm.ccsd_solver(fock, two, eps=eps, maxSteps=5000, max_diis=0, mixing=0.5,
                                        sparse=True)
        g1, g2 = jacobi_gap(fock, two, t1, t2)
        out["tight_e"] = np.array(float(e))
        out["tight_iters"] = np.array(c.n)
        out["tight_eps"] = np.array(eps)
        out["tight_t1"] = t1
        if store_t2:
            put_block(out, "tight_t2", t2)
        out["tight_t2_norm"] = np.array(float(np.linalg.norm(t2)))
        out["tight_gap"] = np.array([g1, g2])
        print(f"[{tag}] tight E_corr={e!r} iters={c.n} gap={g1:.2e},{g2:.2e} "
              f"total {time.perf_counter() - t0:.1f}s", flush=True)
    np.savez_compressed(os.path.join(HERE, f"{tag}.npz"), **out)


def case_soa_diis():
    """Pulsed DIIS of the torch solver (CCM/soa/coupled_cluster.py:479-567)."""
    import torch
    import NuLattice.CCM.soa.coupled_cluster as soa
    from NuLattice._torch_types import TwoBodyOperator
    # torch would route einsum path planning through the stand-in; keep its own
    torch.backends.opt_einsum.enabled = False
    holes, e_ref, fock, two = build(3, "he4", -8.0, 5.5)
    nstat = 4 * 27
    # the torch solver takes the sparse blocks as TwoBodyOperator objects
    two = [TwoBodyOperator.from_list(two[0], nstat, use_torch=True, device="cpu"),
           TwoBodyOperator.from_list(two[1], nstat, use_torch=True, device="cpu")] + list(two[2:])
    out = {}
    for steps in (4, 9, 13):
        e, t1, t2 = soa.ccsd_solver([np.array(f) for f in fock], two, eps=0.0, maxSteps=steps,
                                    max_diis=4, mixing=0.5, sparse=True)
        out[f"diis_e_{steps}"] = np.array(float(e))
        out[f"diis_t1_{steps}"] = t1.numpy()
        out[f"diis_t2norm_{steps}"] = np.array(float(t2.norm()))
    e, t1, t2 = soa.ccsd_solver([np.array(f) for f in fock], two, eps=1e-10, maxSteps=400,
                                max_diis=8, mixing=0.5, sparse=True)
    out["diis_conv_e"] = np.array(float(e))
    np.savez_compressed(os.path.join(HERE, "soa_diis_he4_L3.npz"), **out)
    print("[soa_diis] done", {k: float(v) for k, v in out.items() if v.ndim == 0}, flush=True)


CASES = {
    "dgrams": case_dgrams,
    "o16_L2": lambda: case_system("o16_L2", 2, "o16", -9.0, 6.0),
    "he4_L3_c1": lambda: case_system("he4_L3_c1", 3, "he4", -6.0, 2.0),
    "he4_L3_t5": lambda: case_system("he4_L3_t5", 3, "he4", -8.0, 5.5),
    "he3_L3": lambda: case_system("he3_L3", 3, "he3", -8.0, 5.5),
    "li6x_L3": lambda: case_system("li6x_L3", 3, "li6x", -6.0, 2.0, vs1=-4.0),
    "he4_L4_c2": lambda: case_system("he4_L4_c2", 4, "he4", -6.0, 2.0, store_t2=False),
    "a28_L4": lambda: case_system("a28_L4", 4, "a28", -6.0, 2.0, tight=False, store_t2=False,
                                  traj_steps=2),
    "he4_L5_c3": lambda: case_system("he4_L5_c3", 5, "he4", -6.0, 2.0, store_t2=False, eps=1e-13),
    "a28_L4_tight": lambda: case_system("a28_L4_tight", 4, "a28", -6.0, 2.0, store_t2=False,
                                        traj_steps=1, eps=1e-13),
    "soa_diis": case_soa_diis,
}

if __name__ == "__main__":
    todo = sys.argv[1:] or list(CASES)
    for c in todo:
        CASES[c]()
