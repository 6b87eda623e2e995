"""Host-side logic: Hamiltonian builder, structure detection, channel algebra, C ABI."""
import ctypes

import numpy as np
import torch
import pytest

import golden_io as G
import struct_model as M
from nulattice_b200 import hamiltonian as ham
from nulattice_b200 import structure as S
from oracle import ccsd_oracle as O


def _canon(rows):
    d = {}
    for r in np.asarray(rows).reshape(-1, 5):
        k = tuple(int(x) for x in r[:4])
        d[k] = d.get(k, 0.0) + r[4]
    return {k: v for k, v in d.items() if v != 0}


@pytest.mark.parametrize("tag", ["o16_L2", "he4_L3_c1", "he4_L3_t5", "he3_L3", "li6x_L3", "he4_L4_c2", "a28_L4_tight"])
def test_builder_matches_reference(tag):
    g = G.load(tag)
    vs1 = float(g["vs1"]) if "vs1" in g else float(g["v2"])
    e, f, two = ham.normal_ordered_hamiltonian(int(g["L"]), g["holes"], float(g["v2"]), vs1, float(g["w3"]))
    fr, tr = G.hamiltonian(g)
    assert e == pytest.approx(float(g["e_ref"]), abs=1e-12)
    for a, b in zip(f, fr):
        np.testing.assert_allclose(a, b, atol=1e-13)
    for a, b in zip(two[2:], tr[2:]):
        np.testing.assert_allclose(a, b, atol=1e-13)
    assert _canon(two[0]) == pytest.approx(_canon(tr[0]))
    assert _canon(two[1]) == pytest.approx(_canon(tr[1]))


@pytest.mark.parametrize("L,A,v,w,kin", [(3, 4, -6, 2, 1.0), (4, 4, -3.3, 0.7, 1.0), (4, 28, -6, 2, 1.0),
                                         (3, 28, 1, 1, 0.0), (5, 28, -4.1, 1.3, 1.0)])
def test_builder_sparse_blocks_equal_dense(L, A, v, w, kin):
    """The sparse builder (no dense block is ever formed) gives bit for bit
    the dense builder's numbers, which the reference goldens pin."""
    e1, f1, t1 = ham.normal_ordered_hamiltonian(L, ham.closed_shell_holes(L, A), v, v, w, dense=True, kinetic=kin)
    e2, f2, t2 = ham.normal_ordered_hamiltonian(L, ham.closed_shell_holes(L, A), v, v, w, dense=False, kinetic=kin)
    assert e1 == e2
    for a, b in zip(f1, f2):
        np.testing.assert_array_equal(a, b)
    for a, b in zip(t1[:2], t2[:2]):
        np.testing.assert_array_equal(a, b)
    for a, b in zip(t1[2:], t2[2:]):
        np.testing.assert_array_equal(a, b.to_dense())
        assert np.all(b.values != 0)
        key = np.ravel_multi_index(tuple(b.indices.T), b.shape)
        assert np.all(np.diff(key) > 0)   # unique, in the dense non-zeros' order


def test_units_and_holes():
    assert ham.phys_unit(2.0) == pytest.approx(0.5 * 197.3269804 ** 2 / (938.92 * 4.0))
    assert ham.contact_couplings(-3.0, 1.0) == (-6.0, 2.0)
    h = ham.closed_shell_holes(6, 28)
    assert len(h) == 28 and len({tuple(x[:3]) for x in h}) == 7


@pytest.mark.parametrize("tag,expect", [("o16_L2", True), ("he4_L3_c1", True), ("he3_L3", False),
                                        ("li6x_L3", False)])
def test_detect(tag, expect):
    g = G.load(tag)
    fock, two = G.hamiltonian(g)
    plan, why = S.detect(fock, two)
    assert (plan is not None) == expect, why


def test_detect_rejects_structureless_random():
    r = G.load("dgrams_random")
    plan, why = S.detect([r["f_pp"], r["f_ph"], r["f_hh"]],
                         [G.rows(r, "v_pppp"), G.rows(r, "v_ppph"), r["v_pphh"], r["v_phph"], r["v_phhh"],
                          r["v_hhhh"]])
    assert plan is None and why


def test_compact_layout_roundtrip_and_size():
    g = G.load("he4_L3_c1")
    fock, two = G.hamiltonian(g)
    plan, _ = S.detect(fock, two)
    assert plan.n_t2 == 6 * 26 * 26
    t2 = plan.unpack_t2(np.random.default_rng(0).standard_normal(plan.n_t2))
    np.testing.assert_array_equal(t2, -t2.transpose(1, 0, 2, 3))
    np.testing.assert_array_equal(t2, -t2.transpose(0, 1, 3, 2))
    np.testing.assert_array_equal(plan.unpack_t2(plan.pack_t2(t2)), t2)


def test_a28_config_sizes():
    e, fock, two = ham.normal_ordered_hamiltonian(4, ham.closed_shell_holes(4, 28), -6, -6, 2, dense=False)
    plan, why = S.detect(fock, two)
    assert plan is not None, why
    assert plan.n_labels == 4 and len(plan.channels) == 6
    assert plan.n_t2 == 6 * 57 * 57 * 49


@pytest.mark.parametrize("tag", ["o16_L2", "he4_L3_c1", "he4_L3_t5"])
def test_channel_model_matches_reference_trajectory(tag):
    g = G.load(tag)
    fock, two = G.hamiltonian(g)
    plan, _ = S.detect(fock, two)
    H = O.Hamiltonian(fock, two)
    t1, B = O.t1_init(H), plan.pack_t2(O.t2_init(H))
    for _ in range(int(g["traj_steps"])):
        t1, B = M.iterate(plan, fock, t1, B, 0.5)
    np.testing.assert_allclose(t1, g["traj_t1"], atol=1e-14)
    np.testing.assert_allclose(plan.unpack_t2(B), G.dense(g, "traj_t2"), atol=1e-14)


def test_channel_model_a28_two_steps():
    g = G.load("a28_L4")
    e, fock, two = ham.normal_ordered_hamiltonian(4, g["holes"], -6.0, -6.0, 2.0, dense=False)
    plan, _ = S.detect(fock, two)
    H_f = [np.asarray(f) for f in fock]
    t1 = O.t1_init(O.Hamiltonian(fock, [two[0], two[1]] + [b.to_dense() for b in two[2:]]))
    B = np.zeros(plan.n_t2)
    for _ in range(int(g["traj_steps"])):
        t1, B = M.iterate(plan, H_f, t1, B, 0.5)
    assert float(np.sum(H_f[1] * t1)) == pytest.approx(float(g["traj_e"]), rel=1e-12)
    np.testing.assert_allclose(t1, g["traj_t1"], atol=1e-13)
    assert 2.0 * np.linalg.norm(B) == pytest.approx(float(g["traj_t2_norm"]), rel=1e-12)


def test_library_exports_declared_symbols():
    from nulattice_b200 import _lib
    L = _lib.lib()
    syms = _lib.exported_symbols()
    assert len(syms) >= 8
    for s in syms:
        assert hasattr(L, s), s
    assert L.nlb_version() >= 1
    assert ctypes.sizeof(_lib.Ctrl) == 1064
    assert ctypes.sizeof(_lib.StructProblem) == 360


def test_lambda_and_batch_struct_layouts():
    from nulattice_b200 import _lib
    assert ctypes.sizeof(_lib.LambdaState) == 120
    assert ctypes.sizeof(_lib.BatchItem) == 480
    assert ctypes.sizeof(_lib.BatchConfig) == 64


def test_batch_instances_are_seeded_and_in_range():
    from nulattice_b200 import batch as B
    a = B.draw_instances(64, 0)
    assert a == B.draw_instances(64, 0) and len(a) == 64
    assert {x[0] for x in a} <= {4, 28} and {x[1] for x in a} <= {4, 5, 6}
    assert all(-4.0 <= x[2] <= -2.0 and 0.0 <= x[3] <= 2.0 for x in a)
    # the draw order is A, L, C2, C3 per instance
    rng = np.random.default_rng(0)
    first = (int(rng.choice([4, 28])), int(rng.choice([4, 5, 6])), float(rng.uniform(-4, -2)), float(rng.uniform(0, 2)))
    assert a[0] == first


def test_batch_hamiltonian_is_the_builder_output():
    """H(C2, C3) combined from the (kinetic, contact, three-body) parts equals
    the direct build, block by block."""
    from nulattice_b200 import batch as B
    from nulattice_b200 import hamiltonian as ham
    from nulattice_b200 import structure as S
    L, A, C2, C3 = 3, 28, -3.3, 0.7
    e1, f1, t1 = B.instance_hamiltonian(L, A, C2, C3)
    v, w = ham.contact_couplings(C2, C3)
    e2, f2, t2 = ham.normal_ordered_hamiltonian(L, ham.closed_shell_holes(L, A), v, v, w, dense=False)
    assert e1 == pytest.approx(e2, rel=1e-14)
    for a, b in zip(f1, f2):
        np.testing.assert_allclose(a, b, atol=1e-13)
    for a, b in zip(t1, t2):
        ia, va = S._coo(a)
        ib, vb = S._coo(b)
        oa, ob = np.lexsort(ia.T[::-1]), np.lexsort(ib.T[::-1])
        np.testing.assert_array_equal(ia[oa], ib[ob])
        np.testing.assert_allclose(va[oa], vb[ob], atol=1e-13)


def test_batch_shards_are_disjoint_complete_and_balanced():
    from nulattice_b200 import batch as B
    inst = B.draw_instances(64, 0)
    for world in (1, 2, 4, 8):
        parts = [B.shard(inst, r, world) for r in range(world)]
        got = sorted(x for p in parts for x in p)
        assert got == sorted(inst)
        loads = [sum(B.instance_cost(a, l) for a, l, _, _ in p) for p in parts]
        biggest = max(B.instance_cost(a, l) for a, l, _, _ in inst)
        assert max(loads) - min(loads) <= biggest
    assert B.instance_cost(28, 6) == 6 * 209 * 209 * 49


def test_dense_blocks_are_row_major_whatever_the_input_strides():
    """The general engine's element-wise kernels index its blocks (and the
    residuals cloned from them) in row-major order: a block handed over with
    permuted strides, as np.einsum returns them, is stored row-major."""
    from nulattice_b200 import dense as Dn
    x = np.random.default_rng(1).standard_normal((3, 4, 2, 5))
    for y in (x.transpose(2, 0, 3, 1), np.einsum("abcd->dcba", x, optimize=True), x[:, ::2]):
        t = Dn._dense_block(y, None, "cpu")
        assert t.is_contiguous() and t.dtype.is_floating_point
        np.testing.assert_array_equal(t.numpy(), y)
        assert Dn._dense_block(torch.as_tensor(y), None, "cpu").is_contiguous()


PAIRS = [("StructProblem", "nlb_struct_problem"), ("Ctrl", "nlb_ctrl"), ("StructState", "nlb_struct_state"),
         ("LambdaState", "nlb_lambda_state"), ("BatchItem", "nlb_batch_item"), ("BatchConfig", "nlb_batch_config"),
         ("ContractDesc", "nlb_contract_desc"), ("PwProblem", "nlb_pw_problem"), ("PwState", "nlb_pw_state"),
         ("PpphPlan", "nlb_ppph_plan"), ("PpppPlan", "nlb_pppp_plan")]


def test_ctypes_mirrors_match_the_c_header(tmp_path):
    """Every ctypes mirror in _lib has the size and the field offsets that a
    C compiler gives the struct of include/nulattice_b200.h."""
    import os
    import shutil
    import subprocess
    from nulattice_b200 import _lib
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    inc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "nulattice_b200.h"', "int main(void) {"]
    want = []
    for py, c in PAIRS:
        cls = getattr(_lib, py)
        lines.append(f'printf("%zu\\n", sizeof({c}));')
        want.append((py, "sizeof", ctypes.sizeof(cls)))
        for name, _ in cls._fields_:
            lines.append(f'printf("%zu\\n", offsetof({c}, {name}));')
            want.append((py, name, getattr(cls, name).offset))
    lines += ["return 0;", "}"]
    src = tmp_path / "abi.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "abi"
    subprocess.run([cc, "-I", inc, str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    assert len(got) == len(want)
    bad = [(w, g) for w, g in zip(want, got) if w[2] != g]
    assert not bad, bad


def test_dense_work_size_matches_the_header():
    """The ctypes constant sizing the dense engine's work buffers equals the
    header's NLB_DENSE_WORK_DOUBLES."""
    import os
    import re
    from nulattice_b200 import _lib
    hdr = open(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include",
                            "nulattice_b200.h")).read()
    assert int(re.search(r"#define NLB_DENSE_WORK_DOUBLES (\d+)", hdr).group(1)) == _lib.NLB_DENSE_WORK_DOUBLES


def test_channel_model_a28_ten_unmixed_steps():
    """Ten unmixed Jacobi steps of the reference's NumPy solver at A=28, L=4
    (golden a28_L4_tight) through the CPU model of the channel kernels."""
    g = G.load("a28_L4_tight")
    e, fock, two = ham.normal_ordered_hamiltonian(4, g["holes"], -6.0, -6.0, 2.0, dense=False)
    plan, _ = S.detect(fock, two)
    H_f = [np.asarray(f) for f in fock]
    t1 = O.t1_init(O.Hamiltonian(fock, [two[0], two[1]] + [b.to_dense() for b in two[2:]]))
    B = np.zeros(plan.n_t2)
    for _ in range(10):
        t1, B = M.iterate(plan, H_f, t1, B, 0.0)
    assert float(np.sum(H_f[1] * t1)) == pytest.approx(float(g["m0_e"]), rel=1e-12)
    np.testing.assert_allclose(t1, g["m0_t1"], atol=1e-12)
    assert 2.0 * np.linalg.norm(B) == pytest.approx(float(g["m0_t2_norm"]), rel=1e-11)
