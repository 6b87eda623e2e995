"""The tensor-core contraction (tcgen05.mma kind::tf32, 3xTF32 split, FP32
accumulation in tensor memory) against FP64 references, and the general
engine's mixed-precision solve that uses it."""
import numpy as np
import pytest
import torch

import golden_io as G
from nulattice_b200 import ccsd_solver
from nulattice_b200 import dense as D

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda", 0)


def _tc_einsum():
    E = D.GpuEinsum(torch.cuda.current_stream(DEV).cuda_stream)
    E.tensor_cores = True
    return E


def _rand(shape, seed):
    g = torch.Generator().manual_seed(seed)
    return torch.randn(shape, generator=g, dtype=torch.float64).to(DEV)


# 3xTF32 keeps about 21 bits of each product and accumulates in FP32: the
# error bound is taken relative to sum_k |A_mk| |B_kn|
TOL = 1e-5


@pytest.mark.parametrize("M,N,K", [(128, 128, 32), (200, 300, 500), (1000, 64, 2000), (128, 128, 40000),
                                   (4096, 2048, 96), (33, 517, 1031)])
def test_gemm_matches_fp64(M, N, K):
    """Tile edges, split-K (few tiles, long K) and alpha/beta."""
    A, B, C0 = _rand((M, K), M + 3 * K), _rand((K, N), N + 5 * K), _rand((M, N), 7 * M + N)
    out = C0.clone()
    E = _tc_einsum()
    E.pair("mk,kn->mn", A, B, out, 0.5, 2.0)
    torch.cuda.synchronize()
    assert E.tc_gemms == 1
    ref = 0.5 * (A @ B) + 2.0 * C0
    scale = (A.abs() @ B.abs()).max()
    assert torch.isfinite(out).all()
    assert float((out - ref).abs().max() / scale) < TOL


def test_strided_ring_contraction():
    """A ring-diagram shape of ccDgrams.py (bkcj,acik->abij): multi-index
    rows and columns gathered from strided tensors."""
    p, h = 40, 4
    V, T = _rand((p, h, p, h), 11), _rand((p, p, h, h), 12)
    out = torch.zeros((p, p, h, h), dtype=torch.float64, device=DEV)
    E = _tc_einsum()
    E.pair("bkcj,acik->abij", V, T, out)
    torch.cuda.synchronize()
    assert E.tc_gemms == 1
    ref = torch.einsum("bkcj,acik->abij", V, T)
    scale = torch.einsum("bkcj,acik->abij", V.abs(), T.abs()).max()
    assert float((out - ref).abs().max() / scale) < TOL


def test_repeats_bit_for_bit():
    """Fixed tile and split order: two calls give identical results."""
    A, B = _rand((700, 3000), 21), _rand((3000, 500), 22)
    outs = []
    for _ in range(2):
        out = torch.zeros((700, 500), dtype=torch.float64, device=DEV)
        _tc_einsum().pair("mk,kn->mn", A, B, out)
        outs.append(out)
    torch.cuda.synchronize()
    assert torch.equal(outs[0], outs[1])


@pytest.mark.parametrize("tag", ["he3_L3", "li6x_L3"])
def test_mixed_general_engine_reaches_reference_fixed_point(tag):
    """Open-shell inputs (non-zero v_pphh / v_phph / v_phhh: ring and
    quadratic diagrams are real GEMMs): the tensor-core phase to 1e-8, then
    FP64 to the reference's tight fixed point within 1e-10."""
    g = G.load(tag)
    fock, two = G.hamiltonian(g)
    info = {}
    e, t1, t2 = ccsd_solver(fock, two, eps=float(g["tight_eps"]), maxSteps=5000, max_diis=8, device=DEV,
                            precision="mixed", mixed_eps=1e-8, info=info)
    ref = float(g["tight_e"])
    assert info["engine"] == "general" and info["status"] == "converged", info
    assert info["tc_gemms"] > 0 and info["mixed_iters"] > 0
    # the tensor-core phase stops on |dE|/max(1,|E|) < 1e-8; on slowly
    # converging inputs (li6x) that is some 1e-5 short of the fixed point,
    # which the FP64 phase then closes
    assert abs(info["mixed_energy"] - ref) <= 1e-4 * abs(ref)
    assert abs(e - ref) <= 1e-10 * abs(ref), (e, ref)
    np.testing.assert_allclose(np.asarray(t1), g["tight_t1"], atol=1e-9)
