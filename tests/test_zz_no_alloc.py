"""The no-allocation step entry point, through the C ABI.

Some callers cannot allocate device memory: an application whose memory
manager has already reserved the whole of HBM, or a latency-critical loop in
which cudaMalloc/cudaFree would synchronise the device.
``nlb_struct_step_noalloc`` serves them from a fixed array in device memory.
These tests check that it gives the same amplitudes as ``nlb_struct_step``
with caller-allocated scratch, on two calls in a row, and that a problem too
large for the array is refused.  The file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest
import torch


def _problem(L, A):
    from nulattice_b200 import hamiltonian as ham
    from nulattice_b200 import structure as S
    v2, w3 = ham.contact_couplings(-3.0, 1.0)
    e_ref, fock, two = ham.normal_ordered_hamiltonian(L, ham.closed_shell_holes(L, A), v2, v2, w3, dense=False)
    plan, why = S.detect(fock, two)
    assert plan is not None, why
    return fock, plan


def test_noalloc_rejects_oversized_problem_without_touching_the_gpu():
    from nulattice_b200 import _lib
    L = _lib.lib()
    prob = _lib.StructProblem()
    prob.p, prob.h, prob.n_labels, prob.n_channels = 2020, 28, 4, 6
    prob.n_g = 6 * 7 * 505 * 49          # L=8, A=28: Ga alone is 8.3 MB in FP64
    prob.n_f2 = 6 * 505 * 7
    state = _lib.StructState()
    state.dtype = _lib.NLB_F64
    state.ctrl = 1  # never dereferenced: the size check comes first
    need = L.nlb_struct_noalloc_scratch_bytes(ctypes.byref(prob), _lib.NLB_F64)
    assert need > (8 << 20)
    rc = L.nlb_struct_step_noalloc(ctypes.byref(prob), ctypes.byref(state), None)
    assert rc == _lib.NLB_ERR_SIZE
    assert b"static" in L.nlb_last_error()


@pytest.mark.gpu
@pytest.mark.parametrize("max_diis", [0, 2])
@pytest.mark.parametrize("dtype_name,tol", [("f64", 1e-13), ("f32", 1e-6)])
def test_noalloc_step_matches_step(dtype_name, tol, max_diis):
    """Two calls in a row against nlb_struct_step on caller-allocated
    scratch.  With max_diis = 2 the no-allocation step also fills the DIIS
    rings, and after the second call nlb_struct_diis extrapolates both
    states (it needs a prep buffer for its partial sums, which this caller
    passes for that call only)."""
    from nulattice_b200 import _lib
    from nulattice_b200.ccsd import StructuredEngine, _mp2_t1, ctypes_void
    dev = torch.device("cuda", 0)
    fock, plan = _problem(4, 28)          # seven full sites: Ga, F2 and the 7-hole kernels
    eng = StructuredEngine(plan, fock, dev)
    L = _lib.lib()
    code = _lib.NLB_F64 if dtype_name == "f64" else _lib.NLB_F32
    tdt = torch.float64 if dtype_name == "f64" else torch.float32
    ref = eng.buffers(code, max_diis)     # ordinary path: caller-allocated scratch
    n1, n2 = plan.p * plan.h, plan.n_t2
    # the no-allocation path: its own amplitudes and control block, no scratch
    t1 = [torch.zeros(n1, dtype=torch.float64, device=dev) for _ in range(2)]
    t2 = [torch.zeros(n2, dtype=tdt, device=dev) for _ in range(2)]
    ctrl = torch.zeros_like(ref["ctrl"])
    st = _lib.StructState()
    st.t1[0], st.t1[1] = t1[0].data_ptr(), t1[1].data_ptr()
    st.t2[0], st.t2[1] = t2[0].data_ptr(), t2[1].data_ptr()
    st.g = st.f2 = st.prep = st.diis_t1 = st.diis_t2 = None
    rings = []
    if max_diis:
        rings = [torch.zeros(max_diis * n1, dtype=torch.float64, device=dev),
                 torch.zeros(max_diis * n2, dtype=tdt, device=dev)]
        st.diis_t1, st.diis_t2 = rings[0].data_ptr(), rings[1].data_ptr()
    st.ctrl = ctrl.data_ptr()
    st.dtype = code

    f_pp, f_ph, f_hh = [np.asarray(f) for f in fock]
    t1_0 = torch.as_tensor(_mp2_t1(f_pp, f_ph, f_hh, 0.0).reshape(-1), device=dev)
    e0 = float((torch.as_tensor(f_ph, device=dev).reshape(-1) * t1_0).sum())
    sp = ctypes_void(torch.cuda.current_stream(dev).cuda_stream)
    crit = _lib.NLB_CRIT_SOA if max_diis else _lib.NLB_CRIT_NUMPY
    for buf_t1, buf_t2, c in ((ref["t1"], ref["t2"], ref["ctrl"]), (t1, t2, ctrl)):
        buf_t1[0].copy_(t1_0)
        buf_t2[0].zero_()
        buf_t2[1].zero_()
        _lib.check(L.nlb_struct_ctrl_init(c.data_ptr(), 0.0, 0.5, 10, crit, max_diis, 0, e0, sp), "init")
    for call in range(2):
        _lib.check(L.nlb_struct_step(eng.prob, ref["state"], sp), "step")
        _lib.check(L.nlb_struct_step_noalloc(eng.prob, st, sp), "step_noalloc")
        if max_diis and call == 1:
            prep = torch.zeros(int(L.nlb_struct_prep_len(eng.prob)), dtype=torch.float64, device=dev)
            sd = _lib.StructState.from_buffer_copy(st)
            sd.prep = prep.data_ptr()
            _lib.check(L.nlb_struct_diis(eng.prob, ref["state"], max_diis, sp), "diis")
            _lib.check(L.nlb_struct_diis(eng.prob, sd, max_diis, sp), "diis (no-allocation state)")
        torch.cuda.synchronize()
        par = (call + 1) % 2
        a1, b1 = ref["t1"][par].cpu().numpy(), t1[par].cpu().numpy()
        a2, b2 = ref["t2"][par][:n2].double().cpu().numpy(), t2[par].double().cpu().numpy()
        scale1, scale2 = max(np.abs(a1).max(), 1e-30), max(np.abs(a2).max(), 1e-30)
        assert np.abs(a1 - b1).max() <= tol * scale1, (call, np.abs(a1 - b1).max())
        assert np.abs(a2 - b2).max() <= tol * scale2, (call, np.abs(a2 - b2).max())
        assert np.abs(a2).max() > 0.0 or call == 0
    if max_diis:
        c_ref = eng.read_ctrl(ref)
        c_na = _lib.Ctrl.from_buffer_copy(ctrl.cpu().numpy().tobytes())
        assert c_ref.diis_applied == c_na.diis_applied == 1
