"""ctypes binding of the C ABI declared in ``include/nulattice_b200.h``.

The shared library is built in-tree (``nulattice_b200/_nlb_ccsd.so``) by
``nulattice_b200.build``.  There is no fallback: if the library is missing or
fails to load, every solver entry point raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_nlb_ccsd.so")

NLB_OK, NLB_ERR_ARG, NLB_ERR_LAUNCH, NLB_ERR_SIZE, NLB_ERR_CUDA = 0, 1, 2, 3, 4
NLB_F64, NLB_F32 = 0, 1
NLB_RUNNING, NLB_CONVERGED, NLB_MAX_ITER, NLB_DIVERGED = 0, 1, 2, 3
NLB_CRIT_SOA, NLB_CRIT_NUMPY = 0, 1
NLB_STAGE_PREP, NLB_STAGE_GTERMS, NLB_STAGE_T2, NLB_STAGE_T1, NLB_STAGE_FINISH = 0, 1, 2, 3, 4
MAX_DIIS = 10

c_int32, c_int64, c_double, c_void_p = ctypes.c_int32, ctypes.c_int64, ctypes.c_double, ctypes.c_void_p

# numpy mirror of nlb_channel (device array of channel descriptors)
CHANNEL_DTYPE = np.dtype([(n, np.int32) for n in ("g1", "g2", "np1", "np2", "nh1", "nh2",
                                                  "pb1", "pb2", "hb1", "hb2")] +
                         [(n, np.int64) for n in ("offset", "ga_off", "f2_off", "hh_ptr_off",
                                                  "hh_col_off", "pp_ptr_off", "pp_col_off")])
assert CHANNEL_DTYPE.itemsize == 96


class StructProblem(ctypes.Structure):
    _fields_ = [("p", c_int32), ("h", c_int32), ("n_labels", c_int32), ("n_channels", c_int32)] + \
               [(n, c_int64) for n in ("n_t2", "n_g", "n_f2", "n_rows", "n_t1c", "n_xc")] + \
               [("max_row", c_int32), ("max_nh", c_int32), ("uniform_nh", c_int32), ("diag_ladders", c_int32),
                ("max_fpp_offdiag", c_int32), ("tune", c_int32)] + [
        (n, c_void_p) for n in ("chan", "t2_end", "g_end", "row_end", "t1c_base", "xc_base",
                                "p_ord", "h_ord", "p_label", "h_label",
                                "p_loc", "h_loc", "p_base", "h_base", "fpp_ptr", "fpp_col", "fpp_val",
                                "fpp_diag", "fph_ptr", "fph_col", "fph_val", "f_ph", "f_hh",
                                "hh_ptr", "hh_col", "hh_val", "pp_ptr", "pp_col", "pp_val",
                                "h_row", "fph_prow", "fpp_prow", "t1c_idx", "xc_ki")]


class Ctrl(ctypes.Structure):
    _fields_ = [(n, c_double) for n in ("e_acc", "dt1_sq", "dt2_sq", "e_prev", "e_last", "eps", "mixing")] + \
               [("gram", c_double * 121)] + \
               [(n, c_int32) for n in ("parity", "iter", "status", "max_steps", "criterion", "max_diis",
                                       "diis_count", "diis_pulse", "diis_applied", "ccs")]


class StructState(ctypes.Structure):
    _fields_ = [("t1", c_void_p * 2), ("t2", c_void_p * 2), ("g", c_void_p), ("f2", c_void_p),
                ("prep", c_void_p),
                ("diis_t1", c_void_p), ("diis_t2", c_void_p), ("ctrl", c_void_p), ("dtype", c_int32)]


class LambdaState(ctypes.Structure):
    _fields_ = [("lam1", c_void_p * 2), ("lam2", c_void_p * 2)] + [
        (n, c_void_p) for n in ("t1", "t2", "prep", "ga", "ha", "acc", "ctrl", "gb", "diis_t1", "diis_t2")] + [
        ("dtype", c_int32), ("reserved", c_int32)]


NLB_LAMBDA_KEEP = 1


class BatchItem(ctypes.Structure):
    _fields_ = [("prob", ctypes.POINTER(StructProblem)), ("f32", StructState), ("f64", StructState),
                ("l32", LambdaState), ("l64", LambdaState), ("t1_init", c_void_p), ("e0", c_double),
                ("dw", c_void_p * 2), ("dv", c_void_p * 2), ("out", c_void_p)]


class BatchConfig(ctypes.Structure):
    _fields_ = [(n, c_double) for n in ("mixing", "mixed_eps", "eps", "lambda_tol_fp32", "lambda_tol")] + [
        (n, c_int32) for n in ("max_steps", "max_diis", "lambda_max_steps", "chunk", "phases", "criterion")]


NLB_PHASE_FWD32, NLB_PHASE_FWD64, NLB_PHASE_LAMBDA = 1, 2, 4


class ContractDesc(ctypes.Structure):
    _fields_ = [(n, c_int32) for n in ("nm", "nn", "nk", "nb")] + \
               [(n, c_int64) for n in ("M", "N", "K", "B")] + \
               [(n, c_int64 * 4) for n in ("ext_m", "ext_n", "ext_k", "ext_b", "sa_m", "sc_m", "sb_n", "sc_n",
                                           "sa_k", "sb_k", "sa_b", "sb_b", "sc_b")]


class PpphPlan(ctypes.Structure):
    _fields_ = [("nnz", c_int64), ("idx", c_void_p), ("val", c_void_p),
                ("perm_adk", c_void_p), ("perm_ak", c_void_p), ("perm_cdk", c_void_p)] + \
               [(n, c_int64) for n in ("n_a", "n_ad", "n_adk", "n_ak", "n_cdk")] + \
               [(n, c_void_p) for n in ("seg_a", "seg_ad", "seg_adk", "seg_ak", "seg_cdk")]


class PpppPlan(ctypes.Structure):
    _fields_ = [("nnz", c_int64), ("idx", c_void_p), ("val", c_void_p), ("perm_ab", c_void_p),
                ("n_ab", c_int64), ("seg_ab", c_void_p)]


NLB_DENSE_WORK_DOUBLES = 57344


class PwProblem(ctypes.Structure):
    _fields_ = [("L", c_int32), ("n_blocks", c_int32), ("n_pmom", c_int32), ("n_hmom", c_int32),
                ("n_t2", c_int64), ("n_m", c_int64), ("n_w", c_int64), ("n_rows", c_int64),
                ("n_tiles", c_int32), ("pad0", c_int32)] + \
               [(n, c_void_p) for n in ("blk_off", "m_off", "w_off", "row_off", "blk_nr", "blk_nc", "blk_K",
                                        "blk_pm0", "blk_hm0", "pm_list", "hm_list", "ppos", "hpos", "kblk",
                                        "pmom", "hmom", "pinv", "hinv", "tiles", "V", "fpp", "fhh")]


class PwState(ctypes.Structure):
    _fields_ = [(n, c_void_p) for n in ("M", "W", "Y", "Xpp", "Xhh", "R", "U", "G", "H", "energy")]


_lib = None
_load_error = None


def lib():
    """The loaded library; raises RuntimeError when it is unavailable."""
    global _lib, _load_error
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"nulattice_b200 CUDA library not built ({LIB_PATH} missing); "
                           "run nulattice_b200.build.build()")
    try:
        L = ctypes.CDLL(LIB_PATH)
    except OSError as e:  # pragma: no cover - depends on the machine
        _load_error = str(e)
        raise RuntimeError(f"cannot load {LIB_PATH}: {e}") from e
    L.nlb_version.restype = c_int32
    L.nlb_last_error.restype = ctypes.c_char_p
    L.nlb_struct_prep_len.restype = c_int64
    L.nlb_struct_prep_len.argtypes = [ctypes.POINTER(StructProblem)]
    L.nlb_struct_smem_bytes.restype = c_int64
    L.nlb_struct_smem_bytes.argtypes = [ctypes.POINTER(StructProblem), c_int32]
    L.nlb_struct_ctrl_init.argtypes = [c_void_p, c_double, c_double, c_int32, c_int32, c_int32, c_int32,
                                       c_double, c_void_p]
    L.nlb_struct_step.argtypes = [ctypes.POINTER(StructProblem), ctypes.POINTER(StructState), c_void_p]
    L.nlb_struct_diis.argtypes = [ctypes.POINTER(StructProblem), ctypes.POINTER(StructState), c_int32,
                                  c_void_p]
    L.nlb_struct_stage.argtypes = [ctypes.POINTER(StructProblem), ctypes.POINTER(StructState), c_int32,
                                   c_void_p]
    L.nlb_struct_stage.restype = c_int32
    L.nlb_struct_energy.argtypes = [ctypes.POINTER(StructProblem), ctypes.POINTER(StructState), c_void_p,
                                    c_void_p]
    L.nlb_convert.argtypes = [c_void_p, c_int32, c_void_p, c_int32, c_int64, c_void_p]
    L.nlb_struct_unpack_t2.argtypes = [ctypes.POINTER(StructProblem), c_void_p, c_int32, c_void_p, c_void_p]
    L.nlb_struct_pack_t2.argtypes = [ctypes.POINTER(StructProblem), c_void_p, c_void_p, c_int32, c_void_p]
    L.nlb_struct_step_noalloc.argtypes = [ctypes.POINTER(StructProblem), ctypes.POINTER(StructState), c_void_p]
    L.nlb_struct_step_noalloc.restype = c_int32
    L.nlb_struct_noalloc_scratch_bytes.argtypes = [ctypes.POINTER(StructProblem), c_int32]
    L.nlb_struct_noalloc_scratch_bytes.restype = c_int64
    for name in ("nlb_struct_ctrl_init", "nlb_struct_step", "nlb_struct_diis", "nlb_struct_energy",
                 "nlb_convert", "nlb_struct_unpack_t2", "nlb_struct_pack_t2"):
        getattr(L, name).restype = c_int32
    L.nlb_contract_f64.argtypes = [ctypes.POINTER(ContractDesc), c_void_p, c_void_p, c_void_p, c_double, c_double,
                                   c_void_p]
    L.nlb_contract_gemm_work.argtypes = [ctypes.POINTER(ContractDesc)]
    L.nlb_contract_gemm_work.restype = c_int64
    L.nlb_contract_gemm_f64.argtypes = [ctypes.POINTER(ContractDesc), c_void_p, c_void_p, c_void_p, c_double,
                                        c_double, c_void_p, c_int64, c_void_p]
    L.nlb_contract_gemm_tc_work.argtypes = [ctypes.POINTER(ContractDesc)]
    L.nlb_contract_gemm_tc_work.restype = c_int64
    L.nlb_contract_gemm_tf32x3.argtypes = [ctypes.POINTER(ContractDesc), c_void_p, c_void_p, c_void_p, c_double,
                                           c_double, c_void_p, c_int64, c_void_p]
    L.nlb_contract_gemm_tf32x3.restype = c_int32
    L.nlb_antisym_acc_f64.argtypes = [c_void_p, c_void_p, c_int64, c_int64, c_int32, c_double, c_void_p]
    L.nlb_ppph_intermediates_f64.argtypes = [ctypes.POINTER(PpphPlan), c_void_p, c_void_p, c_int64, c_int64,
                                             c_void_p, c_void_p]
    L.nlb_pppp_ladders_f64.argtypes = [ctypes.POINTER(PpppPlan), c_void_p, c_void_p, c_int64, c_int64,
                                       c_void_p, c_void_p, c_void_p]
    L.nlb_jacobi_f64.argtypes = [c_void_p] * 8 + [c_int64, c_int64, c_double] + [c_void_p] * 5
    L.nlb_dense_energy_f64.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, c_int64, c_int64, c_void_p,
                                       c_void_p, c_void_p]
    L.nlb_lambda_acc_len.argtypes = [ctypes.POINTER(StructProblem)]
    L.nlb_lambda_acc_len.restype = c_int64
    L.nlb_lambda_ha_len.argtypes = [ctypes.POINTER(StructProblem)]
    L.nlb_lambda_ha_len.restype = c_int64
    L.nlb_lambda_gb_len.argtypes = [ctypes.POINTER(StructProblem)]
    L.nlb_lambda_gb_len.restype = c_int64
    L.nlb_lambda_lattice.argtypes = [ctypes.POINTER(StructProblem)]
    L.nlb_lambda_lattice.restype = c_int32
    L.nlb_lambda_init.argtypes = [ctypes.POINTER(StructProblem), ctypes.POINTER(LambdaState), c_double, c_double,
                                  c_int32, c_int32, c_int32, c_void_p]
    L.nlb_lambda_step.argtypes = [ctypes.POINTER(StructProblem), ctypes.POINTER(LambdaState), c_void_p]
    L.nlb_lambda_diis.argtypes = [ctypes.POINTER(StructProblem), ctypes.POINTER(LambdaState), c_int32, c_void_p]
    L.nlb_lambda_coupling.argtypes = [ctypes.POINTER(StructProblem), ctypes.POINTER(LambdaState), c_void_p,
                                      c_void_p, c_void_p, c_void_p]
    L.nlb_batch_create.argtypes = [ctypes.POINTER(BatchItem), c_int32, ctypes.POINTER(BatchConfig),
                                   ctypes.POINTER(c_void_p)]
    L.nlb_batch_launch.argtypes = [c_void_p, c_void_p]
    L.nlb_batch_destroy.argtypes = [c_void_p]
    for name in ("nlb_batch_create", "nlb_batch_launch", "nlb_batch_destroy"):
        getattr(L, name).restype = c_int32
    for name in ("nlb_lambda_init", "nlb_lambda_step", "nlb_lambda_diis", "nlb_lambda_coupling"):
        getattr(L, name).restype = c_int32
    L.nlb_antisym_project_f64.argtypes = [c_void_p, c_int64, c_int64, c_void_p]
    L.nlb_antisym_project_f64.restype = c_int32
    L.nlb_vec_diis_f64.argtypes = [c_void_p, c_void_p, c_int64, c_int32, c_void_p, c_void_p, c_void_p]
    L.nlb_vec_diis_f32.argtypes = [c_void_p, c_void_p, c_int64, c_int32, c_void_p, c_void_p, c_void_p]
    for name in ("nlb_contract_f64", "nlb_antisym_acc_f64", "nlb_ppph_intermediates_f64", "nlb_pppp_ladders_f64",
                 "nlb_jacobi_f64", "nlb_dense_energy_f64", "nlb_vec_diis_f64", "nlb_vec_diis_f32"):
        getattr(L, name).restype = c_int32
    L.nlb_pw_init.argtypes = [ctypes.POINTER(PwProblem), c_void_p, c_double, c_void_p]
    L.nlb_pw_energy.argtypes = [ctypes.POINTER(PwProblem), c_void_p, ctypes.POINTER(PwState), c_void_p]
    L.nlb_pw_step.argtypes = [ctypes.POINTER(PwProblem), c_void_p, c_void_p, c_void_p, c_double,
                              ctypes.POINTER(PwState), c_void_p]
    L.nlb_pw_energy_f32.argtypes = [ctypes.POINTER(PwProblem), c_void_p, ctypes.POINTER(PwState), c_void_p]
    L.nlb_pw_step_f32.argtypes = [ctypes.POINTER(PwProblem), c_void_p, c_void_p, c_void_p, c_double,
                                  ctypes.POINTER(PwState), c_void_p]
    for name in ("nlb_pw_init", "nlb_pw_energy", "nlb_pw_step", "nlb_pw_energy_f32", "nlb_pw_step_f32"):
        getattr(L, name).restype = c_int32
    _lib = L
    return L


def check(rc, what=""):
    if rc != NLB_OK:
        msg = lib().nlb_last_error().decode(errors="replace")
        raise RuntimeError(f"nulattice_b200 {what} failed (code {rc}): {msg}")


def exported_symbols():
    """Names declared in include/nulattice_b200.h (checked by the tests)."""
    hdr = os.path.join(os.path.dirname(HERE), "include", "nulattice_b200.h")
    import re
    txt = open(hdr).read()
    return sorted(set(re.findall(r"\b(nlb_[a-z0-9_]+)\s*\(", txt)))
