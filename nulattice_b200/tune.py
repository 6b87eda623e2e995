"""Autotuner for the launch shapes of the lattice kernels.

The lattice T2 kernel, the Lambda row pass and the Lambda column pass have
several launch shapes (threads per block x resident blocks per SM, and the
column pass's row chunks), selected by the problem's ``tune`` word
(``nlb_struct_problem.tune``).  :func:`tune` times every shape on the
problem's own buffers with CUDA events, keeps the fastest, writes the word
into the problem and caches it per GPU and problem shape in a JSON file
(``$NLB_TUNE_CACHE``, default ``~/.cache/nulattice_b200/tune.json``).
"""
from __future__ import annotations

import ctypes
import json
import os
import statistics

import numpy as np
import torch

from . import _lib
from .ccsd import _mp2_t1, ctypes_void

FWD_F32 = {0: "256x2", 1: "512x1", 2: "384x1", 3: "512x1 x2", 4: "384x1 x2", 5: "rows2 256x1", 6: "rows2 384x1",
           7: "rows2 448x1", 8: "rows2 512x1"}
FWD_F64 = {0: "512x1", 1: "256x1"}
LAM_F32 = {0: "256x2", 1: "512x1"}


def word(fwd32=0, lam32=0, chunks=0, fwd64=0):
    return (fwd32 & 15) | ((lam32 & 15) << 4) | ((chunks & 255) << 8) | ((fwd64 & 15) << 16)


def known_word(eng):
    """Launch shapes without timing: the cached word of ``eng``'s problem
    shape on this GPU if :func:`tune` stored one, else the shapes it picks
    on B200 at L=6, A=28 (two-row T2 kernel with 384 threads, Lambda column
    pass in two row chunks).  Non-lattice problems: 0 (no choices)."""
    L = _lib.lib()
    if not L.nlb_lambda_lattice(eng.prob):
        return 0
    path = _cache_path()
    if os.path.exists(path):
        try:
            cache = json.load(open(path))
            entry = cache.get(_key(eng))
            if entry is not None:
                return int(entry["word"])
        except (OSError, ValueError, KeyError, TypeError):
            pass
    chunks = 2 if max(ch.np1 for ch in eng.plan.channels) >= 8 else 0
    return word(fwd32=6, chunks=chunks)


def describe(w):
    return {"t2_fp32": FWD_F32.get(w & 15), "lambda_fp32": LAM_F32.get((w >> 4) & 15),
            "lambda_chunks": (w >> 8) & 255 or "auto", "t2_fp64": FWD_F64.get((w >> 16) & 15)}


def t2_kernel_fp32(w):
    """Template name of the FP32 lattice T2 kernel the word selects."""
    v = w & 15
    if v in (5, 6, 7, 8):
        return f"k_t2_pair<{ {5: 256, 6: 384, 7: 448, 8: 512}[v] }, 1>"
    nt, mb = {0: (256, 2), 1: (512, 1), 2: (384, 1), 3: (512, 1), 4: (384, 1)}.get(v, (256, 2))
    return f"k_t2_lat<float, 7, {nt}, {mb}, {'true' if v in (3, 4) else 'false'}>"


def _cache_path():
    return os.environ.get("NLB_TUNE_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "nulattice_b200",
                                                         "tune.json"))


def _key(eng):
    pl, prob = eng.plan, eng.prob
    name = torch.cuda.get_device_name(eng.dev)
    return f"{name}|p={pl.p}|h={pl.h}|n_t2={pl.n_t2}|nh={prob.uniform_nh}|ch={prob.n_channels}"


def _time(fn, reps):
    ts = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        torch.cuda.synchronize()
        ts.append(a.elapsed_time(b))
    return statistics.median(ts)


def tune(eng, lam=True, reps=7, use_cache=True, info=None):
    """Choose the launch shapes for engine ``eng`` and set ``eng.prob.tune``.

    Only lattice problems (seven holes per label) have choices; others keep
    the defaults.  Returns the tuning word."""
    L = _lib.lib()
    info = {} if info is None else info
    if not L.nlb_lambda_lattice(eng.prob):
        eng.prob.tune = 0
        return 0
    key = _key(eng)
    path = _cache_path()
    cache = {}
    if use_cache and os.path.exists(path):
        try:
            cache = json.load(open(path))
        except (OSError, ValueError):
            cache = {}
    if use_cache and key in cache:
        eng.prob.tune = int(cache[key]["word"])
        info.update(cache[key], cached=True)
        return eng.prob.tune
    dev = eng.dev
    sp = ctypes_void(torch.cuda.current_stream(dev).cuda_stream)
    pl = eng.plan
    t1 = torch.as_tensor(_mp2_t1(eng.f_pp_np, eng.f_ph_np, eng.f_hh_np, 0.0).reshape(-1), device=dev)
    e0 = float(np.sum(eng.f_ph_np.reshape(-1) * t1.cpu().numpy()))
    times = {}
    best = {}
    for code, variants, shift, name in ((_lib.NLB_F32, FWD_F32, 0, "t2_fp32"), (_lib.NLB_F64, FWD_F64, 16, "t2_fp64")):
        b = eng.buffers(code, 0)
        b["t1"][0].copy_(t1)
        b["t2"][0].zero_()
        _lib.check(L.nlb_struct_ctrl_init(b["ctrl"].data_ptr(), 0.0, 0.5, 1 << 30, _lib.NLB_CRIT_SOA, 0, 0, e0, sp),
                   "ctrl_init")
        for _ in range(3):   # a few real steps: realistic amplitudes
            _lib.check(L.nlb_struct_step(eng.prob, b["state"], sp), "step")
        res = {}
        for v in variants:
            eng.prob.tune = v << shift

            def run():
                _lib.check(L.nlb_struct_stage(eng.prob, b["state"], _lib.NLB_STAGE_T2, sp), "stage")
            run()
            res[v] = _time(run, reps)
        best[name] = min(res, key=res.get)
        times[name] = {variants[v]: round(res[v] * 1e3, 1) for v in res}
    lam32, chunks = 0, 0
    if lam:
        from .adjoint import LambdaSolver
        solver = LambdaSolver(eng)
        b = solver.buffers(_lib.NLB_F32, 0)
        b32 = eng.buffers(_lib.NLB_F32, 0)
        b["t1"].copy_(b32["t1"][0])
        b["t2"].copy_(b32["t2"][0])
        cands = [0] + [c for c in (2, 4, 8, 16, 32) if c * 4 <= max(ch.np1 for ch in pl.channels)]
        res = {}
        for lv in LAM_F32:
            for c in cands:
                eng.prob.tune = word(lam32=lv, chunks=c)
                _lib.check(L.nlb_lambda_init(eng.prob, b["state"], 0.0, 0.5, 1 << 30, 0, 0, sp), "lambda_init")

                def run():
                    _lib.check(L.nlb_lambda_step(eng.prob, b["state"], sp), "lambda_step")
                run()
                res[(lv, c)] = _time(run, reps)
        lam32, chunks = min(res, key=res.get)
        times["lambda_fp32"] = {f"{LAM_F32[lv]}/chunks={c or 'auto'}": round(t * 1e3, 1) for (lv, c), t in res.items()}
    w = word(fwd32=best["t2_fp32"], lam32=lam32, chunks=chunks, fwd64=best["t2_fp64"])
    eng.prob.tune = w
    entry = {"word": w, "choice": describe(w), "us": times}
    info.update(entry, cached=False)
    if use_cache:
        cache[key] = entry
        try:
            os.makedirs(os.path.dirname(path), exist_ok=True)
            json.dump(cache, open(path, "w"), indent=1)
        except OSError:
            pass
    return w

