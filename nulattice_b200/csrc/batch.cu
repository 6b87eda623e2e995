// Batched scan: many structured CCSD problems (uneven sizes) solved together,
// with their coupling derivatives, in ONE CUDA graph launch.
//
// The graph runs four device-side loops (conditional WHILE nodes): the
// forward solve in FP32, its FP64 finish, the Lambda equations in FP32 and
// their FP64 finish.  Each loop body holds one branch per instance (a chunk of
// steps of that instance, DIIS pulses included) and ends in a kernel that
// keeps the loop going while any instance is still running; an instance that
// has converged (or failed) keeps riding along, its kernels returning at once.
// Between the loops, handoff kernels move each instance's converged
// amplitudes (current parity, read on the device) into the next phase's
// buffers, so nothing returns to the host until the end.  The kernels are the
// single-instance ones of ccsd_struct.cu and lambda.cu, launched per instance.

#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include <vector>

#include "nulattice_b200.h"

void nlb_internal_set_error(const char* msg);

namespace {

int bfail(int code, const char* msg) {
    nlb_internal_set_error(msg);
    return code;
}

int bcuda(cudaError_t e, const char* where) {
    if (e == cudaSuccess) return NLB_OK;
    char buf[512];
    snprintf(buf, sizeof(buf), "%s: %s", where, cudaGetErrorString(e));
    nlb_internal_set_error(buf);
    return NLB_ERR_CUDA;
}

constexpr int kT = 256;

int grid_for(int64_t n) {
    int64_t g = (n + kT - 1) / kT;
    if (g > 148 * 8) g = 148 * 8;
    return (int)(g < 1 ? 1 : g);
}

// Loop condition: go on while any instance of the phase is running, at most
// `cap` iterations of the body; each instance's branch in the body is an IF
// node that runs only while that instance is running.
__global__ void k_batch_cond(cudaGraphConditionalHandle h, const cudaGraphConditionalHandle* inst,
                             nlb_ctrl* const* ctrls, int n, int* counter, int cap) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int any = 0;
    for (int i = 0; i < n; ++i) {
        const int run = ctrls[i]->status == NLB_RUNNING;
        any |= run;
        cudaGraphSetConditional(inst[i], run ? 1u : 0u);
    }
    const int it = ++(*counter);
    cudaGraphSetConditional(h, (any && it < cap) ? 1u : 0u);
}

// Forward FP32 -> FP64: the converged FP32 amplitudes (current parity) become
// buffer 0 of the FP64 phase, whose control block starts from the FP32
// energy; an FP32 phase that did not converge passes its status on.
__global__ void k_batch_fwd_handoff(const nlb_ctrl* c32, nlb_ctrl* c64, const nlb_struct_state s32,
                                    nlb_struct_state s64, int64_t n1, int64_t n2, double eps, double mixing,
                                    int max_steps, int max_diis, int criterion) {
    const int par = c32->parity;
    const double* t1 = s32.t1[par];
    const float* t2 = static_cast<const float*>(s32.t2[par]);
    double* o1 = s64.t1[0];
    double* o2 = static_cast<double*>(s64.t2[0]);
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n1 + n2; e += stride) {
        if (e < n1) o1[e] = t1[e];
        else o2[e - n1] = (double)t2[e - n1];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        const double e0 = c32->e_last;
        c64->e_acc = 0.0; c64->dt1_sq = 0.0; c64->dt2_sq = 0.0;
        c64->e_prev = e0; c64->e_last = e0; c64->eps = eps; c64->mixing = mixing;
        for (int k = 0; k < 121; ++k) c64->gram[k] = 0.0;
        const int left = max_steps - c32->iter;
        c64->parity = 0; c64->iter = 0; c64->max_steps = left;
        c64->criterion = criterion; c64->max_diis = max_diis; c64->diis_count = 0; c64->diis_pulse = 0;
        c64->diis_applied = 0; c64->ccs = 0;
        c64->status = (c32->status == NLB_CONVERGED) ? (left > 0 ? NLB_RUNNING : NLB_MAX_ITER) : c32->status;
    }
}

// Converged FP64 amplitudes (current parity) into buffer 0, and as FP32 into
// `t2f` (the Lambda FP32 phase reads them there).
__global__ void k_batch_amp_handoff(const nlb_ctrl* c64, nlb_struct_state s64, float* t2f, int64_t n1, int64_t n2) {
    const int par = c64->parity;
    const double* t1 = s64.t1[par];
    const double* t2 = static_cast<const double*>(s64.t2[par]);
    double* o1 = s64.t1[0];
    double* o2 = static_cast<double*>(s64.t2[0]);
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n1 + n2; e += stride) {
        if (e < n1) {
            if (par) o1[e] = t1[e];
        } else {
            const double v = t2[e - n1];
            if (par) o2[e - n1] = v;
            if (t2f) t2f[e - n1] = (float)v;
        }
    }
}

// Converged FP32 multipliers (current parity) into buffer 0 of the FP64 phase.
__global__ void k_batch_lam_handoff(const nlb_ctrl* l32, nlb_lambda_state s32, nlb_lambda_state s64, int64_t n1,
                                    int64_t n2) {
    const int par = l32->parity;
    const double* a = s32.lam1[par];
    const float* b = static_cast<const float*>(s32.lam2[par]);
    double* o1 = s64.lam1[0];
    double* o2 = static_cast<double*>(s64.lam2[0]);
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n1 + n2; e += stride) {
        if (e < n1) o1[e] = a[e];
        else o2[e - n1] = (double)b[e - n1];
    }
}

// A Lambda phase runs only for instances whose forward solve converged.
__global__ void k_batch_gate(const nlb_ctrl* fwd, nlb_ctrl* lam) {
    if (threadIdx.x == 0 && blockIdx.x == 0 && fwd->status != NLB_CONVERGED) lam->status = fwd->status;
}

// out[0] E_corr of the last forward phase, [3] its status, [4] forward
// iterations (both phases), [5] Lambda status, [6] Lambda iterations (both
// phases), [7] FP32 forward iterations; [1], [2] hold the coupling terms
// (nlb_lambda_coupling), or without a Lambda phase the parity of the last
// forward phase and the FP32 energy.  Phases that did not run are null.
__global__ void k_batch_report(const nlb_ctrl* c32, const nlb_ctrl* c64, const nlb_ctrl* l32, const nlb_ctrl* l64,
                               double* out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const nlb_ctrl* last = c64 ? c64 : c32;
    out[0] = last->e_last;
    if (!l64) {   // forward only: the parity of the last phase and the FP32 energy
        out[1] = (double)last->parity;
        out[2] = c32 ? c32->e_last : last->e_last;
    }
    out[3] = (double)last->status;
    out[4] = (double)((c32 ? c32->iter : 0) + (c64 ? c64->iter : 0));
    out[5] = l64 ? (double)l64->status : 0.0;
    out[6] = (double)((l32 ? l32->iter : 0) + (l64 ? l64->iter : 0));
    out[7] = c32 ? (double)c32->iter : 0.0;
}

struct Batch {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t cs = nullptr;
    cudaStream_t aux = nullptr;   // captures the body of one instance's IF node
    std::vector<cudaStream_t> streams;
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> join;
    void* dmem = nullptr;   // ctrl pointer lists and loop counters
    int n = 0;
};

void release(Batch* b) {
    if (!b) return;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    for (cudaStream_t s : b->streams) cudaStreamDestroy(s);
    if (b->cs) cudaStreamDestroy(b->cs);
    if (b->aux) cudaStreamDestroy(b->aux);
    if (b->fork) cudaEventDestroy(b->fork);
    for (cudaEvent_t e : b->join) cudaEventDestroy(e);
    if (b->dmem) cudaFree(b->dmem);
    delete b;
}

// Fork one branch per instance from the capturing stream, run fn(i, stream)
// on it, join back.
template <typename F>
int parallel(Batch* b, F fn) {
    int rc = bcuda(cudaEventRecord(b->fork, b->cs), "batch fork");
    if (rc) return rc;
    // every forked branch is joined back, also after an error, so that the
    // capture can always be ended cleanly
    for (int i = 0; i < b->n; ++i) {
        cudaStream_t s = b->streams[i];
        if (cudaStreamWaitEvent(s, b->fork, 0) != cudaSuccess) {
            if (!rc) rc = bcuda(cudaGetLastError(), "batch fork wait");
            continue;
        }
        if (!rc) rc = fn(i, s);
        const int rj = bcuda(cudaEventRecord(b->join[i], s), "batch join");
        const int rw = rj ? rj : bcuda(cudaStreamWaitEvent(b->cs, b->join[i], 0), "batch join wait");
        if (!rc) rc = rw;
    }
    return rc;
}

// Append a captured segment to the top graph after node `prev`.
template <typename F>
int append_segment(Batch* b, cudaGraphNode_t* prev, F fn) {
    cudaGraph_t child = nullptr;
    int rc = bcuda(cudaStreamBeginCapture(b->cs, cudaStreamCaptureModeRelaxed), "batch capture");
    if (rc) return rc;
    const int rc_fn = fn();
    rc = bcuda(cudaStreamEndCapture(b->cs, &child), "batch capture end");
    if (rc_fn) {
        if (child) cudaGraphDestroy(child);
        return rc_fn;
    }
    if (rc) return rc;
    cudaGraphNode_t node;
    rc = bcuda(cudaGraphAddChildGraphNode(&node, b->graph, *prev ? prev : nullptr, *prev ? 1 : 0, child),
               "batch child graph");
    cudaGraphDestroy(child);
    if (!rc) *prev = node;
    return rc;
}

// Zeroed parameters of a conditional node (the parameter union has no
// default constructor).
struct CondParams {
    alignas(cudaGraphNodeParams) unsigned char raw[sizeof(cudaGraphNodeParams)];
    CondParams(cudaGraphConditionalHandle h, cudaGraphConditionalNodeType type) {
        memset(raw, 0, sizeof(raw));
        cudaGraphNodeParams& p = get();
        p.type = cudaGraphNodeTypeConditional;
        p.conditional.handle = h;
        p.conditional.type = type;
        p.conditional.size = 1;
    }
    cudaGraphNodeParams& get() { return *reinterpret_cast<cudaGraphNodeParams*>(raw); }
};

// Append a device-side while loop.  Its body holds, per instance, an IF node
// whose body is captured from fn(i, stream), and ends in the condition kernel
// over `ctrls` (device array of n control blocks).  `hdev` receives the n
// per-instance handles (device memory, read by the condition kernel).
template <typename F>
int append_loop(Batch* b, cudaGraphNode_t* prev, nlb_ctrl* const* ctrls, cudaGraphConditionalHandle* hdev,
                int* counter, int cap, F fn) {
    cudaGraphConditionalHandle h;
    int rc = bcuda(cudaGraphConditionalHandleCreate(&h, b->graph, 1, cudaGraphCondAssignDefault), "batch handle");
    if (rc) return rc;
    CondParams lp(h, cudaGraphCondTypeWhile);
    cudaGraphNode_t node;
    rc = bcuda(cudaGraphAddNode(&node, b->graph, *prev ? prev : nullptr, *prev ? 1 : 0, &lp.get()), "batch loop node");
    if (rc) return rc;
    cudaGraph_t body = lp.get().conditional.phGraph_out[0];
    std::vector<cudaGraphConditionalHandle> hs(b->n);
    for (int i = 0; i < b->n && !rc; ++i)
        rc = bcuda(cudaGraphConditionalHandleCreate(&hs[i], body, 1, cudaGraphCondAssignDefault), "batch handle");
    if (!rc) rc = bcuda(cudaMemcpy(hdev, hs.data(), sizeof(cudaGraphConditionalHandle) * b->n, cudaMemcpyHostToDevice),
                        "batch handles");
    if (rc) return rc;
    rc = bcuda(cudaStreamBeginCaptureToGraph(b->cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed),
               "batch body capture");
    if (rc) return rc;
    int rc_fn = parallel(b, [&](int i, cudaStream_t s) {
        // IF node on the branch, its body captured on the instance's own stream
        cudaStreamCaptureStatus cst;
        cudaGraph_t cg = nullptr;
        const cudaGraphNode_t* deps = nullptr;
        size_t nd = 0;
        int q = bcuda(cudaStreamGetCaptureInfo(s, &cst, nullptr, &cg, &deps, &nd), "batch capture info");
        if (q) return q;
        CondParams ip(hs[i], cudaGraphCondTypeIf);
        cudaGraphNode_t inode;
        q = bcuda(cudaGraphAddNode(&inode, cg, deps, nd, &ip.get()), "batch instance node");
        if (q) return q;
        q = bcuda(cudaStreamUpdateCaptureDependencies(s, &inode, 1, cudaStreamSetCaptureDependencies),
                  "batch capture dependencies");
        if (q) return q;
        cudaStream_t aux = b->aux;
        q = bcuda(cudaStreamBeginCaptureToGraph(aux, ip.get().conditional.phGraph_out[0], nullptr, nullptr, 0,
                                                cudaStreamCaptureModeRelaxed), "batch instance capture");
        if (q) return q;
        const int qf = fn(i, aux);
        cudaGraph_t outg = nullptr;
        q = bcuda(cudaStreamEndCapture(aux, &outg), "batch instance capture end");
        return qf ? qf : q;
    });
    if (!rc_fn) {
        k_batch_cond<<<1, 32, 0, b->cs>>>(h, hdev, ctrls, b->n, counter, cap);
        rc_fn = bcuda(cudaGetLastError(), "batch condition kernel");
    }
    cudaGraph_t out = nullptr;
    rc = bcuda(cudaStreamEndCapture(b->cs, &out), "batch body capture end");
    if (rc_fn) return rc_fn;
    if (rc) return rc;
    *prev = node;
    return NLB_OK;
}

int steps(const nlb_batch_item& it, const nlb_struct_state* st, int chunk, int max_diis, cudaStream_t s) {
    for (int k = 0; k < chunk; ++k) {
        int rc = nlb_struct_step(it.prob, st, s);
        if (!rc && max_diis > 0 && (k + 1) % max_diis == 0) rc = nlb_struct_diis(it.prob, st, max_diis, s);
        if (rc) return rc;
    }
    return NLB_OK;
}

int lsteps(const nlb_batch_item& it, const nlb_lambda_state* st, int chunk, int max_diis, cudaStream_t s) {
    for (int k = 0; k < chunk; ++k) {
        int rc = nlb_lambda_step(it.prob, st, s);
        if (!rc && max_diis > 0 && (k + 1) % max_diis == 0) rc = nlb_lambda_diis(it.prob, st, max_diis, s);
        if (rc) return rc;
    }
    return NLB_OK;
}

int build(Batch* b, const nlb_batch_item* items, const nlb_batch_config& cfg) {
    const int n = b->n;
    const int chunk = cfg.chunk;
    const int md = cfg.max_diis;
    // device lists of control blocks per phase, and four loop counters
    nlb_ctrl** lists = static_cast<nlb_ctrl**>(b->dmem);
    cudaGraphConditionalHandle* handles = reinterpret_cast<cudaGraphConditionalHandle*>(lists + 4 * n);
    int* counters = reinterpret_cast<int*>(handles + 4 * n);
    {
        std::vector<nlb_ctrl*> h(4 * n);
        for (int i = 0; i < n; ++i) {
            h[i] = items[i].f32.ctrl;
            h[n + i] = items[i].f64.ctrl;
            h[2 * n + i] = items[i].l32.dtype ? items[i].l32.ctrl : items[i].l64.ctrl;
            h[3 * n + i] = items[i].l64.ctrl;
        }
        int rc = bcuda(cudaMemcpy(lists, h.data(), sizeof(nlb_ctrl*) * 4 * n, cudaMemcpyHostToDevice), "batch lists");
        if (rc) return rc;
    }
    const int cap_f = (cfg.max_steps + chunk - 1) / chunk + 1;
    const int cap_l = (cfg.lambda_max_steps + chunk - 1) / chunk + 1;
    const bool f32 = cfg.phases & NLB_PHASE_FWD32, f64 = cfg.phases & NLB_PHASE_FWD64,
               lam = cfg.phases & NLB_PHASE_LAMBDA;
    cudaGraphNode_t prev = nullptr;
    int rc;
    // prologue: start amplitudes and control block of the first forward phase
    rc = append_segment(b, &prev, [&]() {
        int r = bcuda(cudaMemsetAsync(counters, 0, 4 * sizeof(int), b->cs), "batch counters");
        if (r) return r;
        return parallel(b, [&](int i, cudaStream_t s) {
            const nlb_batch_item& it = items[i];
            const nlb_struct_state& st = f32 ? it.f32 : it.f64;
            const int64_t n1 = (int64_t)it.prob->p * it.prob->h, n2 = it.prob->n_t2;
            int q = bcuda(cudaMemcpyAsync(st.t1[0], it.t1_init, sizeof(double) * n1, cudaMemcpyDeviceToDevice, s),
                          "batch t1 start");
            if (!q && n2 > 0)
                q = bcuda(cudaMemsetAsync(st.t2[0], 0, (f32 ? sizeof(float) : sizeof(double)) * n2, s), "batch t2 start");
            if (!q) q = nlb_struct_ctrl_init(st.ctrl, f32 ? cfg.mixed_eps : cfg.eps, cfg.mixing, cfg.max_steps,
                                             cfg.criterion, md, 0, it.e0, s);
            return q;
        });
    });
    if (rc) return rc;
    if (f32) {
        // forward, FP32
        rc = append_loop(b, &prev, lists, handles, counters + 0, cap_f,
                         [&](int i, cudaStream_t s) { return steps(items[i], &items[i].f32, chunk, md, s); });
        if (rc) return rc;
    }
    if (f32 && f64) {
        // handoff to FP64
        rc = append_segment(b, &prev, [&]() {
            return parallel(b, [&](int i, cudaStream_t s) {
                const nlb_batch_item& it = items[i];
                const int64_t n1 = (int64_t)it.prob->p * it.prob->h, n2 = it.prob->n_t2;
                k_batch_fwd_handoff<<<grid_for(n1 + n2), kT, 0, s>>>(it.f32.ctrl, it.f64.ctrl, it.f32, it.f64, n1, n2,
                                                                   cfg.eps, cfg.mixing, cfg.max_steps, md,
                                                                   cfg.criterion);
                return bcuda(cudaGetLastError(), "batch forward handoff");
            });
        });
        if (rc) return rc;
    }
    if (f64) {
        // forward, FP64 (finish)
        rc = append_loop(b, &prev, lists + n, handles + n, counters + 1, cap_f,
                         [&](int i, cudaStream_t s) { return steps(items[i], &items[i].f64, chunk, md, s); });
        if (rc) return rc;
    }
    if (!lam) {
        return append_segment(b, &prev, [&]() {
            return parallel(b, [&](int i, cudaStream_t s) {
                const nlb_batch_item& it = items[i];
                k_batch_report<<<1, 32, 0, s>>>(f32 ? it.f32.ctrl : nullptr, f64 ? it.f64.ctrl : nullptr, nullptr,
                                               nullptr, it.out);
                return bcuda(cudaGetLastError(), "batch report");
            });
        });
    }
    // handoff to the Lambda equations
    rc = append_segment(b, &prev, [&]() {
        return parallel(b, [&](int i, cudaStream_t s) {
            const nlb_batch_item& it = items[i];
            const int64_t n1 = (int64_t)it.prob->p * it.prob->h, n2 = it.prob->n_t2;
            float* t2f = it.l32.dtype ? static_cast<float*>(const_cast<void*>(it.l32.t2)) : nullptr;
            k_batch_amp_handoff<<<grid_for(n1 + n2), kT, 0, s>>>(it.f64.ctrl, it.f64, t2f, n1, n2);
            int q = bcuda(cudaGetLastError(), "batch amplitude handoff");
            const nlb_lambda_state* ls = it.l32.dtype ? &it.l32 : &it.l64;
            const double tol = it.l32.dtype ? (cfg.lambda_tol_fp32 > cfg.lambda_tol ? cfg.lambda_tol_fp32
                                                                                     : cfg.lambda_tol)
                                            : cfg.lambda_tol;
            if (!q) q = nlb_lambda_init(it.prob, ls, tol, cfg.mixing, cfg.lambda_max_steps, md, 0, s);
            if (!q) {
                k_batch_gate<<<1, 32, 0, s>>>(it.f64.ctrl, ls->ctrl);
                q = bcuda(cudaGetLastError(), "batch gate");
            }
            return q;
        });
    });
    if (rc) return rc;
    // Lambda, FP32 (lattice instances; the others run their FP64 Lambda here)
    rc = append_loop(b, &prev, lists + 2 * n, handles + 2 * n, counters + 2, cap_l, [&](int i, cudaStream_t s) {
        const nlb_batch_item& it = items[i];
        return lsteps(it, it.l32.dtype ? &it.l32 : &it.l64, chunk, md, s);
    });
    if (rc) return rc;
    // handoff to the FP64 Lambda finish (lattice instances)
    rc = append_segment(b, &prev, [&]() {
        return parallel(b, [&](int i, cudaStream_t s) {
            const nlb_batch_item& it = items[i];
            if (!it.l32.dtype) return (int)NLB_OK;
            const int64_t n1 = (int64_t)it.prob->p * it.prob->h, n2 = it.prob->n_t2;
            k_batch_lam_handoff<<<grid_for(n1 + n2), kT, 0, s>>>(it.l32.ctrl, it.l32, it.l64, n1, n2);
            int q = bcuda(cudaGetLastError(), "batch multiplier handoff");
            if (!q) q = nlb_lambda_init(it.prob, &it.l64, cfg.lambda_tol, cfg.mixing, cfg.lambda_max_steps, md,
                                        NLB_LAMBDA_KEEP, s);
            if (!q) {
                k_batch_gate<<<1, 32, 0, s>>>(it.f64.ctrl, it.l64.ctrl);
                q = bcuda(cudaGetLastError(), "batch gate");
            }
            return q;
        });
    });
    if (rc) return rc;
    // Lambda, FP64 finish
    rc = append_loop(b, &prev, lists + 3 * n, handles + 3 * n, counters + 3, cap_l, [&](int i, cudaStream_t s) {
        const nlb_batch_item& it = items[i];
        return it.l32.dtype ? lsteps(it, &it.l64, chunk, md, s) : (int)NLB_OK;
    });
    if (rc) return rc;
    // coupling terms and the report
    rc = append_segment(b, &prev, [&]() {
        return parallel(b, [&](int i, cudaStream_t s) {
            const nlb_batch_item& it = items[i];
            int q = (int)NLB_OK;
            for (int d = 0; d < 2 && !q; ++d) q = nlb_lambda_coupling(it.prob, &it.l64, it.dw[d], it.dv[d], it.out + 1 + d, s);
            if (!q) {
                k_batch_report<<<1, 32, 0, s>>>(f32 ? it.f32.ctrl : nullptr, it.f64.ctrl,
                                               it.l32.dtype ? it.l32.ctrl : nullptr, it.l64.ctrl, it.out);
                q = bcuda(cudaGetLastError(), "batch report");
            }
            return q;
        });
    });
    return rc;
}

}  // namespace

extern "C" {

int nlb_batch_create(const nlb_batch_item* items, int32_t n, const nlb_batch_config* cfg, void** handle) {
    if (!items || !cfg || !handle || n <= 0) return bfail(NLB_ERR_ARG, "nlb_batch_create: bad arguments");
    *handle = nullptr;
    if (cfg->chunk < 1 || (cfg->max_diis > 0 && cfg->chunk % cfg->max_diis != 0))
        return bfail(NLB_ERR_ARG, "nlb_batch_create: chunk must be a positive multiple of max_diis");
    const int ph = cfg->phases;
    if (!(ph & (NLB_PHASE_FWD32 | NLB_PHASE_FWD64)) || (ph & ~7) ||
        ((ph & NLB_PHASE_LAMBDA) && !(ph & NLB_PHASE_FWD64)))
        return bfail(NLB_ERR_ARG, "nlb_batch_create: phases need a forward phase; Lambda needs the FP64 forward phase");
    if (cfg->criterion != NLB_CRIT_SOA && cfg->criterion != NLB_CRIT_NUMPY)
        return bfail(NLB_ERR_ARG, "nlb_batch_create: bad criterion");
    for (int i = 0; i < n; ++i) {
        const nlb_batch_item& it = items[i];
        if (!it.prob || !it.t1_init || !it.out) return bfail(NLB_ERR_ARG, "nlb_batch_create: null item field");
        if (((ph & NLB_PHASE_FWD32) && it.f32.dtype != NLB_F32) || ((ph & NLB_PHASE_FWD64) && it.f64.dtype != NLB_F64))
            return bfail(NLB_ERR_ARG, "nlb_batch_create: forward state dtypes must be F32 and F64");
        if (ph & NLB_PHASE_LAMBDA) {
            if (!it.dw[0] || !it.dw[1] || !it.dv[0] || !it.dv[1])
                return bfail(NLB_ERR_ARG, "nlb_batch_create: null derivative ladders");
            if (it.l64.dtype != NLB_F64 || (it.l32.dtype != 0 && it.l32.dtype != NLB_F32))
                return bfail(NLB_ERR_ARG, "nlb_batch_create: Lambda state dtypes must be (F32 or 0) and F64");
            if (it.l64.t1 != it.f64.t1[0] || it.l64.t2 != it.f64.t2[0] || (it.l32.dtype && it.l32.t1 != it.f64.t1[0]))
                return bfail(NLB_ERR_ARG,
                             "nlb_batch_create: Lambda states must read t1/t2 from buffer 0 of the FP64 state");
        }
    }
    Batch* b = new Batch();
    b->n = n;
    int rc = bcuda(cudaStreamCreateWithFlags(&b->cs, cudaStreamNonBlocking), "batch stream");
    if (!rc) rc = bcuda(cudaStreamCreateWithFlags(&b->aux, cudaStreamNonBlocking), "batch stream");
    b->streams.resize(n, nullptr);
    b->join.resize(n, nullptr);
    for (int i = 0; i < n && !rc; ++i) rc = bcuda(cudaStreamCreateWithFlags(&b->streams[i], cudaStreamNonBlocking), "batch stream");
    if (!rc) rc = bcuda(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming), "batch event");
    for (int i = 0; i < n && !rc; ++i) rc = bcuda(cudaEventCreateWithFlags(&b->join[i], cudaEventDisableTiming), "batch event");
    if (!rc)
        rc = bcuda(cudaMalloc(&b->dmem, sizeof(nlb_ctrl*) * 4 * n + sizeof(cudaGraphConditionalHandle) * 4 * n +
                                            16 * sizeof(int)), "batch lists");
    if (!rc) rc = bcuda(cudaGraphCreate(&b->graph, 0), "batch graph");
    if (!rc) rc = build(b, items, *cfg);
    if (!rc) rc = bcuda(cudaGraphInstantiate(&b->exec, b->graph, 0), "batch instantiate");
    if (rc) {
        release(b);
        return rc;
    }
    *handle = b;
    return NLB_OK;
}

int nlb_batch_launch(void* handle, nlb_stream_t stream) {
    if (!handle) return bfail(NLB_ERR_ARG, "nlb_batch_launch: null handle");
    Batch* b = static_cast<Batch*>(handle);
    return bcuda(cudaGraphLaunch(b->exec, (cudaStream_t)stream), "nlb_batch_launch");
}

int nlb_batch_destroy(void* handle) {
    release(static_cast<Batch*>(handle));
    return NLB_OK;
}

}  // extern "C"
