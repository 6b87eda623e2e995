// Structured CCSD kernels for sm_100a (B200).
//
// Closed-site lattice inputs conserve a label (spin-isospin) on every state,
// and every two-body block except the particle-particle and hole-hole ones is
// zero.  The reference's t1Iter / t2Iter (CCM/coupled_cluster.py:342-545)
// then reduce to the terms computed here on the compact channel layout of T2
// (one dense block B[a'][b'][i'][j'] per label pair g1 < g2; the other three
// antisymmetric images are implied):
//
//   R2 = f_pp stencil along a and b          (P(ab) X_pp t2, sparse part)
//      - t1 (f_ph^T B) along a and b         (P(ab) X_pp t2, rank-h part)
//      + X_hh mixing along i and j           (P(ij) X_hh t2)
//      + sum v_hhhh tau + sum v_pppp tau     (ladders, tau = t2 + t1 t1)
//   t2' = m t2 + (1-m) (t2 + R2 / D2)
//
//   R1 = f_ph + f_ck t2_acik + X_pp t1 + t1 X_hh
//   t1' = m t1 + (1-m) (t1 + R1 / D1),   E = sum f_ai t1'_ai
//
// Every launch reads the current buffers (ctrl->parity) and writes the other
// ones, so a step is position independent and can be queued or captured.
// The T2 update is bandwidth bound: each stored amplitude is read once from
// HBM, its stencil neighbours come from L1/L2, and it is written once (plus
// once more into the DIIS error ring when DIIS is on).

#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include "nulattice_b200.h"

static thread_local char g_err[512] = "";

static int fail(int code, const char* msg) {
    snprintf(g_err, sizeof(g_err), "%s", msg);
    return code;
}

static int check_launch(const char* where) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        snprintf(g_err, sizeof(g_err), "%s: %s", where, cudaGetErrorString(e));
        return NLB_ERR_LAUNCH;
    }
    return NLB_OK;
}

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ int find_seg(const int64_t* end, int n, int64_t e) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (e < end[mid]) hi = mid; else lo = mid + 1;
    }
    return lo;
}

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide sum; every thread of the block must call it.
__device__ double block_sum(double v) {
    __shared__ double s[32];
    v = warp_sum(v);
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) s[w] = v;
    __syncthreads();
    int nw = (blockDim.x + 31) >> 5;
    v = (threadIdx.x < nw) ? s[threadIdx.x] : 0.0;
    if (w == 0) v = warp_sum(v);
    return v;  // valid in thread 0
}

// ---------------------------------------------------------------- prep ----
// Q[k,j] = sum_c f_ck t1_cj; X_hh for the T2 equation (-f_hh - Q) and for the
// T1 equation (-f_hh - Q/2); diagonals of X_pp: f_aa - S_a and f_aa - S_a/2,
// S_a = sum_k f_ak t1_ak (coupled_cluster.py:385-399, 501-515).
__global__ void k_prep(nlb_struct_problem P, nlb_struct_state S) {
    const nlb_ctrl* c = S.ctrl;
    if (c->status != NLB_RUNNING) return;
    const double* t1 = S.t1[c->parity];
    const int h = P.h, p = P.p;
    double* Q = S.prep;
    double* Xh2 = Q + (int64_t)h * h;
    double* Xh1 = Xh2 + (int64_t)h * h;
    double* dXp2 = Xh1 + (int64_t)h * h;
    double* dXp1 = dXp2 + p;
    int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid < (int64_t)h * h) {
        int k = (int)(tid / h), j = (int)(tid % h);
        int g = P.h_label[k];
        int row = P.h_base[g] + P.h_loc[k];
        int pb = P.p_base[g];
        double q = 0.0;
        for (int e = P.fph_ptr[row]; e < P.fph_ptr[row + 1]; ++e)
            q += P.fph_val[e] * t1[(int64_t)P.p_ord[pb + P.fph_col[e]] * h + j];
        Q[tid] = q;
        Xh2[tid] = -P.f_hh[tid] - q;
        Xh1[tid] = -P.f_hh[tid] - 0.5 * q;
    } else if (tid < (int64_t)h * h + p) {
        int a = (int)(tid - (int64_t)h * h);
        double s = 0.0;
        for (int k = 0; k < h; ++k) s += P.f_ph[(int64_t)a * h + k] * t1[(int64_t)a * h + k];
        dXp2[a] = P.fpp_diag[a] - s;
        dXp1[a] = P.fpp_diag[a] - 0.5 * s;
    }
}

// ----------------------------------------------------------- G terms ----
// Gb[a',k',hp] = sum_c f_ck B[a',c',hp]  (k a hole of label g2)
// Ga[b',k',hp] = sum_c f_ck B[c',b',hp]  (k a hole of label g1)
// They carry the rank-h part of X_pp (f_ph t1^T) in the T2 equation and the
// Fock term f_ck t2_acik of the T1 equation.
template <typename T>
__global__ void k_gterms(nlb_struct_problem P, nlb_struct_state S) {
    const nlb_ctrl* c = S.ctrl;
    if (c->status != NLB_RUNNING || c->ccs) return;
    const T* B = static_cast<const T*>(S.t2[c->parity]);
    T* G = static_cast<T*>(S.g);
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < P.n_g; e += stride) {
        const int ci = find_seg(P.g_end, P.n_channels, e);
        const nlb_channel ch = P.chan[ci];
        int64_t loc = e - ch.gb_off;
        const int nhp = ch.nh1 * ch.nh2;
        const int64_t n_gb = (int64_t)ch.np1 * ch.nh2 * nhp;
        const T* Bc = B + ch.offset;
        T acc = T(0);
        if (loc < n_gb) {
            const int hp = (int)(loc % nhp);
            const int64_t r = loc / nhp;
            const int kq = (int)(r % ch.nh2), ap = (int)(r / ch.nh2);
            const int row = ch.hb2 + kq;
            for (int q = P.fph_ptr[row]; q < P.fph_ptr[row + 1]; ++q)
                acc += (T)P.fph_val[q] * Bc[((int64_t)ap * ch.np2 + P.fph_col[q]) * nhp + hp];
        } else {
            loc -= n_gb;
            const int hp = (int)(loc % nhp);
            const int64_t r = loc / nhp;
            const int kq = (int)(r % ch.nh1), bp = (int)(r / ch.nh1);
            const int row = ch.hb1 + kq;
            for (int q = P.fph_ptr[row]; q < P.fph_ptr[row + 1]; ++q)
                acc += (T)P.fph_val[q] * Bc[((int64_t)P.fph_col[q] * ch.np2 + bp) * nhp + hp];
        }
        G[e] = acc;
    }
}

// --------------------------------------------------------- T2 update ----
template <typename T>
__global__ void __launch_bounds__(kThreads) k_t2_update(nlb_struct_problem P, nlb_struct_state S) {
    const nlb_ctrl* c = S.ctrl;
    if (c->status != NLB_RUNNING || c->ccs) return;
    const int par = c->parity;
    const T* __restrict__ B = static_cast<const T*>(S.t2[par]);
    T* __restrict__ Bo = static_cast<T*>(S.t2[par ^ 1]);
    const double* __restrict__ t1 = S.t1[par];
    const int h = P.h;
    const double* Xh2 = S.prep + (int64_t)h * h;
    const double* dXp2 = S.prep + 3 * (int64_t)h * h;
    const T* __restrict__ G = static_cast<const T*>(S.g);
    T* E2 = (S.diis_t2 != nullptr && c->max_diis > 0 && c->diis_count < c->max_diis)
                ? static_cast<T*>(S.diis_t2) + (int64_t)c->diis_count * P.n_t2 : nullptr;
    const T m = (T)c->mixing, om = (T)(1.0 - c->mixing);
    double nrm = 0.0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < P.n_t2; e += stride) {
        const int ci = find_seg(P.t2_end, P.n_channels, e);
        const nlb_channel ch = P.chan[ci];
        const int64_t loc = e - ch.offset;
        const int nh1 = ch.nh1, nh2 = ch.nh2, np2 = ch.np2;
        const int nhp = nh1 * nh2;
        const int hp = (int)(loc % nhp);
        const int64_t ab = loc / nhp;
        const int bp = (int)(ab % np2), ap = (int)(ab / np2);
        const int ip = hp / nh2, jp = hp % nh2;
        const int a = P.p_ord[ch.pb1 + ap], b = P.p_ord[ch.pb2 + bp];
        const int i = P.h_ord[ch.hb1 + ip], j = P.h_ord[ch.hb2 + jp];
        const T* Bc = B + ch.offset;
        const T* row = Bc + ab * nhp;
        const T x = row[hp];
        T R = T(0);
        // f_pp along b and along a
        const int rb = ch.pb2 + bp;
        for (int q = P.fpp_ptr[rb]; q < P.fpp_ptr[rb + 1]; ++q)
            R += (T)P.fpp_val[q] * Bc[((int64_t)ap * np2 + P.fpp_col[q]) * nhp + hp];
        const int ra = ch.pb1 + ap;
        for (int q = P.fpp_ptr[ra]; q < P.fpp_ptr[ra + 1]; ++q)
            R += (T)P.fpp_val[q] * Bc[((int64_t)P.fpp_col[q] * np2 + bp) * nhp + hp];
        // rank-h part of X_pp: -t1_bk Gb[a',k'] - t1_ak Ga[b',k']
        const T* Gb = G + ch.gb_off + (int64_t)ap * nh2 * nhp + hp;
        for (int kq = 0; kq < nh2; ++kq)
            R -= (T)t1[(int64_t)b * h + P.h_ord[ch.hb2 + kq]] * Gb[(int64_t)kq * nhp];
        const T* Ga = G + ch.ga_off + (int64_t)bp * nh1 * nhp + hp;
        for (int kq = 0; kq < nh1; ++kq)
            R -= (T)t1[(int64_t)a * h + P.h_ord[ch.hb1 + kq]] * Ga[(int64_t)kq * nhp];
        // X_hh along i and along j
        for (int kq = 0; kq < nh1; ++kq)
            R += (T)Xh2[(int64_t)P.h_ord[ch.hb1 + kq] * h + i] * row[kq * nh2 + jp];
        for (int kq = 0; kq < nh2; ++kq)
            R += (T)Xh2[(int64_t)P.h_ord[ch.hb2 + kq] * h + j] * row[ip * nh2 + kq];
        // hole-hole ladder on tau
        {
            const int32_t* ptr = P.hh_ptr + ch.hh_ptr_off;
            const int32_t* col = P.hh_col + ch.hh_col_off;
            const double* val = P.hh_val + ch.hh_col_off;
            for (int q = ptr[hp]; q < ptr[hp + 1]; ++q) {
                const int in = col[q];
                const int kq = in / nh2, lq = in % nh2;
                const T tau = row[in] + (T)(t1[(int64_t)a * h + P.h_ord[ch.hb1 + kq]] *
                                            t1[(int64_t)b * h + P.h_ord[ch.hb2 + lq]]);
                R += (T)val[q] * tau;
            }
        }
        // particle-particle ladder on tau
        {
            const int32_t* ptr = P.pp_ptr + ch.pp_ptr_off;
            const int32_t* col = P.pp_col + ch.pp_col_off;
            const double* val = P.pp_val + ch.pp_col_off;
            for (int q = ptr[ab]; q < ptr[ab + 1]; ++q) {
                const int in = col[q];
                const int cq = in / np2, dq = in % np2;
                const T tau = Bc[(int64_t)in * nhp + hp] +
                              (T)(t1[(int64_t)P.p_ord[ch.pb1 + cq] * h + i] *
                                  t1[(int64_t)P.p_ord[ch.pb2 + dq] * h + j]);
                R += (T)val[q] * tau;
            }
        }
        const double dd = -((dXp2[a] + dXp2[b]) + (Xh2[(int64_t)i * h + i] + Xh2[(int64_t)j * h + j]));
        const T tn = x + R / (T)dd;
        const T out = m * x + om * tn;
        Bo[e] = out;
        const T d = out - x;
        if (E2) E2[e] = d;
        nrm += (double)d * (double)d;
    }
    const double s = block_sum(nrm);
    if (threadIdx.x == 0) atomicAdd(&S.ctrl->dt2_sq, 4.0 * s);
}

// --------------------------------------------------------- T1 update ----
template <typename T>
__global__ void __launch_bounds__(kThreads) k_t1_update(nlb_struct_problem P, nlb_struct_state S) {
    nlb_ctrl* c = S.ctrl;
    if (c->status != NLB_RUNNING) return;
    const int par = c->parity;
    const double* t1 = S.t1[par];
    double* t1o = S.t1[par ^ 1];
    const int h = P.h, p = P.p;
    const double* Q = S.prep;
    const double* Xh1 = S.prep + 2 * (int64_t)h * h;
    const double* dXp1 = S.prep + 3 * (int64_t)h * h + p;
    const T* G = static_cast<const T*>(S.g);
    double* E1 = (S.diis_t1 != nullptr && c->max_diis > 0 && c->diis_count < c->max_diis)
                     ? S.diis_t1 + (int64_t)c->diis_count * p * h : nullptr;
    const double m = c->mixing;
    double eacc = 0.0, nrm = 0.0;
    const int64_t n = (int64_t)p * h;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += stride) {
        const int a = (int)(idx / h), i = (int)(idx % h);
        const int g = P.p_label[a];
        if (P.h_label[i] != g) {
            t1o[idx] = 0.0;
            if (E1) E1[idx] = 0.0;
            continue;
        }
        const int ap = P.p_loc[a], ip = P.h_loc[i];
        double H1 = P.f_ph[idx];
        if (!c->ccs) {
            for (int cc = 0; cc < P.n_channels; ++cc) {
                const nlb_channel ch = P.chan[cc];
                const int nhp = ch.nh1 * ch.nh2;
                if (ch.g1 == g) {
                    const T* Gb = G + ch.gb_off + (int64_t)ap * ch.nh2 * nhp + ip * ch.nh2;
                    for (int kq = 0; kq < ch.nh2; ++kq) H1 += (double)Gb[(int64_t)kq * nhp + kq];
                } else if (ch.g2 == g) {
                    const T* Ga = G + ch.ga_off + (int64_t)ap * ch.nh1 * nhp + ip;
                    for (int kq = 0; kq < ch.nh1; ++kq) H1 += (double)Ga[(int64_t)kq * nhp + kq * ch.nh2];
                }
            }
        }
        const int pb = P.p_base[g];
        const int r = pb + ap;
        for (int q = P.fpp_ptr[r]; q < P.fpp_ptr[r + 1]; ++q)
            H1 += P.fpp_val[q] * t1[(int64_t)P.p_ord[pb + P.fpp_col[q]] * h + i];
        for (int k = 0; k < h; ++k) {
            const double tk = t1[(int64_t)a * h + k];
            if (tk != 0.0) H1 += tk * (Xh1[(int64_t)k * h + i] - 0.5 * Q[(int64_t)k * h + i]);
        }
        const double D1 = -(dXp1[a] + Xh1[(int64_t)i * h + i]);
        const double x = t1[idx];
        const double tn = x + H1 / D1;
        const double out = m * x + (1.0 - m) * tn;
        t1o[idx] = out;
        const double d = out - x;
        if (E1) E1[idx] = d;
        nrm += d * d;
        eacc += P.f_ph[idx] * out;
    }
    const double se = block_sum(eacc);
    const double sn = block_sum(nrm);
    if (threadIdx.x == 0) {
        atomicAdd(&c->e_acc, se);
        atomicAdd(&c->dt1_sq, sn);
    }
}

// -------------------------------------------------- convergence test ----
__global__ void k_finish(nlb_ctrl* c) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    if (c->status != NLB_RUNNING) return;
    const double E = c->e_acc, prev = c->e_prev;
    c->iter += 1;
    c->parity ^= 1;
    c->e_last = E;
    c->diis_pulse = 0;
    bool done;
    if (c->criterion == NLB_CRIT_SOA)
        done = fabs(E - prev) / fmax(1.0, fabs(E)) < c->eps;
    else
        done = (E == 0.0 && prev == 0.0) || fabs(E - prev) / fabs(E) < c->eps;
    if (done) {
        c->status = NLB_CONVERGED;
        return;
    }
    if (c->max_diis > 0 && c->criterion == NLB_CRIT_SOA) {
        c->diis_count += 1;
        if (c->diis_count == c->max_diis) {
            c->diis_pulse = 1;
            for (int k = 0; k < 121; ++k) c->gram[k] = 0.0;
        }
    }
    if (fabs(E) > 1e10 || isnan(E))
        c->status = NLB_DIVERGED;
    else if (c->iter >= c->max_steps)
        c->status = NLB_MAX_ITER;
    c->e_prev = E;
    c->e_acc = 0.0;
    c->dt1_sq = 0.0;
    c->dt2_sq = 0.0;
}

// ---------------------------------------------------------------- DIIS ----
// Gram matrix of the stored error vectors: <e_a, e_b> over the dense t1 and
// the dense t2 (four images per stored amplitude).
constexpr int kMaxDiis = 10;

template <typename T>
__global__ void __launch_bounds__(kThreads) k_diis_gram(nlb_struct_problem P, nlb_struct_state S) {
    nlb_ctrl* c = S.ctrl;
    if (!c->diis_pulse) return;
    const int m = c->max_diis;
    double acc[kMaxDiis * (kMaxDiis + 1) / 2];
    for (int k = 0; k < kMaxDiis * (kMaxDiis + 1) / 2; ++k) acc[k] = 0.0;
    const int64_t n1 = (int64_t)P.p * P.h;
    const int64_t n2 = c->ccs ? 0 : P.n_t2;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const T* E2 = static_cast<const T*>(S.diis_t2);
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n1 + n2; e += stride) {
        double v[kMaxDiis];
        double w;
        if (e < n1) {
            for (int s = 0; s < m; ++s) v[s] = S.diis_t1[(int64_t)s * n1 + e];
            w = 1.0;
        } else {
            for (int s = 0; s < m; ++s) v[s] = (double)E2[(int64_t)s * P.n_t2 + (e - n1)];
            w = 4.0;
        }
        int k = 0;
        for (int s = 0; s < m; ++s)
            for (int t = s; t < m; ++t) acc[k++] += w * v[s] * v[t];
    }
    int k = 0;
    for (int s = 0; s < m; ++s)
        for (int t = s; t < m; ++t) {
            const double tot = block_sum(acc[k++]);
            if (threadIdx.x == 0) atomicAdd(&c->gram[s * kMaxDiis + t], tot);
        }
}

// Bordered DIIS system [B/max|B|, -1; -1, 0] c = [0, -1], solved by Gaussian
// elimination with partial pivoting in FP64.  A zero pivot skips the
// extrapolation (the torch solver catches the failed solve and goes on).
// Leaves in gram[0] the weight of the current amplitudes and in gram[1+s]
// the weight of error vector s (t_new = w0 t_m + sum_s w_s e_s).
__global__ void k_diis_solve(nlb_ctrl* c) {
    if (threadIdx.x != 0 || blockIdx.x != 0 || !c->diis_pulse) return;
    const int m = c->max_diis, n = m + 1;
    double A[(kMaxDiis + 1) * (kMaxDiis + 1)], rhs[kMaxDiis + 1];
    double mx = 0.0;
    for (int s = 0; s < m; ++s)
        for (int t = s; t < m; ++t) mx = fmax(mx, fabs(c->gram[s * kMaxDiis + t]));
    const double nrm = mx + 1e-16;
    for (int s = 0; s < n; ++s) {
        rhs[s] = (s == m) ? -1.0 : 0.0;
        for (int t = 0; t < n; ++t) {
            double v;
            if (s < m && t < m) v = c->gram[(s <= t) ? s * kMaxDiis + t : t * kMaxDiis + s] / nrm;
            else if (s == m && t == m) v = 0.0;
            else v = -1.0;
            A[s * n + t] = v;
        }
    }
    bool ok = true;
    for (int col = 0; col < n && ok; ++col) {
        int piv = col;
        for (int r = col + 1; r < n; ++r)
            if (fabs(A[r * n + col]) > fabs(A[piv * n + col])) piv = r;
        if (A[piv * n + col] == 0.0 || !isfinite(A[piv * n + col])) { ok = false; break; }
        if (piv != col) {
            for (int t = 0; t < n; ++t) { double tmp = A[col * n + t]; A[col * n + t] = A[piv * n + t]; A[piv * n + t] = tmp; }
            double tmp = rhs[col]; rhs[col] = rhs[piv]; rhs[piv] = tmp;
        }
        for (int r = col + 1; r < n; ++r) {
            const double f = A[r * n + col] / A[col * n + col];
            for (int t = col; t < n; ++t) A[r * n + t] -= f * A[col * n + t];
            rhs[r] -= f * rhs[col];
        }
    }
    double x[kMaxDiis + 1];
    if (ok) {
        for (int r = n - 1; r >= 0; --r) {
            double s = rhs[r];
            for (int t = r + 1; t < n; ++t) s -= A[r * n + t] * x[t];
            x[r] = s / A[r * n + r];
            if (!isfinite(x[r])) ok = false;
        }
    }
    c->diis_applied = ok ? 1 : 0;
    if (!ok) return;
    // t_new = sum_k x_k t_{k+1},  t_{k+1} = t_m - sum_{s>k} e_s
    double tot = 0.0;
    for (int k = 0; k < m; ++k) tot += x[k];
    c->gram[0] = tot;
    double run = 0.0;
    for (int s = 0; s < m; ++s) {
        c->gram[1 + s] = -run;
        run += x[s];
    }
}

template <typename T>
__global__ void __launch_bounds__(kThreads) k_diis_extrap(nlb_struct_problem P, nlb_struct_state S) {
    const nlb_ctrl* c = S.ctrl;
    if (!c->diis_pulse || !c->diis_applied) return;
    const int m = c->max_diis;
    const int par = c->parity;
    const double w0 = c->gram[0];
    double w[kMaxDiis];
    for (int s = 0; s < m; ++s) w[s] = c->gram[1 + s];
    const int64_t n1 = (int64_t)P.p * P.h;
    const int64_t n2 = c->ccs ? 0 : P.n_t2;
    double* t1 = S.t1[par];
    T* t2 = static_cast<T*>(S.t2[par]);
    const T* E2 = static_cast<const T*>(S.diis_t2);
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n1 + n2; e += stride) {
        if (e < n1) {
            double v = w0 * t1[e];
            for (int s = 0; s < m; ++s) v += w[s] * S.diis_t1[(int64_t)s * n1 + e];
            t1[e] = v;
        } else {
            const int64_t q = e - n1;
            double v = w0 * (double)t2[q];
            for (int s = 0; s < m; ++s) v += w[s] * (double)E2[(int64_t)s * P.n_t2 + q];
            t2[q] = (T)v;
        }
    }
}

__global__ void k_diis_done(nlb_ctrl* c) {
    if (threadIdx.x == 0 && blockIdx.x == 0 && c->diis_pulse) {
        c->diis_pulse = 0;
        c->diis_count = 0;
    }
}

// ------------------------------------------------------------- energy ----
__global__ void k_energy(nlb_struct_problem P, nlb_struct_state S, double* out) {
    const double* t1 = S.t1[S.ctrl->parity];
    const int64_t n = (int64_t)P.p * P.h;
    double acc = 0.0;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x)
        acc += P.f_ph[e] * t1[e];
    const double s = block_sum(acc);
    if (threadIdx.x == 0) atomicAdd(out, s);
}

__global__ void k_zero1(double* x) { *x = 0.0; }

__global__ void k_ctrl_init(nlb_ctrl* c, double eps, double mixing, int max_steps, int criterion,
                            int max_diis, int ccs, double e0) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    c->e_acc = 0.0; c->dt1_sq = 0.0; c->dt2_sq = 0.0;
    c->e_prev = e0; c->e_last = e0; c->eps = eps; c->mixing = mixing;
    for (int k = 0; k < 121; ++k) c->gram[k] = 0.0;
    c->parity = 0; c->iter = 0; c->status = NLB_RUNNING; c->max_steps = max_steps;
    c->criterion = criterion; c->max_diis = max_diis; c->diis_count = 0; c->diis_pulse = 0;
    c->diis_applied = 0; c->ccs = ccs;
    if (max_steps <= 0) c->status = NLB_MAX_ITER;
}

// ---------------------------------------------------- layout helpers ----
template <typename S, typename D>
__global__ void k_convert(const S* src, D* dst, int64_t n) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x)
        dst[e] = (D)src[e];
}

template <typename T>
__global__ void k_unpack(nlb_struct_problem P, const T* t2c, double* t2) {
    const int64_t p = P.p, h = P.h;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < P.n_t2; e += (int64_t)gridDim.x * blockDim.x) {
        const int ci = find_seg(P.t2_end, P.n_channels, e);
        const nlb_channel ch = P.chan[ci];
        const int64_t loc = e - ch.offset;
        const int nhp = ch.nh1 * ch.nh2;
        const int hp = (int)(loc % nhp);
        const int64_t ab = loc / nhp;
        const int a = P.p_ord[ch.pb1 + (int)(ab / ch.np2)], b = P.p_ord[ch.pb2 + (int)(ab % ch.np2)];
        const int i = P.h_ord[ch.hb1 + hp / ch.nh2], j = P.h_ord[ch.hb2 + hp % ch.nh2];
        const double v = (double)t2c[e];
        t2[((a * p + b) * h + i) * h + j] = v;
        t2[((b * p + a) * h + i) * h + j] = -v;
        t2[((a * p + b) * h + j) * h + i] = -v;
        t2[((b * p + a) * h + j) * h + i] = v;
    }
}

template <typename T>
__global__ void k_pack(nlb_struct_problem P, const double* t2, T* t2c) {
    const int64_t p = P.p, h = P.h;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < P.n_t2; e += (int64_t)gridDim.x * blockDim.x) {
        const int ci = find_seg(P.t2_end, P.n_channels, e);
        const nlb_channel ch = P.chan[ci];
        const int64_t loc = e - ch.offset;
        const int nhp = ch.nh1 * ch.nh2;
        const int hp = (int)(loc % nhp);
        const int64_t ab = loc / nhp;
        const int a = P.p_ord[ch.pb1 + (int)(ab / ch.np2)], b = P.p_ord[ch.pb2 + (int)(ab % ch.np2)];
        const int i = P.h_ord[ch.hb1 + hp / ch.nh2], j = P.h_ord[ch.hb2 + hp % ch.nh2];
        t2c[e] = (T)t2[((a * p + b) * h + i) * h + j];
    }
}

int g_num_sms = 0;

int num_sms() {
    if (g_num_sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev);
        if (g_num_sms <= 0) g_num_sms = 148;
    }
    return g_num_sms;
}

// Resident blocks per SM of each kernel, queried once.
struct OccEntry { const void* fn; int bps; };
OccEntry g_occ[64];
int g_nocc = 0;

int blocks_per_sm(const void* fn) {
    for (int k = 0; k < g_nocc; ++k)
        if (g_occ[k].fn == fn) return g_occ[k].bps;
    int bps = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, fn, kThreads, 0) != cudaSuccess || bps <= 0) bps = 2;
    if (g_nocc < 64) g_occ[g_nocc++] = OccEntry{fn, bps};
    return bps;
}

// Persistent-style grid: as many blocks as fit at once, never more than the work.
template <typename K>
int grid_for(K kernel, int64_t work) {
    const int bps = blocks_per_sm(reinterpret_cast<const void*>(kernel));
    int64_t full = (int64_t)num_sms() * bps;
    int64_t need = (work + kThreads - 1) / kThreads;
    if (need < 1) need = 1;
    return (int)(need < full ? need : full);
}

int valid(const nlb_struct_problem* P, const nlb_struct_state* S) {
    if (!P || !S || !S->ctrl) return fail(NLB_ERR_ARG, "null problem/state");
    if (P->p <= 0 || P->h <= 0 || P->n_channels < 0) return fail(NLB_ERR_SIZE, "bad p/h/channels");
    if (S->dtype != NLB_F64 && S->dtype != NLB_F32) return fail(NLB_ERR_ARG, "dtype must be NLB_F64 or NLB_F32");
    if (!S->t1[0] || !S->t1[1] || !S->prep) return fail(NLB_ERR_ARG, "null t1/prep buffer");
    if (P->n_t2 > 0 && (!S->t2[0] || !S->t2[1] || !S->g)) return fail(NLB_ERR_ARG, "null t2/g buffer");
    return NLB_OK;
}

template <typename T>
int step_t(const nlb_struct_problem* P, const nlb_struct_state* S, cudaStream_t st) {
    const int64_t nprep = (int64_t)P->h * P->h + P->p;
    k_prep<<<(unsigned)((nprep + kThreads - 1) / kThreads), kThreads, 0, st>>>(*P, *S);
    if (P->n_t2 > 0) {
        k_gterms<T><<<grid_for(k_gterms<T>, P->n_g), kThreads, 0, st>>>(*P, *S);
        k_t2_update<T><<<grid_for(k_t2_update<T>, P->n_t2), kThreads, 0, st>>>(*P, *S);
    }
    k_t1_update<T><<<grid_for(k_t1_update<T>, (int64_t)P->p * P->h), kThreads, 0, st>>>(*P, *S);
    k_finish<<<1, 32, 0, st>>>(S->ctrl);
    return check_launch("nlb_struct_step");
}

template <typename T>
int diis_t(const nlb_struct_problem* P, const nlb_struct_state* S, cudaStream_t st) {
    const int64_t n = (int64_t)P->p * P->h + P->n_t2;
    k_diis_gram<T><<<grid_for(k_diis_gram<T>, n), kThreads, 0, st>>>(*P, *S);
    k_diis_solve<<<1, 32, 0, st>>>(S->ctrl);
    k_diis_extrap<T><<<grid_for(k_diis_extrap<T>, n), kThreads, 0, st>>>(*P, *S);
    k_diis_done<<<1, 32, 0, st>>>(S->ctrl);
    return check_launch("nlb_struct_diis");
}

}  // namespace

extern "C" {

int nlb_version(void) { return 1; }

const char* nlb_last_error(void) { return g_err; }

int64_t nlb_struct_prep_len(int32_t p, int32_t h) { return 3 * (int64_t)h * h + 2 * (int64_t)p; }

int nlb_struct_ctrl_init(nlb_ctrl* ctrl, double eps, double mixing, int32_t max_steps, int32_t criterion,
                         int32_t max_diis, int32_t ccs, double e0, nlb_stream_t stream) {
    if (!ctrl) return fail(NLB_ERR_ARG, "null ctrl");
    if (max_diis < 0 || max_diis > kMaxDiis) return fail(NLB_ERR_ARG, "max_diis must be in [0, 10]");
    if (criterion != NLB_CRIT_SOA && criterion != NLB_CRIT_NUMPY) return fail(NLB_ERR_ARG, "bad criterion");
    k_ctrl_init<<<1, 32, 0, (cudaStream_t)stream>>>(ctrl, eps, mixing, max_steps, criterion, max_diis, ccs, e0);
    return check_launch("nlb_struct_ctrl_init");
}

int nlb_struct_step(const nlb_struct_problem* prob, const nlb_struct_state* st, nlb_stream_t stream) {
    int rc = valid(prob, st);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    return st->dtype == NLB_F64 ? step_t<double>(prob, st, s) : step_t<float>(prob, st, s);
}

int nlb_struct_diis(const nlb_struct_problem* prob, const nlb_struct_state* st, nlb_stream_t stream) {
    int rc = valid(prob, st);
    if (rc) return rc;
    if (!st->diis_t1 || (prob->n_t2 > 0 && !st->diis_t2)) return fail(NLB_ERR_ARG, "null DIIS ring");
    cudaStream_t s = (cudaStream_t)stream;
    return st->dtype == NLB_F64 ? diis_t<double>(prob, st, s) : diis_t<float>(prob, st, s);
}

int nlb_struct_energy(const nlb_struct_problem* prob, const nlb_struct_state* st, double* e_out,
                      nlb_stream_t stream) {
    int rc = valid(prob, st);
    if (rc) return rc;
    if (!e_out) return fail(NLB_ERR_ARG, "null e_out");
    cudaStream_t s = (cudaStream_t)stream;
    k_zero1<<<1, 1, 0, s>>>(e_out);
    k_energy<<<grid_for(k_energy, (int64_t)prob->p * prob->h), kThreads, 0, s>>>(*prob, *st, e_out);
    return check_launch("nlb_struct_energy");
}

int nlb_convert(const void* src, int32_t src_dtype, void* dst, int32_t dst_dtype, int64_t n,
                nlb_stream_t stream) {
    if (!src || !dst || n < 0) return fail(NLB_ERR_ARG, "bad convert args");
    if (n == 0) return NLB_OK;
    cudaStream_t s = (cudaStream_t)stream;
    const int grid = (int)((n + kThreads - 1) / kThreads < 4096 ? (n + kThreads - 1) / kThreads : 4096);
    if (src_dtype == NLB_F64 && dst_dtype == NLB_F32)
        k_convert<double, float><<<grid, kThreads, 0, s>>>((const double*)src, (float*)dst, n);
    else if (src_dtype == NLB_F32 && dst_dtype == NLB_F64)
        k_convert<float, double><<<grid, kThreads, 0, s>>>((const float*)src, (double*)dst, n);
    else if (src_dtype == NLB_F64 && dst_dtype == NLB_F64)
        k_convert<double, double><<<grid, kThreads, 0, s>>>((const double*)src, (double*)dst, n);
    else if (src_dtype == NLB_F32 && dst_dtype == NLB_F32)
        k_convert<float, float><<<grid, kThreads, 0, s>>>((const float*)src, (float*)dst, n);
    else
        return fail(NLB_ERR_ARG, "bad dtype");
    return check_launch("nlb_convert");
}

int nlb_struct_unpack_t2(const nlb_struct_problem* prob, const void* t2c, int32_t dtype, double* t2_dense,
                         nlb_stream_t stream) {
    if (!prob || !t2c || !t2_dense) return fail(NLB_ERR_ARG, "null unpack args");
    if (prob->n_t2 == 0) return NLB_OK;
    cudaStream_t s = (cudaStream_t)stream;
    const int grid = (int)((prob->n_t2 + kThreads - 1) / kThreads < 8192 ? (prob->n_t2 + kThreads - 1) / kThreads : 8192);
    if (dtype == NLB_F64) k_unpack<double><<<grid, kThreads, 0, s>>>(*prob, (const double*)t2c, t2_dense);
    else if (dtype == NLB_F32) k_unpack<float><<<grid, kThreads, 0, s>>>(*prob, (const float*)t2c, t2_dense);
    else return fail(NLB_ERR_ARG, "bad dtype");
    return check_launch("nlb_struct_unpack_t2");
}

int nlb_struct_pack_t2(const nlb_struct_problem* prob, const double* t2_dense, void* t2c, int32_t dtype,
                       nlb_stream_t stream) {
    if (!prob || !t2c || !t2_dense) return fail(NLB_ERR_ARG, "null pack args");
    if (prob->n_t2 == 0) return NLB_OK;
    cudaStream_t s = (cudaStream_t)stream;
    const int grid = (int)((prob->n_t2 + kThreads - 1) / kThreads < 8192 ? (prob->n_t2 + kThreads - 1) / kThreads : 8192);
    if (dtype == NLB_F64) k_pack<double><<<grid, kThreads, 0, s>>>(*prob, t2_dense, (double*)t2c);
    else if (dtype == NLB_F32) k_pack<float><<<grid, kThreads, 0, s>>>(*prob, t2_dense, (float*)t2c);
    else return fail(NLB_ERR_ARG, "bad dtype");
    return check_launch("nlb_struct_pack_t2");
}

}  // extern "C"
