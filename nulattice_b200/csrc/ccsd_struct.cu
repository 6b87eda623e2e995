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

void nlb_internal_set_error(const char* msg) { snprintf(g_err, sizeof(g_err), "%s", msg); }

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

#include "common.cuh"
constexpr int kRowThreads = 256;   // T2 row kernel

// ----------------------------------------------------------- prep + Ga ----
// Ga[k'][b'][i'j'] = sum_c f_ck B[c'][b'][i'j']  (k = hole k' of label g1):
// the f_ph^T t2 half-contraction along the first particle index.  With t1 it
// gives the rank-h part of X_pp t2 along a, and it holds the T1 Fock term
// f_ck t2_acik for particles of label g2.
// The dressed-Fock tables (from t1) and Ga (from t2) in one launch: they
// read different amplitudes and are independent.  The first n_channels *
// max_nh * gx blocks each take one chunk of a Ga row (channel, hole k'),
// read its f_ph column list once and stream the chunk coalesced, four
// elements per thread; the blocks after them form the dressed-Fock tables.
constexpr int kGaVec = 4;    // Ga elements per thread

template <typename T>
__global__ void __launch_bounds__(kThreads) k_prep_ga(nlb_struct_problem P, nlb_struct_state S, int64_t nprep,
                                                      int gx) {
    const nlb_ctrl* c = S.ctrl;
    if (c->status != NLB_RUNNING) return;
    const int64_t nga_blocks = (c->ccs || P.n_t2 == 0) ? 0 : (int64_t)P.n_channels * P.max_nh * gx;
    const int64_t all_ga = (int64_t)P.n_channels * P.max_nh * gx;
    if ((int64_t)blockIdx.x >= all_ga) {
        const double* t1 = S.t1[c->parity];
        const int64_t nb = gridDim.x - all_ga;
        for (int64_t u = ((int64_t)blockIdx.x - all_ga) * blockDim.x + threadIdx.x; u < nprep; u += nb * blockDim.x)
            prep_body(P, t1, S.prep, u);
        return;
    }
    if ((int64_t)blockIdx.x >= nga_blocks) return;
    const int yr = blockIdx.x / gx, bx = blockIdx.x - yr * gx;
    const int ci = yr / P.max_nh, kq = yr - ci * P.max_nh;
    const nlb_channel& ch = P.chan[ci];
    if (kq >= ch.nh1) return;
    const int rowlen = ch.np2 * ch.nh1 * ch.nh2;
    const int row = ch.hb1 + kq;
    const int q0 = P.fph_ptr[row], q1 = P.fph_ptr[row + 1];
    const T* __restrict__ Bc = static_cast<const T*>(S.t2[c->parity]) + ch.offset;
    // Ga layout per channel: [b'][k'][i'j'] (the k' values of one (b', i'j')
    // one hole-pair stride apart, so a reader needs one address per b')
    const int nhp = ch.nh1 * ch.nh2;
    T* __restrict__ Gr = static_cast<T*>(S.g) + ch.ga_off + (int64_t)kq * nhp;
    // Ga[k'][e] = sum_c f_ck B[c'][e], the f_ph entries of hole k in order
    constexpr int QR = 8;    // entries kept in registers (a lattice hole has at most six)
    T fv[QR];
    int64_t fo[QR];
#pragma unroll
    for (int u = 0; u < QR; ++u) {
        fv[u] = (q0 + u < q1) ? (T)P.fph_val[q0 + u] : T(0);
        fo[u] = (q0 + u < q1) ? (int64_t)P.fph_col[q0 + u] * rowlen : 0;
    }
    const int nq = q1 - q0;
    const int step = gx * blockDim.x * kGaVec;
    for (int e0 = bx * blockDim.x * kGaVec + threadIdx.x; e0 < rowlen; e0 += step) {
        T v[kGaVec];
#pragma unroll
        for (int r = 0; r < kGaVec; ++r) {
            const int e = e0 + r * (int)blockDim.x;
            T acc = T(0);
            if (e < rowlen) {
#pragma unroll
                for (int u = 0; u < QR; ++u)
                    if (u < nq) acc += fv[u] * Bc[fo[u] + e];
                for (int q = q0 + QR; q < q1; ++q)
                    acc += (T)P.fph_val[q] * Bc[(int64_t)P.fph_col[q] * rowlen + e];
            }
            v[r] = acc;
        }
#pragma unroll
        for (int r = 0; r < kGaVec; ++r) {
            const int e = e0 + r * (int)blockDim.x;
            if (e < rowlen) {
                const int bq = e / nhp;
                Gr[(int64_t)bq * (ch.nh1 - 1) * nhp + e] = v[r];   // (bq * nh1 + kq) * nhp + e % nhp
            }
        }
    }
}


// --------------------------------------------------------- T2 update ----
// One block per row task (channel, a').  The row B[a'][:][:] is staged in
// shared memory; everything along b, i and j reads it from there.  Only the
// terms along a (f_pp neighbours of a' and the Ga rows) read other rows,
// which sit in L2.  Per row the block also forms Gb[k'][i'j'] = sum_c f_ck
// B[a'][c'][i'j'] (rank-h part of X_pp along b) and the T1 Fock term
// F2[a'][i'] = sum_k' Gb[k'][i'k'].
//
// A thread owns work items (b', i') and walks j' (NH > 0: every label has NH
// holes, the j' loop is unrolled and the per-item lists live in registers;
// NH == 0: any hole counts).
constexpr int kMaxNb = 8;   // stencil entries kept in registers (lattice: <= 7)

template <typename T, int NH>
__global__ void __launch_bounds__(kRowThreads, 2) k_t2_rows(nlb_struct_problem P, nlb_struct_state S) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const nlb_ctrl* c = S.ctrl;
    if (c->status != NLB_RUNNING || c->ccs) return;
    const int par = c->parity;
    const T* __restrict__ B = static_cast<const T*>(S.t2[par]);
    T* __restrict__ Bo = static_cast<T*>(S.t2[par ^ 1]);
    const T* __restrict__ Ga = static_cast<const T*>(S.g);
    T* __restrict__ F2 = static_cast<T*>(S.f2);
    const PrepView V = prep_view(S.prep, P);
    T* E2 = (S.diis_t2 != nullptr && c->max_diis > 0 && c->diis_count < c->max_diis)
                ? static_cast<T*>(S.diis_t2) + (int64_t)c->diis_count * P.n_t2 : nullptr;
    const T m = (T)c->mixing, om = (T)(1.0 - c->mixing);
    const int mh = P.max_nh;
    const bool diag_lad = NH > 0 && P.diag_ladders;
    T* srow = reinterpret_cast<T*>(smem_raw);   // [max_row]  the row B[a']
    T* sacc = srow + P.max_row;                 // [max_row]  terms along a
    T* sgb = sacc + P.max_row;                  // [max_nh^3] Gb
    T* sx1 = sgb + mh * mh * mh;                // [max_nh^2] X_hh of label g1
    T* sx2 = sx1 + mh * mh;                     // [max_nh^2] X_hh of label g2
    T* st1a = sx2 + mh * mh;                    // [max_nh]   t1[a, H_g1]
    T* shh = st1a + mh;                         // [max_nh^2] diagonal hole-hole ladder
    T* sdh2 = shh + mh * mh;                    // [max_nh]   diag X_hh of label g2
    double nrm = 0.0;
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int64_t task = blockIdx.x; task < P.n_rows; task += gridDim.x) {
        const int ci = find_seg(P.row_end, P.n_channels, task);
        const nlb_channel& ch = P.chan[ci];
        const int ap = (int)(task - (ci ? P.row_end[ci - 1] : 0));
        const int nh1 = NH ? NH : ch.nh1, nh2 = NH ? NH : ch.nh2, np2 = ch.np2;
        const int nhp = nh1 * nh2;
        const int rowlen = np2 * nhp;
        const int64_t rbase = ch.offset + (int64_t)ap * rowlen;
        const T* __restrict__ Brow = B + rbase;
        const int32_t* hptr = P.hh_ptr + ch.hh_ptr_off;
        const int32_t* hcol = P.hh_col + ch.hh_col_off;
        const double* hval = P.hh_val + ch.hh_col_off;
        const int32_t* pptr = P.pp_ptr + ch.pp_ptr_off;
        const int32_t* pcol = P.pp_col + ch.pp_col_off;
        const double* pval = P.pp_val + ch.pp_col_off;
        for (int e = tid; e < rowlen; e += nt) srow[e] = Brow[e];
        const int x1b = P.xc_base[ch.g1], x2b = P.xc_base[ch.g2];
        for (int e = tid; e < nh1 * nh1; e += nt) sx1[e] = (T)V.xc[x1b + e];
        for (int e = tid; e < nh2 * nh2; e += nt) sx2[e] = (T)V.xc[x2b + e];
        const int t1a_b = P.t1c_base[ch.g1] + ap * nh1;
        for (int e = tid; e < nh1; e += nt) st1a[e] = (T)V.t1c[t1a_b + e];
        for (int e = tid; e < nh2; e += nt) sdh2[e] = (T)V.dhc[ch.hb2 + e];
        if (diag_lad)
            for (int e = tid; e < nhp; e += nt) shh[e] = (hptr[e + 1] > hptr[e]) ? (T)hval[hptr[e]] : T(0);
        __syncthreads();
        // Gb[k'][hp] = sum_c f_ck B[a'][c'][hp] for the holes k of label g2
        for (int e = tid; e < nh2 * nhp; e += nt) {
            const int kq = e / nhp, hp = e - kq * nhp;
            const int row = ch.hb2 + kq;
            T acc = T(0);
            for (int q = P.fph_ptr[row]; q < P.fph_ptr[row + 1]; ++q)
                acc += (T)P.fph_val[q] * srow[P.fph_col[q] * nhp + hp];
            sgb[e] = acc;
        }
        // Phase A (one thread per element, coalesced): the terms along a,
        // f_pp neighbours of a' in other rows and -t1_ak Ga[k'].
        const T* __restrict__ Gac = Ga + ch.ga_off;
        const T* __restrict__ Bch = B + ch.offset;
        {
            const int ra0 = P.fpp_ptr[ch.pb1 + ap], ra1 = P.fpp_ptr[ch.pb1 + ap + 1];
            const int na = min(ra1 - ra0, kMaxNb);
            int acol[kMaxNb];
            T aval[kMaxNb];
#pragma unroll
            for (int q = 0; q < kMaxNb; ++q) {
                acol[q] = q < na ? P.fpp_col[ra0 + q] : ap;
                aval[q] = q < na ? (T)P.fpp_val[ra0 + q] : T(0);
            }
            __syncthreads();  // st1a / srow visible
            for (int e = tid; e < rowlen; e += nt) {
                T acc = T(0);
#pragma unroll
                for (int q = 0; q < kMaxNb; ++q)
                    acc += aval[q] * ((acol[q] == ap) ? srow[e] : Bch[(int64_t)acol[q] * rowlen + e]);
                for (int q = ra0 + kMaxNb; q < ra1; ++q) {
                    const int col = P.fpp_col[q];
                    acc += (T)P.fpp_val[q] * ((col == ap) ? srow[e] : Bch[(int64_t)col * rowlen + e]);
                }
                // Ga[b'][k'][i'j'] of element e = b' * nhp + i'j'
                const T* ge = Gac + (int64_t)(e / nhp) * (nh1 - 1) * nhp + e;
                if (NH) {
#pragma unroll
                    for (int k = 0; k < (NH ? NH : 1); ++k) acc -= st1a[k] * ge[k * nhp];
                } else {
                    for (int k = 0; k < nh1; ++k) acc -= st1a[k] * ge[k * nhp];
                }
                sacc[e] = acc;
            }
        }
        __syncthreads();
        for (int iq = tid; iq < nh1; iq += nt) {
            T acc = T(0);
            for (int kq = 0; kq < nh2; ++kq) acc += sgb[kq * nhp + iq * nh2 + kq];
            F2[ch.f2_off + (int64_t)ap * nh1 + iq] = acc;
        }
        const double da = V.dpc[ch.pb1 + ap];
        const int t1b_b = P.t1c_base[ch.g2];
        if (diag_lad) {
            // Phase B, fixed hole count and diagonal ladders: a thread owns (b', i')
            // and keeps the j' vector in registers.
            constexpr int NHc = NH ? NH : 1;
            constexpr int NHP = NHc * NHc;
            for (int w = tid; w < np2 * NHc; w += nt) {
                const int bp = w / NHc, ip = w - bp * NHc;
                const int base = bp * NHP + ip * NHc;
                T r[NHc], R[NHc], t1b[NHc];
#pragma unroll
                for (int j = 0; j < NHc; ++j) {
                    r[j] = srow[base + j];
                    R[j] = sacc[base + j];
                    t1b[j] = (T)V.t1c[t1b_b + bp * NHc + j];
                }
                // f_pp along b
                const int rbi = ch.pb2 + bp;
                const int rb0 = P.fpp_ptr[rbi], rb1 = P.fpp_ptr[rbi + 1];
                for (int q = rb0; q < rb1; ++q) {
                    const T v = (T)P.fpp_val[q];
                    const T* src = srow + P.fpp_col[q] * NHP + ip * NHc;
#pragma unroll
                    for (int j = 0; j < NHc; ++j) R[j] += v * src[j];
                }
                // rank-h part of X_pp along b
#pragma unroll
                for (int k = 0; k < NHc; ++k) {
                    const T t = t1b[k];
                    const T* g = sgb + k * NHP + ip * NHc;
#pragma unroll
                    for (int j = 0; j < NHc; ++j) R[j] -= t * g[j];
                }
                // X_hh along i (other i' of the same b') and along j (registers)
#pragma unroll
                for (int k = 0; k < NHc; ++k) {
                    const T xk = sx1[k * NHc + ip];
                    const T* src = srow + bp * NHP + k * NHc;
#pragma unroll
                    for (int j = 0; j < NHc; ++j) R[j] += xk * src[j];
                }
#pragma unroll
                for (int j = 0; j < NHc; ++j) {
                    T acc = T(0);
#pragma unroll
                    for (int k = 0; k < NHc; ++k) acc += sx2[k * NHc + j] * r[k];
                    R[j] += acc;
                }
                // both ladders are diagonal and act on tau = t2 + t1 t1
                const int ab = ap * np2 + bp;
                const int q0 = pptr[ab];
                const T cpp = (pptr[ab + 1] > q0) ? (T)pval[q0] : T(0);
                const T ta = st1a[ip];
                const double dpart = da + V.dpc[ch.pb2 + bp];
                const double dhi = V.dhc[ch.hb1 + ip];
#pragma unroll
                for (int j = 0; j < NHc; ++j) {
                    const T tau = r[j] + ta * t1b[j];
                    R[j] += (shh[ip * NHc + j] + cpp) * tau;
                    const double dd = -(dpart + (dhi + (double)sdh2[j]));
                    const T tn = r[j] + R[j] / (T)dd;
                    const T out = m * r[j] + om * tn;
                    Bo[rbase + base + j] = out;
                    const T d = out - r[j];
                    if (E2) E2[rbase + base + j] = d;
                    nrm += (double)d * (double)d;
                }
            }
        } else {
            // Phase B, general: any hole count, ladders from their CSR lists.
            for (int w = tid; w < np2 * nh1; w += nt) {
                const int bp = w / nh1, ip = w - bp * nh1;
                const int base = bp * nhp + ip * nh2;
                const int rbi = ch.pb2 + bp;
                const int rb0 = P.fpp_ptr[rbi], rb1 = P.fpp_ptr[rbi + 1];
                const double dab = da + V.dpc[ch.pb2 + bp];
                const double dhi = V.dhc[ch.hb1 + ip];
                const int ab = ap * np2 + bp;
                const int p0 = pptr[ab], p1 = pptr[ab + 1];
                for (int jp = 0; jp < nh2; ++jp) {
                    const int hp = ip * nh2 + jp;
                    const int e = base + jp;
                    const T x = srow[e];
                    T R = sacc[e];
                    for (int q = rb0; q < rb1; ++q) R += (T)P.fpp_val[q] * srow[P.fpp_col[q] * nhp + hp];
                    for (int k = 0; k < nh2; ++k) R -= (T)V.t1c[t1b_b + bp * nh2 + k] * sgb[k * nhp + hp];
                    for (int k = 0; k < nh1; ++k) R += sx1[k * nh1 + ip] * srow[bp * nhp + k * nh2 + jp];
                    for (int k = 0; k < nh2; ++k) R += sx2[k * nh2 + jp] * srow[base + k];
                    for (int q = hptr[hp]; q < hptr[hp + 1]; ++q) {
                        const int in = hcol[q];
                        const int kq = in / nh2, lq = in - kq * nh2;
                        const T tl = (T)V.t1c[t1b_b + bp * nh2 + lq];
                        R += (T)hval[q] * (srow[bp * nhp + in] + st1a[kq] * tl);
                    }
                    for (int q = p0; q < p1; ++q) {
                        const int in = pcol[q];
                        const int cq = in / np2, dq = in - cq * np2;
                        const T bin = (in == ab) ? x : Bch[(int64_t)in * nhp + hp];
                        const double tt =
                            V.t1c[P.t1c_base[ch.g1] + cq * nh1 + ip] * V.t1c[t1b_b + dq * nh2 + jp];
                        R += (T)pval[q] * (bin + (T)tt);
                    }
                    const double dd = -(dab + (dhi + V.dhc[ch.hb2 + jp]));
                    const T tn = x + R / (T)dd;
                    const T out = m * x + om * tn;
                    Bo[rbase + e] = out;
                    const T d = out - x;
                    if (E2) E2[rbase + e] = d;
                    nrm += (double)d * (double)d;
                }
            }
        }
        __syncthreads();
    }
    const double s = block_sum(nrm);
    if (threadIdx.x == 0) V.slots(kRedDt2)[blockIdx.x] = 4.0 * s;
}

// ------------------------------------------------ T2 update, lattice path ----
// Closed-site lattice inputs: every label has NH holes and both ladders only
// couple a pair to itself.  Same residual as k_t2_rows, organised so that one
// pass over the row does everything, coalesced over the row:
//
// * the block is NB = NT / NH^2 groups of NH^2 threads; a thread keeps one
//   hole pair (i', j') for the whole row and its group walks b' = q, q + NB,
//   ..., so the X_hh columns of i' and j', the hole-hole ladder entry and the
//   hole part of the denominator are registers;
// * rows arrive in shared memory by cp.async (16-byte copies for the aligned
//   middle, element copies for the ragged ends), double-buffered: the next
//   row is in flight while the block works on the current one;
// * per-b' data sits next to the row in 32-byte records read with vector
//   loads: t1[b', H_g2] and the particle-particle ladder entry of (a', b'),
//   the f_pp row of b' as pre-scaled offsets and values;
// * the terms along a (f_pp neighbours of a' and the Ga rows) are read from
//   L2 with one coalesced load per term, issued one b' step ahead; the
//   neighbour rows of consecutive a' overlap because each block takes a
//   contiguous range of rows;
// * the rows' b' columns are split evenly over the blocks, so a block may
//   start or end inside a row (1254 rows on 148 blocks at L=6 would
//   otherwise leave some blocks nine rows and others eight).
//
// Launched only when every f_pp row has at most kLatNa off-diagonal entries
// (max_fpp_offdiag), so the f_pp row of b' with its diagonal fits the
// kLatNb - 1 used slots of its record.
constexpr int kLatNb = 8;    // record slots per b' (at most 7 used)
constexpr int kLatNa = 6;    // off-diagonal f_pp entries of a' kept in registers

struct LatSmem {
    int64_t row0, row1, gb, rec, dp, off, val, total;
};

// Shared-memory layout of k_t2_lat for element size el and NH holes per label
// (pair: the per-b' record holds 8 (f_pp value, t1) pairs instead of 8 t1).
__host__ __device__ inline LatSmem lat_smem(int64_t max_row, int nh, int64_t el, bool pair = false) {
    const int64_t np2 = max_row / (nh * nh);
    const int64_t rowb = lat_round16(el * (max_row + 16 / el + 4));
    LatSmem s;
    s.row0 = 0;
    s.row1 = rowb;
    s.gb = 2 * rowb;
    s.rec = s.gb + lat_round16(el * nh * nh * nh);
    s.dp = s.rec + lat_round16(el * np2 * kLatNb * (pair ? 2 : 1));
    s.off = s.dp + lat_round16(el * np2);
    s.val = s.off + lat_round16(4 * np2 * kLatNb);
    s.total = s.val + lat_round16(el * np2 * kLatNb);
    return s;
}

// Queue the asynchronous copy of the row starting at `src` (rowlen elements)
// into the buffer `dst`; returns the element shift that makes the 16-byte
// copies aligned on both sides.
template <typename T, int NT>
__device__ __forceinline__ int lat_issue_row(T* dst, const T* src, int rowlen) {
    constexpr int VEC = 16 / (int)sizeof(T);
    const int mis = (int)((reinterpret_cast<uintptr_t>(src) / sizeof(T)) & (VEC - 1));
    T* d = dst + mis;
    const int head = min((VEC - mis) & (VEC - 1), rowlen);
    const int nvec = (rowlen - head) / VEC;
    const int tail0 = head + nvec * VEC;
    for (int e = threadIdx.x; e < head; e += NT) cp_async_el<sizeof(T)>(d + e, src + e);
    for (int v = threadIdx.x; v < nvec; v += NT) cp_async16(d + head + v * VEC, src + head + v * VEC);
    for (int e = tail0 + threadIdx.x; e < rowlen; e += NT) cp_async_el<sizeof(T)>(d + e, src + e);
    cp_async_commit();
    return mis;
}

//
// PAIR (FP32 only): the three pairs of independent sums (along b / rank-h
// along b, X_hh along i / along j, along a / rank-h along a) run as packed
// FP32x2 fused multiply-adds, with the f_pp values and t1 of b' interleaved
// in the per-b' record so that each coefficient pair is one register pair.
template <typename T, int NH, int NT, int MINB, bool PAIR = false>
__global__ void __launch_bounds__(NT, MINB) k_t2_lat(nlb_struct_problem P, nlb_struct_state S) {
    static_assert(!PAIR || sizeof(T) == 4, "packed pairs are FP32x2");
    constexpr int NHP = NH * NH;
    constexpr int NB = NT / NHP;
    static_assert(NB >= 1 && NH <= 7, "block must hold one hole-pair group; a record holds 7 holes");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const nlb_ctrl* c = S.ctrl;
    if (c->status != NLB_RUNNING || c->ccs) return;
    const int par = c->parity;
    const T* __restrict__ B = static_cast<const T*>(S.t2[par]);
    T* __restrict__ Bo = static_cast<T*>(S.t2[par ^ 1]);
    const T* __restrict__ Ga = static_cast<const T*>(S.g);
    T* __restrict__ F2 = static_cast<T*>(S.f2);
    const PrepView V = prep_view(S.prep, P);
    T* E2 = (S.diis_t2 != nullptr && c->max_diis > 0 && c->diis_count < c->max_diis)
                ? static_cast<T*>(S.diis_t2) + (int64_t)c->diis_count * P.n_t2 : nullptr;
    const T m = (T)c->mixing, om = (T)(1.0 - c->mixing);
    const LatSmem L = lat_smem(P.max_row, NH, sizeof(T), PAIR);
    T* sgb = reinterpret_cast<T*>(smem_raw + L.gb);        // Gb[k'][i'j'] of this row
    // [b'][8]: t1[b', k'] (k' < NH), pp ladder at 7; PAIR: [b'][8][2] (f_pp value, t1[b', k']),
    // pp ladder at [7][1]
    T* srec = reinterpret_cast<T*>(smem_raw + L.rec);
    constexpr int RW = PAIR ? 2 * kLatNb : kLatNb;         // record width
    T* sdp = reinterpret_cast<T*>(smem_raw + L.dp);        // [b']: particle part of the denominator
    int32_t* soff = reinterpret_cast<int32_t*>(smem_raw + L.off);   // [b'][8] f_pp columns * NH^2
    T* sval = reinterpret_cast<T*>(smem_raw + L.val);      // [b'][8] f_pp values (0 = padding)

    const int tid = threadIdx.x;
    const bool active = tid < NB * NHP;
    const int grp = tid / NHP, hp = tid - grp * NHP;
    const int ip = hp / NH, jp = hp - ip * NH;
    double nrm = 0.0;
    int cur_ci = -1;
    T x1[NH], x2[NH], hh = T(0), dh = T(0);
    float2 x12[NH];   // PAIR: (x1[k], x2[k])

    // work units: max(np2, 1) b' columns per row, rows in channel order, cut
    // into gridDim.x equal contiguous ranges [w0, w1) (a block may start or
    // end inside a row: it stages the row and forms Gb, updates the columns
    // of its range, and the block holding column 0 writes the row's F2);
    // W is below 2^31 because the lattice path holds a row in shared memory
    int64_t W = 0;
    for (int cc = 0; cc < P.n_channels; ++cc) W += lat_units(P, cc);
    const int w0 = (int)((int64_t)blockIdx.x * W / gridDim.x);
    const int w1 = (int)((int64_t)(blockIdx.x + 1) * W / gridDim.x);
    int ci = 0, ap = 0, blo = 0, wc = 0;
    auto issue = [&](int cc, int a, int stage) {
        const nlb_channel& cn = P.chan[cc];
        const int rl = cn.np2 * NHP;
        return lat_issue_row<T, NT>(reinterpret_cast<T*>(smem_raw + (stage ? L.row1 : L.row0)),
                                    B + cn.offset + (int64_t)a * rl, rl);
    };
    int mis = 0;
    if (w0 < w1) {
        while (wc + lat_units(P, ci) <= w0) wc += (int)lat_units(P, ci++);
        const int u = P.chan[ci].np2 > 0 ? P.chan[ci].np2 : 1;
        ap = (w0 - wc) / u;
        blo = w0 - wc - ap * u;
        mis = issue(ci, ap, 0);
    }
    for (int pass = 0; w0 < w1; ++pass) {
        const int buf = pass & 1;
        const nlb_channel& ch = P.chan[ci];
        const int np2 = ch.np2;
        const int rowlen = np2 * NHP;
        const int upp = np2 > 0 ? np2 : 1;                      // units per row
        const int wp = wc + ap * upp;                           // first unit of this row
        const int bhi = w1 - wp < np2 ? w1 - wp : np2;          // b' columns [blo, bhi)
        const int64_t rbase = ch.offset + (int64_t)ap * rowlen;
        // (shared addresses computed from smem_raw directly, never through a
        // pointer array, so that every access stays a shared-memory access)
        const T* srow = reinterpret_cast<const T*>(smem_raw + (buf ? L.row1 : L.row0)) + mis;

        // per-channel tables (the block's rows are contiguous: usually unchanged)
        if (ci != cur_ci) {
            cur_ci = ci;
            const int x1b = P.xc_base[ch.g1], x2b = P.xc_base[ch.g2];
#pragma unroll
            for (int k = 0; k < NH; ++k) {
                x1[k] = (T)V.xc[x1b + k * NH + ip];
                x2[k] = (T)V.xc[x2b + k * NH + jp];
                x12[k] = make_float2((float)x1[k], (float)x2[k]);
            }
            const int32_t* hptr = P.hh_ptr + ch.hh_ptr_off;
            hh = (hptr[hp + 1] > hptr[hp]) ? (T)P.hh_val[ch.hh_col_off + hptr[hp]] : T(0);
            dh = (T)(V.dhc[ch.hb1 + ip] + V.dhc[ch.hb2 + jp]);
            const int t1b_b = P.t1c_base[ch.g2];
            for (int w = tid; w < np2 * kLatNb; w += NT) {
                const int bp = w / kLatNb, k = w - bp * kLatNb;
                const int r0 = P.fpp_ptr[ch.pb2 + bp], r1 = P.fpp_ptr[ch.pb2 + bp + 1];
                soff[w] = ((k < r1 - r0) ? P.fpp_col[r0 + k] : bp) * NHP;
                const T v = (k < r1 - r0) ? (T)P.fpp_val[r0 + k] : T(0);
                if constexpr (PAIR) {
                    srec[2 * w] = v;
                    if (k < NH) srec[2 * w + 1] = (T)V.t1c[t1b_b + bp * NH + k];
                } else {
                    if (k < NH) srec[w] = (T)V.t1c[t1b_b + bp * NH + k];
                    sval[w] = v;
                }
            }
        }
        // per-row: a' stencil (off-diagonal part in registers; unused slots
        // point at the row itself with weight 0), t1[a', H_g1], the pp ladder
        // entries and particle denominators of the pairs (a', b')
        const int ra0 = P.fpp_ptr[ch.pb1 + ap], ra1 = P.fpp_ptr[ch.pb1 + ap + 1];
        T adiag = T(0);
        int aoff[kLatNa];
        T aval[kLatNa];
        {
            int q = ra0;
#pragma unroll
            for (int s = 0; s < kLatNa; ++s) {
                aoff[s] = ap * rowlen;
                aval[s] = T(0);
                for (; q < ra1; ++q) {
                    const int col = P.fpp_col[q];
                    if (col == ap) { adiag += (T)P.fpp_val[q]; continue; }
                    aoff[s] = col * rowlen;
                    aval[s] = (T)P.fpp_val[q];
                    ++q;
                    break;
                }
            }
            for (; q < ra1; ++q)
                if (P.fpp_col[q] == ap) adiag += (T)P.fpp_val[q];
        }
        T t1a[NH];
        const int t1a_b = P.t1c_base[ch.g1] + ap * NH;
#pragma unroll
        for (int k = 0; k < NH; ++k) t1a[k] = (T)V.t1c[t1a_b + k];
        const T t1ai = (T)V.t1c[t1a_b + ip];
        const double da = V.dpc[ch.pb1 + ap];
        const int32_t* pptr = P.pp_ptr + ch.pp_ptr_off;
        const double* pval = P.pp_val + ch.pp_col_off;
        for (int bp = blo + tid; bp < bhi; bp += NT) {
            const int ab = ap * np2 + bp;
            srec[bp * RW + RW - 1] = (pptr[ab + 1] > pptr[ab]) ? (T)pval[pptr[ab]] : T(0);
            sdp[bp] = (T)(da + V.dpc[ch.pb2 + bp]);
        }
        cp_async_wait_all();
        __syncthreads();
        // next row in flight while this one is worked on (its buffer was last
        // read by the row before, which ended with a barrier)
        const bool more = wp + upp < w1;
        int nci = ci, nap = ap + 1, nwc = wc, next_mis = 0;
        if (more) {
            while (nap >= P.chan[nci].np1) {   // past the channel's last row
                nwc += (int)lat_units(P, nci++);
                nap = 0;
            }
            next_mis = issue(nci, nap, buf ^ 1);
        }
        // Gb[k'][hp] = sum_c f_ck B[a'][c'][hp] (holes k of label g2), then F2
        for (int e = tid; e < NH * NHP; e += NT) {
            const int kq = e / NHP, h2 = e - kq * NHP;
            const int row = ch.hb2 + kq;
            T acc = T(0);
            for (int q = P.fph_ptr[row]; q < P.fph_ptr[row + 1]; ++q)
                acc += (T)P.fph_val[q] * srow[P.fph_col[q] * NHP + h2];
            sgb[e] = acc;
        }
        __syncthreads();
        if (blo == 0 && tid < NH) {
            T acc = T(0);
#pragma unroll
            for (int kq = 0; kq < NH; ++kq) acc += sgb[kq * NHP + tid * NH + kq];
            F2[ch.f2_off + (int64_t)ap * NH + tid] = acc;
        }
        if (active && blo + grp < bhi) {
            const T* __restrict__ gB = B + ch.offset + hp;
            const T* __restrict__ gG = Ga + ch.ga_off + hp;    // Ga[b'][k'][i'j']: k' at stride NHP
            T* __restrict__ Bout = Bo + rbase + hp;
            T* __restrict__ Eout = E2 ? E2 + rbase + hp : nullptr;
            const T* s_hp = srow + hp;
            const T* s_col = srow + jp;          // B[b'][k'][j'] at eb + k' NH
            const T* s_row = srow + ip * NH;     // B[b'][i'][k'] at eb + k'
            const T* g_hp = sgb + hp;
            T nrm_row = T(0);
            // one element (b', i', j') given its terms along a
            auto element = [&](int bp, int eb, const T (&nb)[kLatNa], const T (&gv)[NH]) {
                const T x = s_hp[eb];
                if constexpr (PAIR) {
                    float2 pr[8];
                    int so[8];
                    {
                        const float* rp = reinterpret_cast<const float*>(srec) + bp * RW;
#pragma unroll
                        for (int u = 0; u < 4; ++u) {
                            const float4 f = *reinterpret_cast<const float4*>(rp + 4 * u);
                            pr[2 * u] = make_float2(f.x, f.y);
                            pr[2 * u + 1] = make_float2(f.z, f.w);
                        }
                    }
                    lds8(soff + bp * kLatNb, so);
                    // (f_pp along b, rank-h part along b)
                    float2 p1 = make_float2(0.f, 0.f);
#pragma unroll
                    for (int q = 0; q < kLatNb - 1; ++q)
                        p1 = __ffma2_rn(pr[q], make_float2(s_hp[so[q]], g_hp[q * NHP]), p1);
                    // (X_hh along i, X_hh along j)
                    float2 p2 = make_float2(0.f, 0.f);
#pragma unroll
                    for (int k = 0; k < NH; ++k)
                        p2 = __ffma2_rn(x12[k], make_float2(s_col[eb + k * NH], s_row[eb + k]), p2);
                    // (f_pp neighbours along a, rank-h part along a)
                    float2 p3 = make_float2(adiag * x, 0.f);
#pragma unroll
                    for (int q = 0; q < kLatNa; ++q)
                        p3 = __ffma2_rn(make_float2(aval[q], t1a[q]), make_float2(nb[q], gv[q]), p3);
#pragma unroll
                    for (int k = kLatNa; k < NH; ++k) p3.y = fmaf(t1a[k], gv[k], p3.y);
                    const T t1bj = srec[bp * RW + 2 * jp + 1];
                    const T lad = (hh + pr[7].y) * (x + t1ai * t1bj);
                    const T acc = ((p3.x - p3.y) + (p1.x - p1.y)) + ((p2.x + p2.y) + lad);
                    const T dd = -(sdp[bp] + dh);
                    const T tn = x + lat_div(acc, dd);
                    const T out = m * x + om * tn;
                    __stcg(Bout + eb, out);
                    const T d = out - x;
                    if (Eout) __stcg(Eout + eb, d);
                    nrm_row += d * d;
                    return;
                }
                T rec[8], sv[8];
                int so[8];
                lds8(srec + bp * kLatNb, rec);
                lds8(soff + bp * kLatNb, so);
                lds8(sval + bp * kLatNb, sv);
                // f_pp along b
                T accb = T(0);
#pragma unroll
                for (int q = 0; q < kLatNb - 1; ++q) accb += sv[q] * s_hp[so[q]];
                // rank-h part along b: -t1_bk Gb[k]
                T accg = T(0);
#pragma unroll
                for (int k = 0; k < NH; ++k) accg += rec[k] * g_hp[k * NHP];
                // X_hh along i and along j
                T accx = T(0), accy = T(0);
#pragma unroll
                for (int k = 0; k < NH; ++k) {
                    accx += x1[k] * s_col[eb + k * NH];
                    accy += x2[k] * s_row[eb + k];
                }
                // along a: f_pp neighbours and the rank-h part -t1_ak Ga[k]
                T acca = adiag * x, accG = T(0);
#pragma unroll
                for (int q = 0; q < kLatNa; ++q) acca += aval[q] * nb[q];
#pragma unroll
                for (int k = 0; k < NH; ++k) accG += t1a[k] * gv[k];
                // both ladders act on tau = t2 + t1 t1
                const T t1bj = srec[bp * kLatNb + jp];
                const T lad = (hh + rec[7]) * (x + t1ai * t1bj);
                const T acc = ((acca - accG) + (accb - accg)) + ((accx + accy) + lad);
                const T dd = -(sdp[bp] + dh);
                const T tn = x + lat_div(acc, dd);
                const T out = m * x + om * tn;
                __stcg(Bout + eb, out);
                const T d = out - x;
                if (Eout) __stcg(Eout + eb, d);
                nrm_row += d * d;
            };
            // the L2 loads of one b' step go out a step ahead of its math
            T rnb[kLatNa], rgv[NH];
            {
                const int eb = (blo + grp) * NHP;
#pragma unroll
                for (int q = 0; q < kLatNa; ++q) rnb[q] = __ldg(gB + aoff[q] + eb);
#pragma unroll
                for (int k = 0; k < NH; ++k) rgv[k] = __ldg(gG + eb * NH + k * NHP);
            }
            for (int bp = blo + grp; bp < bhi; bp += NB) {
                const int eb = bp * NHP;
                T nb[kLatNa], gv[NH];
#pragma unroll
                for (int q = 0; q < kLatNa; ++q) nb[q] = rnb[q];
#pragma unroll
                for (int k = 0; k < NH; ++k) gv[k] = rgv[k];
                const int ebn = (bp + NB < bhi) ? eb + NB * NHP : eb;
#pragma unroll
                for (int q = 0; q < kLatNa; ++q) rnb[q] = __ldg(gB + aoff[q] + ebn);
#pragma unroll
                for (int k = 0; k < NH; ++k) rgv[k] = __ldg(gG + ebn * NH + k * NHP);
                element(bp, eb, nb, gv);
            }
            nrm += (double)nrm_row;
        }
        __syncthreads();
        if (!more) break;
        ci = nci;
        ap = nap;
        wc = nwc;
        blo = 0;
        mis = next_mis;
    }
    const double s = block_sum(nrm);
    if (threadIdx.x == 0) V.slots(kRedDt2)[blockIdx.x] = 4.0 * s;
}

#include "t2_pair.cuh"

// --------------------------------------------------------- T1 update ----
// R1 = f_ph + F2 + f_pp t1 - t1 Q/2 + t1 X_hh(T1 eq); Jacobi + mixing;
// energy sum_ai f_ai t1'_ai (coupled_cluster.py:342-414, 265-286).
template <typename T>
__global__ void __launch_bounds__(kThreads) k_t1_update(nlb_struct_problem P, nlb_struct_state S) {
    // Sixteen lanes per amplitude t1[a, i] of matching labels (the others
    // are zero for label-conserving inputs and stay zero); the lanes share
    // the terms of its residual: the T2 Fock terms of the channels holding
    // the label (F2, or the Ga diagonal), the f_pp neighbours of a and the
    // hole mixing over the label's holes.
    nlb_ctrl* c = S.ctrl;
    if (c->status != NLB_RUNNING) return;
    const int par = c->parity;
    const double* t1 = S.t1[par];
    double* t1o = S.t1[par ^ 1];
    const int h = P.h, p = P.p;
    const PrepView V = prep_view(S.prep, P);
    const T* Ga = static_cast<const T*>(S.g);
    const T* F2 = static_cast<const T*>(S.f2);
    double* E1 = (S.diis_t1 != nullptr && c->max_diis > 0 && c->diis_count < c->max_diis)
                     ? S.diis_t1 + (int64_t)c->diis_count * p * h : nullptr;
    const double m = c->mixing;
    double eacc = 0.0, nrm = 0.0;
    const int64_t n = (int64_t)p * h;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += stride) {
        const int a = (int)(idx / h), i = (int)(idx - (int64_t)a * h);
        if (P.h_label[i] != P.p_label[a]) {
            t1o[idx] = 0.0;
            if (E1) E1[idx] = 0.0;
        }
    }
    // sixteen lanes per amplitude (two amplitudes per warp): every term of
    // its residual is an independent load, so one wave covers all of them
    const int lane = threadIdx.x & 15;
    const int64_t nhalf = stride >> 4;
    for (int64_t q0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 4;
         q0 - (((int64_t)threadIdx.x >> 4) & 1) < P.n_t1c; q0 += nhalf) {
        // both halves of a warp stay in the loop until neither has work
        const bool live = q0 < P.n_t1c;
        const int64_t q = live ? q0 : P.n_t1c - 1;
        int g, a, i, ap, ip;
        if (P.t1c_idx) {
            const int id = P.t1c_idx[q];
            a = id / h;
            i = id - a * h;
            g = P.p_label[a];
            ap = P.p_loc[a];
            ip = P.h_loc[i];
        } else {
            g = find_label(P.t1c_base, P.n_labels, q);
            const int nh_ = P.h_base[g + 1] - P.h_base[g];
            const int loc = (int)(q - P.t1c_base[g]);
            ap = loc / nh_;
            ip = loc - ap * nh_;
            a = P.p_ord[P.p_base[g] + ap];
            i = P.h_ord[P.h_base[g] + ip];
        }
        const int nh = P.h_base[g + 1] - P.h_base[g];
        const int pb = P.p_base[g];
        const int64_t idx = (int64_t)a * h + i;
        double part = 0.0;
        if (!c->ccs) {
            // channels in groups of four whose loads go out together (the
            // sum keeps the channel order)
            for (int c0 = 0; c0 < P.n_channels; c0 += 4) {
                double cp[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    cp[u] = 0.0;
                    if (c0 + u >= P.n_channels) continue;
                    const nlb_channel& ch = P.chan[c0 + u];
                    if (ch.g1 == g) {
                        if (lane == 0) cp[u] = (double)F2[ch.f2_off + (int64_t)ap * ch.nh1 + ip];
                    } else if (ch.g2 == g && lane < ch.nh1) {
                        const int nhp = ch.nh1 * ch.nh2;
                        cp[u] = (double)Ga[ch.ga_off + ((int64_t)ap * ch.nh1 + lane) * nhp + lane * ch.nh2 + ip];
                    }
                }
#pragma unroll
                for (int u = 0; u < 4; ++u) part += cp[u];
                // holes of a channel beyond the sixteen lanes
                for (int u = 0; u < 4 && c0 + u < P.n_channels; ++u) {
                    const nlb_channel& ch = P.chan[c0 + u];
                    if (ch.g1 != g && ch.g2 == g && ch.nh1 > 16) {
                        const int nhp = ch.nh1 * ch.nh2;
                        for (int k = lane + 16; k < ch.nh1; k += 16)
                            part += (double)Ga[ch.ga_off + ((int64_t)ap * ch.nh1 + k) * nhp + k * ch.nh2 + ip];
                    }
                }
            }
        }
        const int r = pb + ap;
        const int f0 = P.fpp_ptr[r], f1 = P.fpp_ptr[r + 1];
        for (int qq = f0 + lane; qq < f1; qq += 16) {
            const int c2 = P.fpp_prow ? P.fpp_prow[qq] : P.p_ord[pb + P.fpp_col[qq]];
            part += P.fpp_val[qq] * t1[(int64_t)c2 * h + i];
        }
        for (int kk = lane; kk < nh; kk += 16) {
            const int k = P.h_ord[P.h_base[g] + kk];
            part += t1[(int64_t)a * h + k] * (V.Xh1[(int64_t)k * h + i] - 0.5 * V.Q[(int64_t)k * h + i]);
        }
#pragma unroll
        for (int o = 8; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
        if (lane == 0 && live) {
            const double H1 = P.f_ph[idx] + part;
            const double D1 = -(V.dXp1[a] + V.Xh1[(int64_t)i * h + i]);
            const double x = t1[idx];
            const double tn = x + H1 / D1;
            const double out = m * x + (1.0 - m) * tn;
            t1o[idx] = out;
            const double d = out - x;
            if (E1) E1[idx] = d;
            nrm += d * d;
            eacc += P.f_ph[idx] * out;
        }
    }
    const double se = block_sum(eacc);
    const double sn = block_sum(nrm);
    if (threadIdx.x == 0) {
        V.slots(kRedE)[blockIdx.x] = se;
        V.slots(kRedDt1)[blockIdx.x] = sn;
    }
}

// -------------------------------------------------- convergence test ----
// One warp: the step's energy and norms from the per-block partials of the
// T1 (n1 blocks) and T2 (n2 blocks) launches, added in slot order.
// Launched with three warps: warp w adds one partial-sum array (energy, T1
// step, T2 step), each in the fixed order of warp_sum_slots.
__global__ void k_finish(nlb_ctrl* c, const double* red, int n1, int n2) {
    __shared__ double sums[3];
    if (blockIdx.x != 0) return;
    if (c->status != NLB_RUNNING) return;
    const int w = threadIdx.x >> 5;
    if (w == 0) sums[0] = warp_sum_slots(red + (int64_t)kRedE * kRedSlots, n1);
    else if (w == 1) sums[1] = warp_sum_slots(red + (int64_t)kRedDt1 * kRedSlots, n1);
    else if (w == 2) sums[2] = c->ccs ? 0.0 : warp_sum_slots(red + (int64_t)kRedDt2 * kRedSlots, n2);
    __syncthreads();
    if (threadIdx.x != 0) return;
    const double e_sum = sums[0], d1 = sums[1], d2 = sums[2];
    c->e_acc = e_sum;
    c->dt1_sq = d1;
    c->dt2_sq = d2;
    const double E = e_sum, prev = c->e_prev;
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
}


// ---------------------------------------------------------------- DIIS ----
// Gram matrix of the stored error vectors: <e_a, e_b> over the dense t1 and
// the dense t2 (four images per stored amplitude).
constexpr int kMaxDiis = 10;

template <typename T, int M>
__global__ void __launch_bounds__(kThreads) k_diis_gram(nlb_struct_problem P, nlb_struct_state S) {
    // FP32 error vectors: products and per-thread partial sums in FP32 (the
    // sums cover a few hundred elements, relative error ~1e-5, well inside
    // what the extrapolation needs), block and grid sums in FP64; FP64
    // vectors: FP64 throughout.  Two elements per thread and step keep
    // 2M loads in flight.
    using A = T;
    nlb_ctrl* c = S.ctrl;
    if (!c->diis_pulse) return;
    constexpr int NP = M * (M + 1) / 2;
    A acc[NP];   // sum of w/4 * e_s e_t: T1 entries weigh 1/4 here, T2 entries 1
#pragma unroll
    for (int k = 0; k < NP; ++k) acc[k] = A(0);
    const int64_t n1 = (int64_t)P.p * P.h;
    const int64_t n2 = c->ccs ? 0 : P.n_t2;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t tid0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    for (int64_t e = tid0; e < n1; e += stride) {
        A v[M];
#pragma unroll
        for (int s = 0; s < M; ++s) v[s] = (A)(0.5 * S.diis_t1[(int64_t)s * n1 + e]);
        int k = 0;
#pragma unroll
        for (int s = 0; s < M; ++s)
#pragma unroll
            for (int t = s; t < M; ++t) acc[k++] += v[s] * v[t];
    }
    // T2 part, weight 4 (four images per stored amplitude)
    const T* E2 = static_cast<const T*>(S.diis_t2);
    for (int64_t e = tid0; e < n2; e += 2 * stride) {
        const int64_t e2 = e + stride;
        const bool two = e2 < n2;
        T v[M], u[M];
#pragma unroll
        for (int s = 0; s < M; ++s) {
            v[s] = E2[(int64_t)s * P.n_t2 + e];
            u[s] = two ? E2[(int64_t)s * P.n_t2 + e2] : T(0);
        }
        int k = 0;
#pragma unroll
        for (int s = 0; s < M; ++s)
#pragma unroll
            for (int t = s; t < M; ++t) {
                acc[k] += v[s] * v[t] + u[s] * u[t];
                ++k;
            }
    }
    // warp reductions, then one shared-memory pass per warp
    __shared__ double red[kThreads / 32][NP];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NP; ++k) {
        const double v = warp_sum(4.0 * (double)acc[k]);
        if (lane == 0) red[wid][k] = v;
    }
    __syncthreads();
    double* part = prep_view(S.prep, P).gram_slots() + (int64_t)blockIdx.x * NP;
    for (int k = threadIdx.x; k < NP; k += blockDim.x) {
        double tot = 0.0;
        for (int w2 = 0; w2 < (int)(blockDim.x >> 5); ++w2) tot += red[w2][k];
        part[k] = tot;
    }
}

// Gram entry k (pair s <= t, row-major over the upper triangle) from the nb
// per-block partials of k_diis_gram, added in a fixed order: one block per
// entry, thread-strided sums then the fixed block tree.
template <int M>
__global__ void __launch_bounds__(kThreads) k_diis_reduce(nlb_ctrl* c, const double* part, int nb) {
    if (!c->diis_pulse) return;
    constexpr int NP = M * (M + 1) / 2;
    const int k = blockIdx.x;
    double s = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) s += part[(int64_t)b * NP + k];
    s = block_sum(s);
    if (threadIdx.x == 0) {
        int r = 0, rem = k;
        while (rem >= M - r) { rem -= M - r; ++r; }
        c->gram[r * kMaxDiis + r + rem] = s;
    }
}

// Bordered DIIS system [B/max|B|, -1; -1, 0] c = [0, -1], solved by Gaussian
// elimination with partial pivoting in FP64.  A zero pivot skips the
// extrapolation (the torch solver catches the failed solve and goes on).
// Leaves in gram[0] the weight of the current amplitudes and in gram[1+s]
// the weight of error vector s (t_new = w0 t_m + sum_s w_s e_s).
__global__ void k_diis_solve(nlb_ctrl* c) {
    // one warp: lane t owns column t of the bordered matrix in shared memory;
    // every entry sees the same operations in the same order as a serial
    // elimination (partial pivoting, first maximum on ties)
    if (blockIdx.x != 0 || !c->diis_pulse) return;
    const int lane = threadIdx.x;
    const int m = c->max_diis, n = m + 1;
    __shared__ double A[kMaxDiis + 1][kMaxDiis + 2];   // column n holds the right-hand side
    __shared__ double xs[kMaxDiis + 1];
    __shared__ int s_ok;
    double mx = 0.0;
    for (int k = lane; k < m * m; k += 32) {
        const int s = k / m, t = k - s * m;
        if (t >= s) mx = fmax(mx, fabs(c->gram[s * kMaxDiis + t]));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    const double nrm = mx + 1e-16;
    for (int k = lane; k < n * (n + 1); k += 32) {
        const int s = k / (n + 1), t = k - s * (n + 1);
        double v;
        if (t == n) v = (s == m) ? -1.0 : 0.0;
        else if (s < m && t < m) v = c->gram[(s <= t) ? s * kMaxDiis + t : t * kMaxDiis + s] / nrm;
        else if (s == m && t == m) v = 0.0;
        else v = -1.0;
        A[s][t] = v;
    }
    if (lane == 0) s_ok = 1;
    __syncwarp();
    for (int col = 0; col < n; ++col) {
        if (lane == 0) {
            int piv = col;
            for (int r = col + 1; r < n; ++r)
                if (fabs(A[r][col]) > fabs(A[piv][col])) piv = r;
            if (A[piv][col] == 0.0 || !isfinite(A[piv][col])) s_ok = 0;
            xs[0] = (double)piv;
        }
        __syncwarp();
        if (!s_ok) break;
        const int piv = (int)xs[0];
        if (piv != col && lane <= n) {
            const double tmp = A[col][lane]; A[col][lane] = A[piv][lane]; A[piv][lane] = tmp;
        }
        __syncwarp();
        for (int r = col + 1; r < n; ++r) {
            const double f = A[r][col] / A[col][col];
            __syncwarp();
            if (lane >= col && lane <= n) A[r][lane] -= f * A[col][lane];
            __syncwarp();
        }
    }
    __syncwarp();
    bool ok = s_ok != 0;
    if (lane == 0) {
        if (ok) {
            for (int r = n - 1; r >= 0; --r) {
                double sum = A[r][n];
                for (int t = r + 1; t < n; ++t) sum -= A[r][t] * xs[t];
                xs[r] = sum / A[r][r];
                if (!isfinite(xs[r])) ok = false;
            }
        }
        c->diis_applied = ok ? 1 : 0;
        if (ok) {
            // t_new = sum_k x_k t_{k+1},  t_{k+1} = t_m - sum_{s>k} e_s
            double tot = 0.0;
            for (int k = 0; k < m; ++k) tot += xs[k];
            c->gram[0] = tot;
            double run = 0.0;
            for (int s = 0; s < m; ++s) {
                c->gram[1 + s] = -run;
                run += xs[s];
            }
        }
    }
}

template <typename T> struct Vec2;
template <> struct Vec2<float> { using type = float2; };
template <> struct Vec2<double> { using type = double2; };

template <typename T, int M>
__global__ void __launch_bounds__(kThreads) k_diis_extrap(nlb_struct_problem P, nlb_struct_state S) {
    const nlb_ctrl* c = S.ctrl;
    if (!c->diis_pulse || !c->diis_applied) return;
    const int par = c->parity;
    const double w0 = c->gram[0];
    double w[M];
#pragma unroll
    for (int s = 0; s < M; ++s) w[s] = c->gram[1 + s];
    const int64_t n1 = (int64_t)P.p * P.h;
    const int64_t n2 = c->ccs ? 0 : P.n_t2;
    double* t1 = S.t1[par];
    T* t2 = static_cast<T*>(S.t2[par]);
    const T* E2 = static_cast<const T*>(S.diis_t2);
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    for (int64_t e = tid; e < n1; e += stride) {
        double v = w0 * t1[e];
#pragma unroll
        for (int s = 0; s < M; ++s) v += w[s] * S.diis_t1[(int64_t)s * n1 + e];
        t1[e] = v;
    }
    // T2: two amplitudes per thread with 8- (FP32) or 16-byte (FP64) loads
    // when every stored vector starts on such a boundary (n_t2 even, aligned
    // buffers); the arithmetic per amplitude is the same as one at a time
    using V = typename Vec2<T>::type;
    const bool aligned = ((reinterpret_cast<uintptr_t>(t2) | reinterpret_cast<uintptr_t>(E2)) % sizeof(V)) == 0;
    const int64_t npair = (P.n_t2 % 2 == 0 && aligned) ? n2 / 2 : 0;
    V* t2v = reinterpret_cast<V*>(t2);
    const V* E2v = reinterpret_cast<const V*>(E2);
    for (int64_t q = tid; q < npair; q += stride) {
        const V a = t2v[q];
        double vx = w0 * (double)a.x, vy = w0 * (double)a.y;
#pragma unroll
        for (int s = 0; s < M; ++s) {
            const V b = E2v[(int64_t)s * (P.n_t2 / 2) + q];
            vx += w[s] * (double)b.x;
            vy += w[s] * (double)b.y;
        }
        V o;
        o.x = (T)vx;
        o.y = (T)vy;
        t2v[q] = o;
    }
    for (int64_t q = 2 * npair + tid; q < n2; q += stride) {
        double v = w0 * (double)t2[q];
#pragma unroll
        for (int s = 0; s < M; ++s) v += w[s] * (double)E2[(int64_t)s * P.n_t2 + q];
        t2[q] = (T)v;
    }
}

__global__ void k_diis_done(nlb_ctrl* c) {
    if (threadIdx.x == 0 && blockIdx.x == 0 && c->diis_pulse) {
        c->diis_pulse = 0;
        c->diis_count = 0;
    }
}

// ------------------------------------------------------------- energy ----
// One block (t1 has p*h entries, a few ten thousand): a fixed summation order.
__global__ void __launch_bounds__(1024) k_energy(nlb_struct_problem P, nlb_struct_state S, double* out) {
    const double* t1 = S.t1[S.ctrl->parity];
    const int64_t n = (int64_t)P.p * P.h;
    double acc = 0.0;
    for (int64_t e = threadIdx.x; e < n; e += blockDim.x) acc += P.f_ph[e] * t1[e];
    const double s = block_sum(acc);
    if (threadIdx.x == 0) *out = s;
}

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
        const nlb_channel& ch = P.chan[ci];
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
        const nlb_channel& ch = P.chan[ci];
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

// Resident blocks per SM of each kernel (for a given dynamic smem), queried once.
struct OccEntry { const void* fn; int64_t smem; int bps; };
OccEntry g_occ[64];
int g_nocc = 0;

int64_t smem_limit();

int blocks_per_sm(const void* fn, int64_t smem, int threads = kThreads) {
    for (int k = 0; k < g_nocc; ++k)
        if (g_occ[k].fn == fn && g_occ[k].smem == smem) return g_occ[k].bps;
    // raise the limit to the device maximum (less the kernel's static shared
    // memory) for every kernel that takes dynamic shared memory: the 48 KB
    // default counts static shared memory too, and lowering the limit for a
    // smaller problem would break launches (and captured graphs) of a larger one
    if (smem > 0) {
        cudaFuncAttributes fa;
        if (cudaFuncGetAttributes(&fa, fn) == cudaSuccess)
            cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(smem_limit() - (int64_t)fa.sharedSizeBytes));
    }
    int bps = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, fn, threads, (size_t)smem) != cudaSuccess || bps <= 0)
        bps = 1;
    if (g_nocc < 64) g_occ[g_nocc++] = OccEntry{fn, smem, bps};
    return bps;
}

// Persistent-style grid: as many blocks as fit at once, never more than the work.
template <typename K>
int grid_for(K kernel, int64_t work) {
    const int bps = blocks_per_sm(reinterpret_cast<const void*>(kernel), 0);
    int64_t full = (int64_t)num_sms() * bps;
    int64_t need = (work + kThreads - 1) / kThreads;
    if (need < 1) need = 1;
    return (int)(need < full ? need : full);
}

int64_t smem_bytes(const nlb_struct_problem* P, int dtype) {
    const int64_t el = dtype == NLB_F64 ? 8 : 4;
    const int64_t mh = P->max_nh;
    return el * (2 * (int64_t)P->max_row + mh * mh * mh + 3 * mh * mh + 2 * mh);
}

int64_t g_smem_limit = 0;

int64_t smem_limit() {
    if (g_smem_limit == 0) {
        int dev = 0, v = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        g_smem_limit = v > 0 ? v : 227 * 1024;
    }
    return g_smem_limit;
}

// The lattice path of the T2 update applies (7 holes per label, diagonal
// ladders, short f_pp rows) and its shared memory fits.
bool use_lat(const nlb_struct_problem* P, size_t el) {
    return P->uniform_nh == 7 && P->diag_ladders && P->max_fpp_offdiag <= kLatNa &&
           lat_smem(P->max_row, 7, (int64_t)el, el == 4).total + 1024 <= smem_limit();
}

int valid(const nlb_struct_problem* P, const nlb_struct_state* S) {
    if (!P || !S || !S->ctrl) return fail(NLB_ERR_ARG, "null problem/state");
    if (P->p <= 0 || P->h <= 0 || P->n_channels < 0) return fail(NLB_ERR_SIZE, "bad p/h/channels");
    if (S->dtype != NLB_F64 && S->dtype != NLB_F32) return fail(NLB_ERR_ARG, "dtype must be NLB_F64 or NLB_F32");
    if (!S->t1[0] || !S->t1[1] || !S->prep) return fail(NLB_ERR_ARG, "null t1/prep buffer");
    if (P->n_t2 > 0 && (!S->t2[0] || !S->t2[1] || !S->g || !S->f2)) return fail(NLB_ERR_ARG, "null t2/g/f2 buffer");
    if (P->n_t2 > 0 && smem_bytes(P, S->dtype) > smem_limit())
        return fail(NLB_ERR_SIZE, "a T2 row does not fit in shared memory");
    return NLB_OK;
}

// Grid of a reducing launch: as many blocks as fit at once (bps per SM),
// never more than the work items nor the partial-sum slots.
int64_t reducing_grid(int bps, int64_t items) {
    int64_t grid = (int64_t)num_sms() * bps;
    if (grid > items) grid = items;
    if (grid > kRedSlots) grid = kRedSlots;
    return grid < 1 ? 1 : grid;
}

// The lattice T2 kernel with NT threads per block (NT / 49 hole-pair groups)
// and at least MINB resident blocks per SM.  Returns the grid; launch = false
// only computes it.
template <typename T, int NT, int MINB, bool PAIR = false>
int64_t launch_lat(const nlb_struct_problem* P, const nlb_struct_state* S, cudaStream_t st, bool launch = true) {
    const int64_t sm = lat_smem(P->max_row, 7, sizeof(T), PAIR).total;
    auto kern = k_t2_lat<T, 7, NT, MINB, PAIR>;
    const int64_t grid = reducing_grid(blocks_per_sm(reinterpret_cast<const void*>(kern), sm, NT), P->n_rows);
    if (launch) kern<<<(unsigned)grid, NT, (size_t)sm, st>>>(*P, *S);
    return grid;
}

// The two-row lattice T2 kernel (FP32) with NT threads per block; falls
// back to the one-row kernel when two double-buffered row pairs do not fit
// in shared memory.
template <int NT, int MINB>
int64_t launch_pair(const nlb_struct_problem* P, const nlb_struct_state* S, cudaStream_t st, bool launch = true) {
    const int64_t sm = pair_smem(P->max_row).total;
    if (sm + 1024 > smem_limit()) return launch_lat<float, 512, 1, true>(P, S, st, launch);
    auto kern = k_t2_pair<NT, MINB>;
    const int64_t grid = reducing_grid(blocks_per_sm(reinterpret_cast<const void*>(kern), sm, NT), P->n_rows);
    if (launch) kern<<<(unsigned)grid, NT, (size_t)sm, st>>>(*P, *S);
    return grid;
}

// The T2 update of one step (lattice or general kernel); returns its grid,
// 0 when there is no T2.  launch = false only computes the grid.
template <typename T>
int64_t t2_update(const nlb_struct_problem* P, const nlb_struct_state* S, cudaStream_t st, bool launch) {
    if (P->n_t2 <= 0) return 0;
    if (use_lat(P, sizeof(T))) {
        // launch shape from the problem's tuning word (FP32: bits 0-3, FP64:
        // bits 16-19), see nlb_struct_problem
        if constexpr (sizeof(T) == 4) {
            const int v = P->tune & 15;
            if (v == 5) return launch_pair<256, 1>(P, S, st, launch);
            if (v == 6) return launch_pair<384, 1>(P, S, st, launch);
            if (v == 7) return launch_pair<448, 1>(P, S, st, launch);
            if (v == 8) return launch_pair<512, 1>(P, S, st, launch);
            if (v == 3) return launch_lat<T, 512, 1, true>(P, S, st, launch);
            if (v == 4) return launch_lat<T, 384, 1, true>(P, S, st, launch);
            if (v == 1) return launch_lat<T, 512, 1>(P, S, st, launch);
            if (v == 2) return launch_lat<T, 384, 1>(P, S, st, launch);
            return launch_lat<T, 256, 2>(P, S, st, launch);
        } else {
            if (((P->tune >> 16) & 15) == 1) return launch_lat<T, 256, 1>(P, S, st, launch);
            return launch_lat<T, 512, 1>(P, S, st, launch);
        }
    }
    const int64_t sm = smem_bytes(P, sizeof(T) == 8 ? NLB_F64 : NLB_F32);
    auto kern = P->uniform_nh == 7 ? k_t2_rows<T, 7> : P->uniform_nh == 1 ? k_t2_rows<T, 1> : k_t2_rows<T, 0>;
    const int64_t grid = reducing_grid(blocks_per_sm(reinterpret_cast<const void*>(kern), sm, kRowThreads), P->n_rows);
    if (launch) kern<<<(unsigned)grid, kRowThreads, (size_t)sm, st>>>(*P, *S);
    return grid;
}

template <typename T>
int64_t t1_grid(const nlb_struct_problem* P) {
    const int64_t need = (16 * (int64_t)P->n_t1c + kThreads - 1) / kThreads;
    return reducing_grid(blocks_per_sm(reinterpret_cast<const void*>(k_t1_update<T>), 0), need);
}

template <typename T>
void stage_t(const nlb_struct_problem* P, const nlb_struct_state* S, int stage, cudaStream_t st) {
    switch (stage) {
        case NLB_STAGE_PREP: {
            const int64_t nprep = (int64_t)P->h * P->h + 2 * (int64_t)P->p + P->n_t1c + P->n_xc + P->h;
            // the dressed-Fock tables and Ga in one launch (the GTERMS stage is then empty)
            const int64_t per_blk = (int64_t)kThreads * kGaVec;
            const int64_t gx = P->n_t2 > 0 ? (P->max_row + per_blk - 1) / per_blk : 1;
            const int64_t ga_blocks = (int64_t)P->n_channels * P->max_nh * gx;
            int64_t gp = (nprep + kThreads - 1) / kThreads;
            if (gp < 1) gp = 1;
            k_prep_ga<T><<<(unsigned)(ga_blocks + gp), kThreads, 0, st>>>(*P, *S, nprep, (int)gx);
            break;
        }
        case NLB_STAGE_GTERMS:
            break;   // Ga is formed with the prep tables
        case NLB_STAGE_T2:
            t2_update<T>(P, S, st, true);
            break;
        case NLB_STAGE_T1:
            k_t1_update<T><<<(unsigned)t1_grid<T>(P), kThreads, 0, st>>>(*P, *S);
            break;
        default:
            k_finish<<<1, 96, 0, st>>>(S->ctrl, prep_view(S->prep, *P).red, (int)t1_grid<T>(P),
                                       (int)t2_update<T>(P, S, st, false));
    }
}

template <typename T>
int step_t(const nlb_struct_problem* P, const nlb_struct_state* S, cudaStream_t st) {
    for (int k = NLB_STAGE_PREP; k <= NLB_STAGE_FINISH; ++k) stage_t<T>(P, S, k, st);
    return check_launch("nlb_struct_step");
}

template <typename T, int M>
void diis_m(const nlb_struct_problem* P, const nlb_struct_state* S, cudaStream_t st) {
    const int64_t n = (int64_t)P->p * P->h + P->n_t2;
    int nb = grid_for(k_diis_gram<T, M>, n);
    if (nb > kGramSlots) nb = kGramSlots;
    k_diis_gram<T, M><<<nb, kThreads, 0, st>>>(*P, *S);
    k_diis_reduce<M><<<M * (M + 1) / 2, kThreads, 0, st>>>(S->ctrl, prep_view(S->prep, *P).gram_slots(), nb);
    k_diis_solve<<<1, 32, 0, st>>>(S->ctrl);
    k_diis_extrap<T, M><<<grid_for(k_diis_extrap<T, M>, (n + 1) / 2), kThreads, 0, st>>>(*P, *S);
    k_diis_done<<<1, 32, 0, st>>>(S->ctrl);
}

template <typename T>
int diis_t(const nlb_struct_problem* P, const nlb_struct_state* S, int m, cudaStream_t st) {
    switch (m) {
        case 1: diis_m<T, 1>(P, S, st); break;
        case 2: diis_m<T, 2>(P, S, st); break;
        case 3: diis_m<T, 3>(P, S, st); break;
        case 4: diis_m<T, 4>(P, S, st); break;
        case 5: diis_m<T, 5>(P, S, st); break;
        case 6: diis_m<T, 6>(P, S, st); break;
        case 7: diis_m<T, 7>(P, S, st); break;
        case 8: diis_m<T, 8>(P, S, st); break;
        case 9: diis_m<T, 9>(P, S, st); break;
        case 10: diis_m<T, 10>(P, S, st); break;
        default: return fail(NLB_ERR_ARG, "max_diis must be in [1, 10]");
    }
    return check_launch("nlb_struct_diis");
}

}  // namespace

// ------------------------------------------------ no-allocation variant ----
// Scratch for nlb_struct_step_noalloc: the dressed-Fock tables, the Ga
// intermediates and the T1 Fock-term partial sums of one step, carved from a
// fixed array in device memory instead of caller-allocated buffers.  Every
// GPU that loads this library holds these 8 MiB until the process exits.
#define NLB_NOALLOC_SCRATCH_BYTES (8u << 20)
static __device__ __align__(256) unsigned char g_noalloc_scratch[NLB_NOALLOC_SCRATCH_BYTES];

namespace {
constexpr int kMaxDevices = 64;
void* g_noalloc_addr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device.  In host code
// the array's name is only a host-side stand-in, so the address comes from
// cudaGetSymbolAddress, once per device, with that device current.
int noalloc_scratch(void** out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        snprintf(g_err, sizeof(g_err), "nlb_struct_step_noalloc: cudaGetDevice: %s", cudaGetErrorString(e));
        return NLB_ERR_CUDA;
    }
    if (dev < 0 || dev >= kMaxDevices) return fail(NLB_ERR_ARG, "nlb_struct_step_noalloc: device index out of range");
    if (g_noalloc_addr[dev] == nullptr) {
        void* ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || ptr == nullptr) {
            snprintf(g_err, sizeof(g_err), "nlb_struct_step_noalloc: cudaGetSymbolAddress: %s",
                     cudaGetErrorString(e));
            return NLB_ERR_CUDA;
        }
        g_noalloc_addr[dev] = ptr;
    }
    *out = g_noalloc_addr[dev];
    return NLB_OK;
}

int64_t align256(int64_t b) { return (b + 255) & ~int64_t(255); }
}  // namespace

extern "C" {

int64_t nlb_struct_noalloc_scratch_bytes(const nlb_struct_problem* prob, int32_t dtype) {
    if (!prob || (dtype != NLB_F64 && dtype != NLB_F32)) return -1;
    if (prob->p <= 0 || prob->h <= 0 || prob->n_g < 0 || prob->n_f2 < 0 || prob->n_t1c < 0 || prob->n_xc < 0)
        return -1;
    const int64_t el = dtype == NLB_F64 ? 8 : 4;
    return align256(nlb_struct_prep_len(prob) * 8) + align256(prob->n_g * el) + align256(prob->n_f2 * el);
}

int nlb_struct_step_noalloc(const nlb_struct_problem* prob, const nlb_struct_state* st, nlb_stream_t stream) {
    if (!prob || !st || !st->ctrl) return fail(NLB_ERR_ARG, "nlb_struct_step_noalloc: null problem/state");
    if (st->dtype != NLB_F64 && st->dtype != NLB_F32) return fail(NLB_ERR_ARG, "nlb_struct_step_noalloc: bad dtype");
    const int64_t need = nlb_struct_noalloc_scratch_bytes(prob, st->dtype);
    if (need < 0) return fail(NLB_ERR_SIZE, "nlb_struct_step_noalloc: negative or zero sizes in the problem");
    if (need > (int64_t)NLB_NOALLOC_SCRATCH_BYTES) {
        snprintf(g_err, sizeof(g_err),
                 "nlb_struct_step_noalloc: problem needs %lld bytes of scratch, more than the %u-byte static "
                 "array; use nlb_struct_step with caller-allocated buffers",
                 (long long)need, NLB_NOALLOC_SCRATCH_BYTES);
        return NLB_ERR_SIZE;
    }
    void* base = nullptr;
    int rc = noalloc_scratch(&base);
    if (rc) return rc;
    const int64_t el = st->dtype == NLB_F64 ? 8 : 4;
    unsigned char* p = static_cast<unsigned char*>(base);
    nlb_struct_state local = *st;
    local.prep = reinterpret_cast<double*>(p);
    p += align256(nlb_struct_prep_len(prob) * 8);
    local.g = p;
    p += align256(prob->n_g * el);
    local.f2 = p;
    // Nothing in the scratch has to start at zero: every step writes the
    // tables, Ga and F2 before reading them, and the CCS mode reads neither.
    rc = valid(prob, &local);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    return local.dtype == NLB_F64 ? step_t<double>(prob, &local, s) : step_t<float>(prob, &local, s);
}


int nlb_version(void) { return 1; }

const char* nlb_last_error(void) { return g_err; }

int64_t nlb_struct_prep_len(const nlb_struct_problem* prob) {
    if (!prob) return 0;
    return 3 * (int64_t)prob->h * prob->h + 3 * (int64_t)prob->p + prob->n_t1c + prob->n_xc + prob->h + kRedLen;
}

int64_t nlb_struct_smem_bytes(const nlb_struct_problem* prob, int32_t dtype) {
    if (!prob) return 0;
    const int64_t b = smem_bytes(prob, dtype);
    return b <= smem_limit() ? b : 0;
}

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

int nlb_struct_stage(const nlb_struct_problem* prob, const nlb_struct_state* st, int32_t stage,
                     nlb_stream_t stream) {
    int rc = valid(prob, st);
    if (rc) return rc;
    if (stage < NLB_STAGE_PREP || stage > NLB_STAGE_FINISH) return fail(NLB_ERR_ARG, "bad stage");
    cudaStream_t s = (cudaStream_t)stream;
    if (st->dtype == NLB_F64) stage_t<double>(prob, st, stage, s); else stage_t<float>(prob, st, stage, s);
    return check_launch("nlb_struct_stage");
}

int nlb_struct_diis(const nlb_struct_problem* prob, const nlb_struct_state* st, int32_t max_diis,
                    nlb_stream_t stream) {
    // reads the amplitudes, the rings and the partial-sum area of st->prep
    // (not st->g / st->f2)
    if (!prob || !st || !st->ctrl) return fail(NLB_ERR_ARG, "nlb_struct_diis: null problem/state");
    if (prob->p <= 0 || prob->h <= 0 || prob->n_t2 < 0) return fail(NLB_ERR_SIZE, "nlb_struct_diis: bad sizes");
    if (st->dtype != NLB_F64 && st->dtype != NLB_F32) return fail(NLB_ERR_ARG, "nlb_struct_diis: bad dtype");
    if (!st->t1[0] || !st->t1[1] || !st->prep) return fail(NLB_ERR_ARG, "nlb_struct_diis: null t1/prep buffer");
    if (prob->n_t2 > 0 && (!st->t2[0] || !st->t2[1])) return fail(NLB_ERR_ARG, "nlb_struct_diis: null t2 buffer");
    if (!st->diis_t1 || (prob->n_t2 > 0 && !st->diis_t2)) return fail(NLB_ERR_ARG, "null DIIS ring");
    if (max_diis < 1 || max_diis > kMaxDiis) return fail(NLB_ERR_ARG, "max_diis must be in [1, 10]");
    cudaStream_t s = (cudaStream_t)stream;
    return st->dtype == NLB_F64 ? diis_t<double>(prob, st, max_diis, s) : diis_t<float>(prob, st, max_diis, s);
}

int nlb_struct_energy(const nlb_struct_problem* prob, const nlb_struct_state* st, double* e_out,
                      nlb_stream_t stream) {
    // reads t1, f_ph and ctrl only
    if (!prob || !st || !st->ctrl) return fail(NLB_ERR_ARG, "nlb_struct_energy: null problem/state");
    if (prob->p <= 0 || prob->h <= 0) return fail(NLB_ERR_SIZE, "nlb_struct_energy: bad p/h");
    if (!st->t1[0] || !st->t1[1] || !prob->f_ph) return fail(NLB_ERR_ARG, "nlb_struct_energy: null t1/f_ph");
    if (!e_out) return fail(NLB_ERR_ARG, "null e_out");
    cudaStream_t s = (cudaStream_t)stream;
    k_energy<<<1, 1024, 0, s>>>(*prob, *st, e_out);
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
