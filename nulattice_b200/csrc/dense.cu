// General (dense) CCSD kernels for sm_100a.
//
// For inputs without the label structure of the closed-site lattice problem
// (open-shell sites, non-SU(4) contacts, arbitrary matrix elements) the
// solver evaluates the reference's full factorised equation set
// (CCM/coupled_cluster.py:342-545, CCM/ccDgrams.py:13-578) on dense
// tensors: every diagram is a chain of pairwise tensor contractions run by
// nlb_contract_f64 (one strided FP64 kernel for all index patterns), the
// sparse v_ppph / v_pppp blocks are scattered by their own kernels, the
// antisymmetrisers pAB / pIJ are folded into one accumulate kernel, and the
// Jacobi update, energy and DIIS are fused elementwise kernels.

#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>

#include "nulattice_b200.h"

// defined in ccsd_struct.cu: records the text returned by nlb_last_error
void nlb_internal_set_error(const char* msg);

namespace {

int dfail(int code, const char* msg) {
    nlb_internal_set_error(msg);
    return code;
}

int dcheck(const char* where) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        char buf[512];
        snprintf(buf, sizeof(buf), "%s: %s", where, cudaGetErrorString(e));
        nlb_internal_set_error(buf);
        return NLB_ERR_LAUNCH;
    }
    return NLB_OK;
}

constexpr int TM = 64, TN = 64, TK = 16;
// most blocks of a reducing launch (partials in the caller's work buffer,
// NLB_DENSE_WORK_DOUBLES = 512 + kDenseSlots * 55)
constexpr int kDenseSlots = 1024;
static_assert(512 + kDenseSlots * 55 <= NLB_DENSE_WORK_DOUBLES, "work buffer");

__device__ __forceinline__ int64_t decode(int64_t lin, const int64_t* ext, const int64_t* str, int nd) {
    int64_t off = 0;
    for (int d = nd - 1; d >= 0; --d) {
        const int64_t e = ext[d];
        const int64_t idx = lin % e;
        lin /= e;
        off += idx * str[d];
    }
    return off;
}

// C[m,n] = alpha * sum_k A[m,k] B[k,n] + beta * C[m,n] over multi-indices.
// 256 threads, 64x64 output tile, 4x4 per thread, K in steps of 16.
__global__ void __launch_bounds__(256) k_contract(nlb_contract_desc d, const double* __restrict__ A,
                                                  const double* __restrict__ B, double* __restrict__ C,
                                                  double alpha, double beta) {
    __shared__ double As[TK][TM + 1];
    __shared__ double Bs[TK][TN + 1];
    __shared__ int64_t oam[TM], ocm[TM], obn[TN], ocn[TN], oak[TK], obk[TK];
    const int tid = threadIdx.x;
    const int64_t m0 = (int64_t)blockIdx.x * TM, n0 = (int64_t)blockIdx.y * TN;
    const int64_t bz = blockIdx.z;
    const int64_t offa_b = decode(bz, d.ext_b, d.sa_b, d.nb);
    const int64_t offb_b = decode(bz, d.ext_b, d.sb_b, d.nb);
    const int64_t offc_b = decode(bz, d.ext_b, d.sc_b, d.nb);
    if (tid < TM) {
        const int64_t m = m0 + tid;
        oam[tid] = m < d.M ? decode(m, d.ext_m, d.sa_m, d.nm) : 0;
        ocm[tid] = m < d.M ? decode(m, d.ext_m, d.sc_m, d.nm) : 0;
    } else if (tid < TM + TN) {
        const int64_t n = n0 + (tid - TM);
        obn[tid - TM] = n < d.N ? decode(n, d.ext_n, d.sb_n, d.nn) : 0;
        ocn[tid - TM] = n < d.N ? decode(n, d.ext_n, d.sc_n, d.nn) : 0;
    }
    const int tx = tid % 16, ty = tid / 16;
    double acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
    for (int64_t k0 = 0; k0 < d.K; k0 += TK) {
        __syncthreads();
        if (tid < TK) {
            const int64_t k = k0 + tid;
            oak[tid] = k < d.K ? decode(k, d.ext_k, d.sa_k, d.nk) : 0;
            obk[tid] = k < d.K ? decode(k, d.ext_k, d.sb_k, d.nk) : 0;
        }
        __syncthreads();
        for (int e = tid; e < TK * TM; e += 256) {
            const int kk = e / TM, mm = e % TM;
            const bool ok = (m0 + mm < d.M) && (k0 + kk < d.K);
            As[kk][mm] = ok ? A[offa_b + oam[mm] + oak[kk]] : 0.0;
        }
        for (int e = tid; e < TK * TN; e += 256) {
            const int kk = e / TN, nn = e % TN;
            const bool ok = (n0 + nn < d.N) && (k0 + kk < d.K);
            Bs[kk][nn] = ok ? B[offb_b + obn[nn] + obk[kk]] : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < TK; ++kk) {
            double a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = As[kk][ty + 16 * i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx + 16 * j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
        }
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int mm = ty + 16 * i;
        if (m0 + mm >= d.M) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int nn = tx + 16 * j;
            if (n0 + nn >= d.N) continue;
            double* c = C + offc_b + ocm[mm] + ocn[nn];
            *c = (beta == 0.0) ? alpha * acc[i][j] : alpha * acc[i][j] + beta * *c;
        }
    }
}

// H[a,b,i,j] += alpha * P(Z): perm 0 Z, 1 Z - Z^T(ab), 2 Z - Z^T(ij), 3 both.
__global__ void k_antisym_acc(const double* __restrict__ Z, double* __restrict__ H, int64_t p, int64_t h,
                              int perm, double alpha) {
    const int64_t n = p * p * h * h;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t j = e % h, i = (e / h) % h, b = (e / (h * h)) % p, a = e / (h * h * p);
        double v = Z[e];
        if (perm == 1 || perm == 3) v -= Z[((b * p + a) * h + i) * h + j];
        if (perm == 2 || perm == 3) v -= Z[((a * p + b) * h + j) * h + i];
        if (perm == 3) v += Z[((b * p + a) * h + j) * h + i];
        H[e] += alpha * v;
    }
}

// In-place projection onto tensors antisymmetric in (a,b) and in (i,j):
// H_abij <- ((H_abij - H_baij) - (H_abji - H_baji)) / 4.  One thread per
// orbit {abij, baij, abji, baji} (a < b, i < j); the grouping makes the
// result exactly antisymmetric in floating point and leaves an exactly
// antisymmetric H unchanged, so it only removes the rounding-level symmetric
// part that sums taken in different orders for the four images of an orbit
// leave behind (the Jacobi map amplifies that part).
__global__ void k_antisym_project(double* H, int64_t p, int64_t h) {
    const int64_t np = p * (p - 1) / 2, nh = h * (h - 1) / 2;
    const int64_t n = np * nh;
    for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < n; u += (int64_t)gridDim.x * blockDim.x) {
        int64_t ab = u / nh, ij = u % nh;
        // unrank pairs a<b and i<j
        int64_t a = (int64_t)((2 * p - 1 - sqrt((double)((2 * p - 1) * (2 * p - 1) - 8 * ab))) / 2);
        while (a > 0 && a * (2 * p - a - 1) / 2 > ab) --a;
        while ((a + 1) * (2 * p - a - 2) / 2 <= ab) ++a;
        const int64_t b = ab - a * (2 * p - a - 1) / 2 + a + 1;
        int64_t i = (int64_t)((2 * h - 1 - sqrt((double)((2 * h - 1) * (2 * h - 1) - 8 * ij))) / 2);
        while (i > 0 && i * (2 * h - i - 1) / 2 > ij) --i;
        while ((i + 1) * (2 * h - i - 2) / 2 <= ij) ++i;
        const int64_t j = ij - i * (2 * h - i - 1) / 2 + i + 1;
        double* x_abij = H + ((a * p + b) * h + i) * h + j;
        double* x_baij = H + ((b * p + a) * h + i) * h + j;
        double* x_abji = H + ((a * p + b) * h + j) * h + i;
        double* x_baji = H + ((b * p + a) * h + j) * h + i;
        const double uu = *x_abij - *x_baij, ww = *x_abji - *x_baji;
        const double v = 0.25 * (uu - ww);
        *x_abij = v;
        *x_baij = -v;
        *x_abji = -v;
        *x_baji = v;
    }
}

// zero the entries with a == b or i == j (antisymmetry forces them to zero)
__global__ void k_antisym_diag(double* H, int64_t p, int64_t h) {
    const int64_t n = p * p * h * h;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t j = e % h, i = (e / h) % h, b = (e / (h * h)) % p, a = e / (h * h * p);
        if (a == b || i == j) H[e] = 0.0;
    }
}

// The seven v_ppph intermediates of CCM/ccDgrams.py:13-45 from the row list
// (c, d, a, k, v).  Deterministic gathers: the plan holds the list sorted by
// each output's key (stable, so repeated keys keep their list order), and one
// thread per (key segment, free hole indices) adds the segment's terms in that
// order into the output it alone owns.  Outputs are zeroed by the caller.
struct PpphEntry {
    int64_t c, d, a, k;
    double v;
};

__device__ __forceinline__ PpphEntry ppph_entry(const nlb_ppph_plan& P, const int32_t* perm, int64_t q) {
    const int64_t e = perm[q];
    return PpphEntry{P.idx[4 * e], P.idx[4 * e + 1], P.idx[4 * e + 2], P.idx[4 * e + 3], P.val[e]};
}

// r1[a,d] -= v t1[c,k] and r3[d,a] += v t1[c,k]: one thread per (a, d) segment
__global__ void k_ppph_ad(nlb_ppph_plan P, const double* __restrict__ t1, int64_t p, int64_t h, double* r1,
                          double* r3) {
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < P.n_ad; s += (int64_t)gridDim.x * blockDim.x) {
        double acc = 0.0;
        PpphEntry e{};
        for (int64_t q = P.seg_ad[s]; q < P.seg_ad[s + 1]; ++q) {
            e = ppph_entry(P, P.perm_adk, q);
            acc += e.v * t1[e.c * h + e.k];
        }
        r1[e.a * p + e.d] -= acc;
        r3[e.d * p + e.a] += acc;
    }
}

// r0[a,j] -= 1/2 v t2[c,d,k,j]: one thread per (a segment, j)
__global__ void k_ppph_a(nlb_ppph_plan P, const double* __restrict__ t2, int64_t p, int64_t h, double* r0) {
    for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < P.n_a * h; u += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = u / h, j = u - s * h;
        double acc = 0.0;
        PpphEntry e{};
        for (int64_t q = P.seg_a[s]; q < P.seg_a[s + 1]; ++q) {
            e = ppph_entry(P, P.perm_adk, q);
            acc += e.v * t2[((e.c * p + e.d) * h + e.k) * h + j];
        }
        r0[e.a * h + j] -= 0.5 * acc;
    }
}

// r4[a,d,j,k] += v t1[c,j]: per (a, d, k) segment and j (list order A);
// r2[c,d,j,k] += v t1[a,j]: per (c, d, k) segment and j (list order C)
__global__ void k_ppph_r24(nlb_ppph_plan P, const double* __restrict__ t1, int64_t p, int64_t h, double* r2,
                           double* r4) {
    const int64_t n4 = P.n_adk * h, n2 = P.n_cdk * h;
    for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < n4 + n2; u += (int64_t)gridDim.x * blockDim.x) {
        const bool four = u < n4;
        const int64_t v = four ? u : u - n4;
        const int64_t s = v / h, j = v - s * h;
        const int64_t* seg = four ? P.seg_adk : P.seg_cdk;
        const int32_t* perm = four ? P.perm_adk : P.perm_cdk;
        double acc = 0.0;
        PpphEntry e{};
        for (int64_t q = seg[s]; q < seg[s + 1]; ++q) {
            e = ppph_entry(P, perm, q);
            acc += e.v * t1[(four ? e.c : e.a) * h + j];
        }
        if (four) r4[((e.a * p + e.d) * h + j) * h + e.k] += acc;
        else r2[((e.c * p + e.d) * h + j) * h + e.k] += acc;
    }
}

// r5[a,i,j,k] += v t2[c,d,i,j] and r6[a,i,j,k] += v t1[c,i] t1[d,j]: one
// thread per (a, k) segment and hole pair (i, j)
__global__ void k_ppph_ak(nlb_ppph_plan P, const double* __restrict__ t1, const double* __restrict__ t2, int64_t p,
                          int64_t h, double* r5, double* r6) {
    const int64_t hh = h * h;
    for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < P.n_ak * hh; u += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = u / hh, ij = u - s * hh, i = ij / h, j = ij - i * h;
        double a5 = 0.0, a6 = 0.0;
        PpphEntry e{};
        for (int64_t q = P.seg_ak[s]; q < P.seg_ak[s + 1]; ++q) {
            e = ppph_entry(P, P.perm_ak, q);
            a5 += e.v * t2[(e.c * p + e.d) * hh + ij];
            a6 += e.v * t1[e.c * h + i] * t1[e.d * h + j];
        }
        r5[((e.a * h + i) * h + j) * h + e.k] += a5;
        r6[((e.a * h + i) * h + j) * h + e.k] += a6;
    }
}

// The two v_pppp ladders of CCM/ccDgrams.py:215-237 (without the 1/2): one
// thread per ((a, b) segment, hole pair), terms in list order.
__global__ void k_pppp(nlb_pppp_plan P, const double* __restrict__ t1, const double* __restrict__ t2, int64_t p,
                       int64_t h, double* l1, double* l2) {
    const int64_t hh = h * h;
    for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < P.n_ab * hh; u += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = u / hh, ij = u - s * hh, i = ij / h, j = ij - i * h;
        double a1 = 0.0, a2 = 0.0;
        int64_t a = 0, b = 0;
        for (int64_t q = P.seg_ab[s]; q < P.seg_ab[s + 1]; ++q) {
            const int64_t e = P.perm_ab[q];
            a = P.idx[4 * e];
            b = P.idx[4 * e + 1];
            const int64_t c = P.idx[4 * e + 2], dd = P.idx[4 * e + 3];
            const double v = P.val[e];
            a1 += v * t2[(c * p + dd) * hh + ij];
            a2 += v * t1[c * h + i] * t1[dd * h + j];
        }
        l1[(a * p + b) * hh + ij] += a1;
        l2[(a * p + b) * hh + ij] += a2;
    }
}

// t_new = m t + (1-m) (t + H / D) with D from the dressed Fock diagonals
// (coupled_cluster.py:410-414, 538-545); also stores the change in `err`.
__global__ void k_jacobi_t1(const double* t1, const double* H1, const double* xpp, const double* xhh, int64_t p,
                            int64_t h, double mixing, double* out, double* err) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < p * h; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t a = e / h, i = e % h;
        const double den = -(xpp[a * p + a] + xhh[i * h + i]);
        const double tn = t1[e] + H1[e] / den;
        const double o = mixing * t1[e] + (1.0 - mixing) * tn;
        out[e] = o;
        if (err) err[e] = o - t1[e];
    }
}

__global__ void k_jacobi_t2(const double* t2, const double* H2, const double* xpp, const double* xhh, int64_t p,
                            int64_t h, double mixing, double* out, double* err) {
    const int64_t n = p * p * h * h;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t j = e % h, i = (e / h) % h, b = (e / (h * h)) % p, a = e / (h * h * p);
        const double den = -((xpp[a * p + a] + xpp[b * p + b]) + (xhh[i * h + i] + xhh[j * h + j]));
        const double tn = t2[e] + H2[e] / den;
        const double o = mixing * t2[e] + (1.0 - mixing) * tn;
        out[e] = o;
        if (err) err[e] = o - t2[e];
    }
}

__device__ double dblock_sum(double v) {
    __shared__ double s[32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) s[w] = v;
    __syncthreads();
    v = (threadIdx.x < (blockDim.x + 31) / 32) ? s[threadIdx.x] : 0.0;
    if (w == 0)
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// E = sum f_ai t1_ai + 1/4 sum v_abij t2_abij + 1/2 sum v_abij t1_ai t1_bj
// (coupled_cluster.py:265-286): one partial per block into part[blockIdx.x].
__global__ void k_energy_dense(const double* f_ph, const double* t1, const double* v, const double* t2, int64_t p,
                               int64_t h, double* part) {
    double acc = 0.0;
    const int64_t n1 = p * h, n2 = p * p * h * h;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n1 + n2;
         e += (int64_t)gridDim.x * blockDim.x) {
        if (e < n1) {
            acc += f_ph[e] * t1[e];
        } else if (v) {
            const int64_t q = e - n1;
            const int64_t j = q % h, i = (q / h) % h, b = (q / (h * h)) % p, a = q / (h * h * p);
            acc += v[q] * (0.25 * t2[q] + 0.5 * t1[a * h + i] * t1[b * h + j]);
        }
    }
    const double s = dblock_sum(acc);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// *out = the n partials at `part` added in slot order (one warp, fixed tree).
__global__ void k_sum_part(const double* part, int n, double* out) {
    double s = 0.0;
    for (int b = threadIdx.x; b < n; b += 32) s += part[b];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) *out = s;
}

// Gram matrix <e_s, e_t> of m stored error vectors: per-block partials of
// the pairs s <= t into part[blockIdx.x * 55 + k]; k_vec_gram_reduce adds them
// in block order into gram (row stride 16).
// (FP32 vectors are widened to FP64 before the products.)
template <typename V>
__global__ void k_vec_gram(const V* E, int64_t n, int m, double* part) {
    double acc[55];
    for (int k = 0; k < 55; ++k) acc[k] = 0.0;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        double v[10];
        for (int s = 0; s < m; ++s) v[s] = (double)E[(int64_t)s * n + e];
        int k = 0;
        for (int s = 0; s < m; ++s)
            for (int t = s; t < m; ++t) acc[k++] += v[s] * v[t];
    }
    const int np = m * (m + 1) / 2;
    for (int k = 0; k < np; ++k) {
        const double tot = dblock_sum(acc[k]);
        if (threadIdx.x == 0) part[(int64_t)blockIdx.x * 55 + k] = tot;
    }
}

// One block per pair k of the upper triangle: its nb partials in block order.
__global__ void k_vec_gram_reduce(const double* part, int nb, int m, double* gram) {
    const int k = blockIdx.x;
    double acc = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) acc += part[(int64_t)b * 55 + k];
    acc = dblock_sum(acc);
    if (threadIdx.x == 0) {
        int s = 0, rem = k;
        while (rem >= m - s) { rem -= m - s; ++s; }
        gram[s * 16 + s + rem] = acc;
    }
}

// Pulsed DIIS extrapolation (soa/coupled_cluster.py:533-561): bordered system
// in FP64 with partial pivoting; coef[0] = applied flag, coef[1+s] = c_s.
__global__ void k_vec_diis_solve(const double* gram, int m, double* coef) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int n = m + 1;
    double A[121], rhs[11], x[11];
    double mx = 0.0;
    for (int s = 0; s < m; ++s)
        for (int t = s; t < m; ++t) mx = fmax(mx, fabs(gram[s * 16 + t]));
    const double nrm = mx + 1e-16;
    for (int s = 0; s < n; ++s) {
        rhs[s] = (s == m) ? -1.0 : 0.0;
        for (int t = 0; t < n; ++t) {
            double v;
            if (s < m && t < m) v = gram[(s <= t) ? s * 16 + t : t * 16 + s] / nrm;
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
    if (ok) {
        for (int r = n - 1; r >= 0; --r) {
            double s = rhs[r];
            for (int t = r + 1; t < n; ++t) s -= A[r * n + t] * x[t];
            x[r] = s / A[r * n + r];
            if (!isfinite(x[r])) ok = false;
        }
    }
    coef[0] = ok ? 1.0 : 0.0;
    for (int s = 0; s < m; ++s) coef[1 + s] = ok ? x[s] : 0.0;
}

// t = sum_s c_s T_s over the stored amplitudes (history slots 1..m).
// (FP64 sums; FP32 vectors are rounded once on the store.)
template <typename V>
__global__ void k_vec_combine(const double* coef, const V* T, int64_t n, int m, V* out) {
    if (coef[0] == 0.0) return;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        double v = 0.0;
        for (int s = 0; s < m; ++s) v += coef[1 + s] * (double)T[(int64_t)s * n + e];
        out[e] = (V)v;
    }
}

int grid1(int64_t n) {
    const int64_t g = (n + 255) / 256;
    return (int)(g < 4096 ? (g > 0 ? g : 1) : 4096);
}

// Packing for the GEMM path of a contraction: X[r * cols + c] =
// src[decode(r) + decode(c)] (row-major panels the library GEMM reads), and
// the strided write-back C = alpha * P + beta * C.
__global__ void k_pack(const double* __restrict__ src, double* __restrict__ dst, int64_t rows, int64_t cols,
                       nlb_contract_desc d, int which) {
    const int64_t n = rows * cols;
    for (int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; l < n; l += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = l / cols, c = l - r * cols;
        int64_t off;
        if (which == 0) off = decode(r, d.ext_m, d.sa_m, d.nm) + decode(c, d.ext_k, d.sa_k, d.nk);   // A[m][k]
        else off = decode(r, d.ext_k, d.sb_k, d.nk) + decode(c, d.ext_n, d.sb_n, d.nn);              // B[k][n]
        dst[l] = src[off];
    }
}

__global__ void k_unpack_c(const double* __restrict__ P, double* __restrict__ C, nlb_contract_desc d, double alpha,
                           double beta) {
    const int64_t n = d.M * d.N;
    for (int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; l < n; l += (int64_t)gridDim.x * blockDim.x) {
        const int64_t m = l / d.N, q = l - m * d.N;
        const int64_t off = decode(m, d.ext_m, d.sc_m, d.nm) + decode(q, d.ext_n, d.sc_n, d.nn);
        const double v = alpha * P[l];
        C[off] = (beta == 0.0) ? v : v + beta * C[off];
    }
}

// One cuBLAS handle per device, bound to the caller's stream at each call,
// with a workspace of its own (allocated with the handle), so that cuBLAS
// never allocates inside a stream capture (setting the stream resets the
// workspace to the library's pool, so it is set again after each).
cublasHandle_t g_blas[64] = {};
void* g_blas_ws[64] = {};
constexpr size_t kBlasWorkspace = 32u << 20;

cublasHandle_t blas_handle(cudaStream_t st) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return nullptr;
    if (!g_blas[dev]) {
        if (cublasCreate(&g_blas[dev]) != CUBLAS_STATUS_SUCCESS) {
            g_blas[dev] = nullptr;
            return nullptr;
        }
        if (cudaMalloc(&g_blas_ws[dev], kBlasWorkspace) != cudaSuccess) {
            cudaGetLastError();
            g_blas_ws[dev] = nullptr;
        }
    }
    if (cublasSetStream(g_blas[dev], st) != CUBLAS_STATUS_SUCCESS) return nullptr;
    if (g_blas_ws[dev] && cublasSetWorkspace(g_blas[dev], g_blas_ws[dev], kBlasWorkspace) != CUBLAS_STATUS_SUCCESS)
        return nullptr;
    return g_blas[dev];
}

// Small outputs with long sums (a few output tiles, K >= kDotMinK): one block
// per output entry, the threads strided over K, a fixed tree.  The tiled
// kernel would give such a contraction a handful of blocks that walk K
// serially.
// (and at most kDotMaxMacs multiply-adds: beyond that the tiles' reuse wins)
constexpr int64_t kDotMaxOut = 1 << 15, kDotMinK = 64, kDotMaxMacs = int64_t(1) << 26;

__global__ void __launch_bounds__(256) k_contract_dot(nlb_contract_desc d, const double* __restrict__ A,
                                                      const double* __restrict__ B, double* __restrict__ C,
                                                      double alpha, double beta) {
    const int64_t o = blockIdx.x;   // (batch, m, n), n fastest
    const int64_t n = o % d.N, mb = o / d.N;
    const int64_t m = mb % d.M, bz = mb / d.M;
    const int64_t oa = decode(bz, d.ext_b, d.sa_b, d.nb) + decode(m, d.ext_m, d.sa_m, d.nm);
    const int64_t ob = decode(bz, d.ext_b, d.sb_b, d.nb) + decode(n, d.ext_n, d.sb_n, d.nn);
    double acc = 0.0;
    for (int64_t k = threadIdx.x; k < d.K; k += blockDim.x)
        acc = fma(A[oa + decode(k, d.ext_k, d.sa_k, d.nk)], B[ob + decode(k, d.ext_k, d.sb_k, d.nk)], acc);
    const double s = dblock_sum(acc);
    if (threadIdx.x == 0) {
        double* c = C + decode(bz, d.ext_b, d.sc_b, d.nb) + decode(m, d.ext_m, d.sc_m, d.nm) +
                    decode(n, d.ext_n, d.sc_n, d.nn);
        *c = (beta == 0.0) ? alpha * s : alpha * s + beta * *c;
    }
}

// Pulsed DIIS over m stored vectors: the Gram matrix (per-block partials,
// then pairs in block order), the bordered solve, the extrapolation.
// work: gram [0, 256), coefficients [256, 512), Gram partials after that.
template <typename V>
void vec_diis(const V* err, const V* hist, int64_t n, int m, double* work, V* out, cudaStream_t s) {
    int nb = grid1(n);
    if (nb > kDenseSlots) nb = kDenseSlots;
    double* part = work + 512;
    k_vec_gram<V><<<nb, 256, 0, s>>>(err, n, m, part);
    k_vec_gram_reduce<<<m * (m + 1) / 2, 256, 0, s>>>(part, nb, m, work);
    k_vec_diis_solve<<<1, 32, 0, s>>>(work, m, work + 256);
    k_vec_combine<V><<<grid1(n), 256, 0, s>>>(work + 256, hist, n, m, out);
}

}  // namespace

extern "C" {

int nlb_contract_f64(const nlb_contract_desc* d, const double* A, const double* B, double* C, double alpha,
                     double beta, nlb_stream_t stream) {
    if (!d || !A || !B || !C) return dfail(NLB_ERR_ARG, "nlb_contract_f64: null argument");
    if (d->nm > 4 || d->nn > 4 || d->nk > 4 || d->nb > 4 || d->nm < 0 || d->nn < 0 || d->nk < 0 || d->nb < 0)
        return dfail(NLB_ERR_ARG, "nlb_contract_f64: at most 4 indices per group");
    if (d->M <= 0 || d->N <= 0 || d->B < 1 || d->K < 0) return NLB_OK;
    if (d->B > 65535) return dfail(NLB_ERR_SIZE, "nlb_contract_f64: too many batch entries");
    const dim3 grid((unsigned)((d->M + TM - 1) / TM), (unsigned)((d->N + TN - 1) / TN), (unsigned)d->B);
    if (grid.y > 65535) return dfail(NLB_ERR_SIZE, "nlb_contract_f64: N too large");
    if (d->K == 0) {
        // empty sum: C = beta C (alpha * 0)
        k_contract<<<grid, 256, 0, (cudaStream_t)stream>>>(*d, A, B, C, 0.0, beta);
    } else if (d->M * d->N * d->B <= kDotMaxOut && d->K >= kDotMinK && d->M * d->N * d->B * d->K <= kDotMaxMacs) {
        k_contract_dot<<<(unsigned)(d->M * d->N * d->B), 256, 0, (cudaStream_t)stream>>>(*d, A, B, C, alpha, beta);
    } else {
        k_contract<<<grid, 256, 0, (cudaStream_t)stream>>>(*d, A, B, C, alpha, beta);
    }
    return dcheck("nlb_contract_f64");
}

int64_t nlb_contract_gemm_work(const nlb_contract_desc* d) {
    if (!d) return 0;
    return (d->M * d->K + d->K * d->N + d->M * d->N) * (int64_t)sizeof(double);
}

int nlb_contract_gemm_f64(const nlb_contract_desc* d, const double* A, const double* B, double* C, double alpha,
                          double beta, double* work, int64_t work_bytes, nlb_stream_t stream) {
    if (!d || !A || !B || !C || !work) return dfail(NLB_ERR_ARG, "nlb_contract_gemm_f64: null argument");
    if (d->nm > 4 || d->nn > 4 || d->nk > 4 || d->nm < 0 || d->nn < 0 || d->nk < 0 || d->nb != 0 || d->B != 1)
        return dfail(NLB_ERR_ARG, "nlb_contract_gemm_f64: no batch indices, at most 4 indices per group");
    if (d->M <= 0 || d->N <= 0) return NLB_OK;
    if (d->K <= 0) return nlb_contract_f64(d, A, B, C, alpha, beta, stream);
    if (work_bytes < nlb_contract_gemm_work(d)) return dfail(NLB_ERR_SIZE, "nlb_contract_gemm_f64: workspace too small");
    if (d->M > 0x7fffffff || d->N > 0x7fffffff || d->K > 0x7fffffff)
        return dfail(NLB_ERR_SIZE, "nlb_contract_gemm_f64: a GEMM side exceeds 2^31");
    cudaStream_t st = (cudaStream_t)stream;
    double* Ap = work;
    double* Bp = Ap + d->M * d->K;
    double* Cp = Bp + d->K * d->N;
    k_pack<<<grid1(d->M * d->K), 256, 0, st>>>(A, Ap, d->M, d->K, *d, 0);
    k_pack<<<grid1(d->K * d->N), 256, 0, st>>>(B, Bp, d->K, d->N, *d, 1);
    int rc = dcheck("nlb_contract_gemm_f64 (pack)");
    if (rc != NLB_OK) return rc;
    cublasHandle_t hb = blas_handle(st);
    if (!hb) return dfail(NLB_ERR_LAUNCH, "nlb_contract_gemm_f64: cuBLAS handle");
    // row-major Cp[M][N] = Ap[M][K] Bp[K][N]  <=>  column-major Cp^T = Bp^T Ap^T
    const double one = 1.0, zero = 0.0;
    if (cublasDgemm(hb, CUBLAS_OP_N, CUBLAS_OP_N, (int)d->N, (int)d->M, (int)d->K, &one, Bp, (int)d->N, Ap,
                    (int)d->K, &zero, Cp, (int)d->N) != CUBLAS_STATUS_SUCCESS)
        return dfail(NLB_ERR_LAUNCH, "nlb_contract_gemm_f64: cublasDgemm failed");
    k_unpack_c<<<grid1(d->M * d->N), 256, 0, st>>>(Cp, C, *d, alpha, beta);
    return dcheck("nlb_contract_gemm_f64 (write-back)");
}

int nlb_antisym_acc_f64(const double* Z, double* H, int64_t p, int64_t h, int32_t perm, double alpha,
                        nlb_stream_t stream) {
    if (!Z || !H || perm < 0 || perm > 3) return dfail(NLB_ERR_ARG, "nlb_antisym_acc_f64: bad argument");
    k_antisym_acc<<<grid1(p * p * h * h), 256, 0, (cudaStream_t)stream>>>(Z, H, p, h, perm, alpha);
    return dcheck("nlb_antisym_acc_f64");
}

int nlb_antisym_project_f64(double* H, int64_t p, int64_t h, nlb_stream_t stream) {
    if (!H) return dfail(NLB_ERR_ARG, "nlb_antisym_project_f64: null argument");
    cudaStream_t s = (cudaStream_t)stream;
    k_antisym_diag<<<grid1(p * p * h * h), 256, 0, s>>>(H, p, h);
    const int64_t n = (p * (p - 1) / 2) * (h * (h - 1) / 2);
    if (n > 0) k_antisym_project<<<grid1(n), 256, 0, s>>>(H, p, h);
    return dcheck("nlb_antisym_project_f64");
}

int nlb_ppph_intermediates_f64(const nlb_ppph_plan* plan, const double* t1, const double* t2, int64_t p,
                               int64_t h, double* const* r, nlb_stream_t stream) {
    if (!plan) return dfail(NLB_ERR_ARG, "nlb_ppph_intermediates_f64: null plan");
    if (plan->nnz == 0) return NLB_OK;
    const nlb_ppph_plan& P = *plan;
    if (!P.idx || !P.val || !P.perm_adk || !P.perm_ak || !P.perm_cdk || !P.seg_a || !P.seg_ad || !P.seg_adk ||
        !P.seg_ak || !P.seg_cdk || !t1 || !t2 || !r)
        return dfail(NLB_ERR_ARG, "nlb_ppph_intermediates_f64: null argument");
    if (P.n_a < 0 || P.n_ad < 0 || P.n_adk < 0 || P.n_ak < 0 || P.n_cdk < 0 || p <= 0 || h <= 0)
        return dfail(NLB_ERR_SIZE, "nlb_ppph_intermediates_f64: bad sizes");
    cudaStream_t s = (cudaStream_t)stream;
    if (P.n_ad) k_ppph_ad<<<grid1(P.n_ad), 256, 0, s>>>(P, t1, p, h, r[1], r[3]);
    if (P.n_a) k_ppph_a<<<grid1(P.n_a * h), 256, 0, s>>>(P, t2, p, h, r[0]);
    if (P.n_adk + P.n_cdk) k_ppph_r24<<<grid1((P.n_adk + P.n_cdk) * h), 256, 0, s>>>(P, t1, p, h, r[2], r[4]);
    if (P.n_ak) k_ppph_ak<<<grid1(P.n_ak * h * h), 256, 0, s>>>(P, t1, t2, p, h, r[5], r[6]);
    return dcheck("nlb_ppph_intermediates_f64");
}

int nlb_pppp_ladders_f64(const nlb_pppp_plan* plan, const double* t1, const double* t2, int64_t p, int64_t h,
                         double* l1, double* l2, nlb_stream_t stream) {
    if (!plan) return dfail(NLB_ERR_ARG, "nlb_pppp_ladders_f64: null plan");
    if (plan->nnz == 0 || plan->n_ab == 0) return NLB_OK;
    if (!plan->idx || !plan->val || !plan->perm_ab || !plan->seg_ab || !t1 || !t2 || !l1 || !l2)
        return dfail(NLB_ERR_ARG, "nlb_pppp_ladders_f64: null argument");
    if (plan->n_ab < 0 || p <= 0 || h <= 0) return dfail(NLB_ERR_SIZE, "nlb_pppp_ladders_f64: bad sizes");
    k_pppp<<<grid1(plan->n_ab * h * h), 256, 0, (cudaStream_t)stream>>>(*plan, t1, t2, p, h, l1, l2);
    return dcheck("nlb_pppp_ladders_f64");
}

int nlb_jacobi_f64(const double* t1, const double* H1, const double* t2, const double* H2, const double* xpp1,
                   const double* xhh1, const double* xpp2, const double* xhh2, int64_t p, int64_t h, double mixing,
                   double* t1_out, double* t2_out, double* e1, double* e2, nlb_stream_t stream) {
    cudaStream_t s = (cudaStream_t)stream;
    if (t1 && H1 && t1_out) k_jacobi_t1<<<grid1(p * h), 256, 0, s>>>(t1, H1, xpp1, xhh1, p, h, mixing, t1_out, e1);
    if (t2 && H2 && t2_out)
        k_jacobi_t2<<<grid1(p * p * h * h), 256, 0, s>>>(t2, H2, xpp2, xhh2, p, h, mixing, t2_out, e2);
    return dcheck("nlb_jacobi_f64");
}

int nlb_dense_energy_f64(const double* f_ph, const double* t1, const double* v_pphh, const double* t2, int64_t p,
                         int64_t h, double* out, double* work, nlb_stream_t stream) {
    if (!f_ph || !t1 || !out || !work) return dfail(NLB_ERR_ARG, "nlb_dense_energy_f64: null argument");
    if (v_pphh && !t2) return dfail(NLB_ERR_ARG, "nlb_dense_energy_f64: v_pphh without t2");
    cudaStream_t s = (cudaStream_t)stream;
    int nb = grid1(p * h + (v_pphh ? p * p * h * h : 0));
    if (nb > kDenseSlots) nb = kDenseSlots;
    k_energy_dense<<<nb, 256, 0, s>>>(f_ph, t1, v_pphh, t2, p, h, work);
    k_sum_part<<<1, 32, 0, s>>>(work, nb, out);
    return dcheck("nlb_dense_energy_f64");
}

int nlb_vec_diis_f64(const double* err, const double* hist, int64_t n, int32_t m, double* work, double* out,
                     nlb_stream_t stream) {
    if (!err || !hist || !work || !out || m < 1 || m > 10) return dfail(NLB_ERR_ARG, "nlb_vec_diis_f64: bad argument");
    vec_diis(err, hist, n, m, work, out, (cudaStream_t)stream);
    return dcheck("nlb_vec_diis_f64");
}

int nlb_vec_diis_f32(const float* err, const float* hist, int64_t n, int32_t m, double* work, float* out,
                     nlb_stream_t stream) {
    if (!err || !hist || !work || !out || m < 1 || m > 10) return dfail(NLB_ERR_ARG, "nlb_vec_diis_f32: bad argument");
    vec_diis(err, hist, n, m, work, out, (cudaStream_t)stream);
    return dcheck("nlb_vec_diis_f32");
}

}  // extern "C"
