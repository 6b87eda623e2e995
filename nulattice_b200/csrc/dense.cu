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
// part that atomics-ordered sums leave behind (the Jacobi map amplifies that
// part; the reference's sequential sums never create it).
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
// (c, d, a, k, v): one thread per (entry, hole pair).  Outputs are zeroed by
// the caller; repeated keys add up through the atomics.
__global__ void k_ppph(const int64_t* __restrict__ idx, const double* __restrict__ val, int64_t nnz,
                       const double* __restrict__ t1, const double* __restrict__ t2, int64_t p, int64_t h,
                       double* r0, double* r1, double* r2, double* r3, double* r4, double* r5, double* r6) {
    const int64_t hh = h * h;
    for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < nnz * hh;
         u += (int64_t)gridDim.x * blockDim.x) {
        const int64_t q = u / hh, ij = u % hh, i = ij / h, j = ij % h;
        const int64_t c = idx[4 * q], dd = idx[4 * q + 1], a = idx[4 * q + 2], k = idx[4 * q + 3];
        const double v = val[q];
        if (ij == 0) {
            atomicAdd(&r1[a * p + dd], -v * t1[c * h + k]);
            atomicAdd(&r3[dd * p + a], v * t1[c * h + k]);
        }
        if (i == 0) {
            // j plays the free hole index here
            atomicAdd(&r0[a * h + j], -0.5 * v * t2[((c * p + dd) * h + k) * h + j]);
            atomicAdd(&r2[((c * p + dd) * h + j) * h + k], v * t1[a * h + j]);
            atomicAdd(&r4[((a * p + dd) * h + j) * h + k], v * t1[c * h + j]);
        }
        atomicAdd(&r5[((a * h + i) * h + j) * h + k], v * t2[((c * p + dd) * h + i) * h + j]);
        atomicAdd(&r6[((a * h + i) * h + j) * h + k], v * t1[c * h + i] * t1[dd * h + j]);
    }
}

// The two v_pppp ladders of CCM/ccDgrams.py:215-237 (without the 1/2).
__global__ void k_pppp(const int64_t* __restrict__ idx, const double* __restrict__ val, int64_t nnz,
                       const double* __restrict__ t1, const double* __restrict__ t2, int64_t p, int64_t h,
                       double* l1, double* l2) {
    const int64_t hh = h * h;
    for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < nnz * hh;
         u += (int64_t)gridDim.x * blockDim.x) {
        const int64_t q = u / hh, ij = u % hh, i = ij / h, j = ij % h;
        const int64_t a = idx[4 * q], b = idx[4 * q + 1], c = idx[4 * q + 2], dd = idx[4 * q + 3];
        const double v = val[q];
        atomicAdd(&l1[(a * p + b) * hh + ij], v * t2[(c * p + dd) * hh + ij]);
        atomicAdd(&l2[(a * p + b) * hh + ij], v * t1[c * h + i] * t1[dd * h + j]);
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
// (coupled_cluster.py:265-286), accumulated into *out.
__global__ void k_energy_dense(const double* f_ph, const double* t1, const double* v, const double* t2, int64_t p,
                               int64_t h, double* out) {
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
    if (threadIdx.x == 0) atomicAdd(out, s);
}

// Gram matrix <e_s, e_t> of m stored error vectors, accumulated into gram
// (row stride 16).
__global__ void k_vec_gram(const double* E, int64_t n, int m, double* gram) {
    double acc[55];
    for (int k = 0; k < 55; ++k) acc[k] = 0.0;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        double v[10];
        for (int s = 0; s < m; ++s) v[s] = E[(int64_t)s * n + e];
        int k = 0;
        for (int s = 0; s < m; ++s)
            for (int t = s; t < m; ++t) acc[k++] += v[s] * v[t];
    }
    int k = 0;
    for (int s = 0; s < m; ++s)
        for (int t = s; t < m; ++t) {
            const double tot = dblock_sum(acc[k++]);
            if (threadIdx.x == 0) atomicAdd(&gram[s * 16 + t], tot);
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
__global__ void k_vec_combine(const double* coef, const double* T, int64_t n, int m, double* out) {
    if (coef[0] == 0.0) return;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        double v = 0.0;
        for (int s = 0; s < m; ++s) v += coef[1 + s] * T[(int64_t)s * n + e];
        out[e] = v;
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

// One cuBLAS handle per device, bound to the caller's stream at each call.
cublasHandle_t g_blas[64] = {};

cublasHandle_t blas_handle(cudaStream_t st) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return nullptr;
    if (!g_blas[dev] && cublasCreate(&g_blas[dev]) != CUBLAS_STATUS_SUCCESS) {
        g_blas[dev] = nullptr;
        return nullptr;
    }
    if (cublasSetStream(g_blas[dev], st) != CUBLAS_STATUS_SUCCESS) return nullptr;
    return g_blas[dev];
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

int nlb_ppph_intermediates_f64(const int64_t* idx, const double* val, int64_t nnz, const double* t1,
                               const double* t2, int64_t p, int64_t h, double* const* r, nlb_stream_t stream) {
    if (nnz == 0) return NLB_OK;
    if (!idx || !val || !t1 || !t2 || !r) return dfail(NLB_ERR_ARG, "nlb_ppph_intermediates_f64: null argument");
    k_ppph<<<grid1(nnz * h * h), 256, 0, (cudaStream_t)stream>>>(idx, val, nnz, t1, t2, p, h, r[0], r[1], r[2], r[3],
                                                                  r[4], r[5], r[6]);
    return dcheck("nlb_ppph_intermediates_f64");
}

int nlb_pppp_ladders_f64(const int64_t* idx, const double* val, int64_t nnz, const double* t1, const double* t2,
                         int64_t p, int64_t h, double* l1, double* l2, nlb_stream_t stream) {
    if (nnz == 0) return NLB_OK;
    if (!idx || !val || !t1 || !t2 || !l1 || !l2) return dfail(NLB_ERR_ARG, "nlb_pppp_ladders_f64: null argument");
    k_pppp<<<grid1(nnz * h * h), 256, 0, (cudaStream_t)stream>>>(idx, val, nnz, t1, t2, p, h, l1, l2);
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
                         int64_t h, double* out, nlb_stream_t stream) {
    if (!f_ph || !t1 || !out) return dfail(NLB_ERR_ARG, "nlb_dense_energy_f64: null argument");
    cudaStream_t s = (cudaStream_t)stream;
    cudaMemsetAsync(out, 0, sizeof(double), s);
    k_energy_dense<<<grid1(p * h + (v_pphh ? p * p * h * h : 0)), 256, 0, s>>>(f_ph, t1, v_pphh, t2, p, h, out);
    return dcheck("nlb_dense_energy_f64");
}

int nlb_vec_diis_f64(const double* err, const double* hist, int64_t n, int32_t m, double* work, double* out,
                     nlb_stream_t stream) {
    if (!err || !hist || !work || !out || m < 1 || m > 10) return dfail(NLB_ERR_ARG, "nlb_vec_diis_f64: bad argument");
    cudaStream_t s = (cudaStream_t)stream;
    cudaMemsetAsync(work, 0, 16 * 16 * sizeof(double), s);
    k_vec_gram<<<grid1(n), 256, 0, s>>>(err, n, m, work);
    k_vec_diis_solve<<<1, 32, 0, s>>>(work, m, work + 256);
    k_vec_combine<<<grid1(n), 256, 0, s>>>(work + 256, hist, n, m, out);
    return dcheck("nlb_vec_diis_f64");
}

}  // extern "C"
