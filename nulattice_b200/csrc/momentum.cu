// Momentum-block CCSD kernels for sm_100a: closed-shell plane-wave inputs
// with a contact interaction <pq||rs> = V[s_p s_q s_r s_s] delta(K).
//
// With every hole momentum filled in all four spin-isospin states, t1 and the
// T1 residual vanish by momentum conservation, and the T2 equation of
// CCM/coupled_cluster.py:476-536 (diagrams of CCM/ccDgrams.py) keeps the
// terms
//   v_pphh + 1/2 v_pppp t2 + 1/2 v_hhhh t2 + 1/4 (v_pphh t2) t2
//   - P(ab)P(ij) v_phph t2 + 1/2 P(ab)P(ij) t2 v_pphh t2
//   + P(ab) X_pp t2 + P(ij) X_hh t2,
// X_pp = f_pp - 1/2 v_pphh t2, X_hh = -f_hh - 1/2 v_pphh t2.  Because V does
// not depend on the momenta, each sum over a particle momentum collapses:
//   M_K[s_c s_d][ij]  = sum_{k_c} t2[(k_c s_c)(K-k_c s_d) ij]       (ladders)
//   R[a,i][s_c s_k]   = sum_{k_k} t2[a (k_k+k_i-k_a s_c) i (k_k s_k)] (rings)
// and the hole-hole ladder, dressed by the quadratic ladder term, is one
// small matrix W_K per block applied from the right.  The blocked layout is
// described with nlb_pw_problem in nulattice_b200.h.

#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>

#include "nulattice_b200.h"

void nlb_internal_set_error(const char* msg);

namespace {

int pfail(int code, const char* msg) {
    nlb_internal_set_error(msg);
    return code;
}

int pcheck(const char* where) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        char buf[512];
        snprintf(buf, sizeof(buf), "%s: %s", where, cudaGetErrorString(e));
        nlb_internal_set_error(buf);
        return NLB_ERR_LAUNCH;
    }
    return NLB_OK;
}

int pgrid(int64_t n) {
    const int64_t g = (n + 255) / 256;
    return (int)(g < 8192 ? (g > 0 ? g : 1) : 8192);
}

// block holding flat position e of an offset table off[0..n] (off[n] = end)
__device__ __forceinline__ int seg_of(const int64_t* off, int n, int64_t e) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (e >= off[mid]) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// total momentum k1 - k2 (mod L in each direction)
__device__ __forceinline__ int msub(int k1, int k2, int L) {
    const int x = (k1 / (L * L) - k2 / (L * L) + L) % L;
    const int y = ((k1 / L) % L - (k2 / L) % L + L) % L;
    const int z = (k1 % L - k2 % L + L) % L;
    return (x * L + y) * L + z;
}

__device__ __forceinline__ int madd(int k1, int k2, int L) {
    const int x = (k1 / (L * L) + k2 / (L * L)) % L;
    const int y = ((k1 / L) % L + (k2 / L) % L) % L;
    const int z = (k1 % L + k2 % L) % L;
    return (x * L + y) * L + z;
}

__device__ double pw_block_sum(double v) {
    __shared__ double s[32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) s[w] = v;
    __syncthreads();
    const int nw = (blockDim.x + 31) >> 5;
    v = (threadIdx.x < nw) ? s[threadIdx.x] : 0.0;
    if (w == 0)
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Decoded position of one blocked amplitude.
struct Amp {
    int b, r, c, nc;
    int sa, sb, si, sj;
    int ma, mb, mi, mj;    // momentum indices (particle / hole lists)
    int64_t off;           // block start
};

__device__ __forceinline__ Amp decode_amp(const nlb_pw_problem& P, int b, int r, int c) {
    Amp A;
    A.b = b; A.r = r; A.c = c;
    A.nc = P.blk_nc[b];
    A.off = P.blk_off[b];
    const int pa = r >> 4, pi = c >> 4;
    A.sa = (r >> 2) & 3; A.sb = r & 3;
    A.si = (c >> 2) & 3; A.sj = c & 3;
    const int L = P.L, K = P.blk_K[b];
    A.ma = P.pm_list[P.blk_pm0[b] + pa];
    A.mi = P.hm_list[P.blk_hm0[b] + pi];
    A.mb = P.pinv[msub(K, P.pmom[A.ma], L)];
    A.mj = P.hinv[msub(K, P.hmom[A.mi], L)];
    return A;
}

// ---------------------------------------------------------------- init ----
__global__ void k_pw_init(nlb_pw_problem P, double* t2, double delta) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < P.n_t2;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int b = seg_of(P.blk_off, P.n_blocks, e);
        const int64_t loc = e - P.blk_off[b];
        const int nc = P.blk_nc[b];
        const Amp A = decode_amp(P, b, (int)(loc / nc), (int)(loc % nc));
        const double v = P.V[((A.sa * 4 + A.sb) * 4 + A.si) * 4 + A.sj];
        const double ea = P.fpp[A.ma * 16 + A.sa * 5], eb = P.fpp[A.mb * 16 + A.sb * 5];
        const double ei = P.fhh[A.mi * 16 + A.si * 5], ej = P.fhh[A.mj * 16 + A.sj * 5];
        t2[e] = v / ((((-ea - eb) + ei) + ej) + delta);
    }
}

// ------------------------------------------------------------ M, energy ----
// M_K[sigma][c] = sum_pa T_K[pa*16 + sigma][c]: one warp per entry, the
// lanes over the row groups pa, summed by a fixed shuffle tree.
template <typename F>
__global__ void k_pw_M(nlb_pw_problem P, const F* __restrict__ t2, F* __restrict__ M) {
    const int lane = threadIdx.x & 31;
    const int64_t wpb = blockDim.x >> 5;
    for (int64_t e = (int64_t)blockIdx.x * wpb + (threadIdx.x >> 5); e < P.n_m; e += (int64_t)gridDim.x * wpb) {
        const int b = seg_of(P.m_off, P.n_blocks, e);
        const int nc = P.blk_nc[b];
        const int64_t loc = e - P.m_off[b];
        const int sg = (int)(loc / nc), c = (int)(loc % nc);
        const int npa = P.blk_nr[b] >> 4;
        const F* T = t2 + P.blk_off[b] + (int64_t)sg * nc + c;
        F acc = 0.0;
        for (int pa = lane; pa < npa; pa += 32) acc += T[(int64_t)pa * 16 * nc];
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) M[e] = acc;
    }
}

// E = 1/4 sum_K sum_{sigma, c} V[sigma][spins of c] M_K[sigma][c] in two
// launches: block x of the first adds the fixed slice x of M (its threads
// strided, then a fixed tree) into part[x]; one block then adds the parts in
// slice order.  The result does not depend on scheduling.
constexpr int kPwEnergyParts = 256;

template <typename F>
__global__ void k_pw_energy_part(nlb_pw_problem P, const F* __restrict__ M, double* __restrict__ part) {
    const int64_t n = P.n_m;
    const int64_t chunk = (n + gridDim.x - 1) / gridDim.x;
    const int64_t e0 = (int64_t)blockIdx.x * chunk;
    const int64_t e1 = e0 + chunk < n ? e0 + chunk : n;
    double acc = 0.0;
    int b = -1;
    for (int64_t e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
        if (b < 0) b = seg_of(P.m_off, P.n_blocks, e);
        while (e >= P.m_off[b + 1]) ++b;   // the thread's entries only move forward
        const int nc = P.blk_nc[b];
        const int64_t loc = e - P.m_off[b];
        const int sg = (int)(loc / nc), c = (int)(loc % nc);
        acc += P.V[sg * 16 + (c & 15)] * (double)M[e];
    }
    const double s = pw_block_sum(acc);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

__global__ void k_pw_energy_sum(const double* __restrict__ part, int n, double* out) {
    double acc = 0.0;
    for (int k = threadIdx.x; k < n; k += blockDim.x) acc += part[k];
    const double s = pw_block_sum(acc);
    if (threadIdx.x == 0) *out = 0.25 * s;
}

// ------------------------------------------------------------ X_pp rows ----
// One warp per row (pa, s_b, s_d) of every block:
//   Y[row][s_c] = sum_c V[s_c s_d][spins of c] T[row][c]
template <typename F>
__global__ void k_pw_xrow(nlb_pw_problem P, const F* __restrict__ t2, F* __restrict__ Y) {
    __shared__ F Vs[256];
    for (int q = threadIdx.x; q < 256; q += blockDim.x) Vs[q] = P.V[q];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int64_t nrows = P.n_rows;
    const int64_t wpb = blockDim.x >> 5;
    for (int64_t row = (int64_t)blockIdx.x * wpb + (threadIdx.x >> 5); row < nrows; row += (int64_t)gridDim.x * wpb) {
        const int b = seg_of(P.row_off, P.n_blocks, row);
        const int r = (int)(row - P.row_off[b]);
        const int nc = P.blk_nc[b];
        const int sd = r & 3;
        const F* T = t2 + P.blk_off[b] + (int64_t)r * nc;
        F a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
        for (int c = lane; c < nc; c += 32) {
            const F x = T[c];
            const int sp = c & 15;
            a0 += Vs[(0 * 4 + sd) * 16 + sp] * x;
            a1 += Vs[(1 * 4 + sd) * 16 + sp] * x;
            a2 += Vs[(2 * 4 + sd) * 16 + sp] * x;
            a3 += Vs[(3 * 4 + sd) * 16 + sp] * x;
        }
        for (int o = 16; o > 0; o >>= 1) {
            a0 += __shfl_xor_sync(0xffffffffu, a0, o);
            a1 += __shfl_xor_sync(0xffffffffu, a1, o);
            a2 += __shfl_xor_sync(0xffffffffu, a2, o);
            a3 += __shfl_xor_sync(0xffffffffu, a3, o);
        }
        if (lane == 0) {
            Y[row * 4 + 0] = a0; Y[row * 4 + 1] = a1; Y[row * 4 + 2] = a2; Y[row * 4 + 3] = a3;
        }
    }
}

// ------------------------------------------------------ X_pp and X_hh ----
// X_pp[m][s_b][s_c] = f_pp - 1/2 sum_K sum_{s_d} Y[(K, pa(m), s_b, s_d)][s_c]   (ccDgrams.py:502-514)
// X_hh[m][s_k][s_j] = -f_hh - 1/2 sum_{m_l} sum_{s_l} sum_sigma
//                     V[sigma][s_k s_l] M_{m+m_l}[sigma][(m, s_j, s_l)]       (ccDgrams.py:515-527)
// One warp per entry: the lanes take the momentum blocks (X_pp) or the
// (m_l, s_l) pairs (X_hh) strided, a fixed shuffle tree adds them.
template <typename F>
__global__ void k_pw_X(nlb_pw_problem P, const F* __restrict__ Y, const F* __restrict__ M,
                       F* __restrict__ Xpp, F* __restrict__ Xhh) {
    const int L = P.L, L3 = L * L * L;
    const int lane = threadIdx.x & 31;
    const int64_t wpb = blockDim.x >> 5;
    const int64_t np = (int64_t)P.n_pmom * 16, nh = (int64_t)P.n_hmom * 16;
    for (int64_t e = (int64_t)blockIdx.x * wpb + (threadIdx.x >> 5); e < np + nh; e += (int64_t)gridDim.x * wpb) {
        F acc = 0.0;
        if (e < np) {
            const int m = (int)(e >> 4), sb = (int)(e >> 2) & 3, sc = (int)e & 3;
            const int k = P.pmom[m];
            for (int b = lane; b < P.n_blocks; b += 32) {
                const int pa = P.ppos[(int64_t)b * L3 + k];
                if (pa < 0) continue;
                const int64_t row = P.row_off[b] + pa * 16 + sb * 4;
#pragma unroll
                for (int sd = 0; sd < 4; ++sd) acc += Y[(row + sd) * 4 + sc];
            }
        } else {
            const int64_t u = e - np;
            const int m = (int)(u >> 4), sk = (int)(u >> 2) & 3, sj = (int)u & 3;
            const int k = P.hmom[m];
            for (int w = lane; w < 4 * P.n_hmom; w += 32) {
                const int l = w >> 2, sl = w & 3;
                const int b = P.kblk[madd(k, P.hmom[l], L)];
                const int pj = P.hpos[(int64_t)b * L3 + k];
                const int nc = P.blk_nc[b];
                const F* Mb = M + P.m_off[b];
                const int col = pj * 16 + sj * 4 + sl;
#pragma unroll 4
                for (int sg = 0; sg < 16; ++sg) acc += F(P.V[sg * 16 + sk * 4 + sl]) * Mb[(int64_t)sg * nc + col];
            }
        }
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) {
            if (e < np) Xpp[e] = F(P.fpp[e]) - F(0.5) * acc;
            else Xhh[e - np] = -F(P.fhh[e - np]) - F(0.5) * acc;
        }
    }
}

// ---------------------------------------------------------------- W_K ----
// W_K[c'][c] = 1/2 V[spins c'][spins c] + 1/4 sum_sigma V[sigma][spins c'] M_K[sigma][c]
// (dgram_klij_abkl and dgram_cdkl_cdij_abkl, ccDgrams.py:240-251, 292-303)
template <typename F>
__global__ void k_pw_W(nlb_pw_problem P, const F* __restrict__ M, F* __restrict__ W) {
    const int64_t n = P.n_w;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const int b = seg_of(P.w_off, P.n_blocks, e);
        const int nc = P.blk_nc[b];
        const int64_t loc = e - P.w_off[b];
        const int cp = (int)(loc / nc), c = (int)(loc % nc);
        const F* Mb = M + P.m_off[b];
        F acc = 0.0;
#pragma unroll 4
        for (int sg = 0; sg < 16; ++sg) acc += F(P.V[sg * 16 + (cp & 15)]) * Mb[(int64_t)sg * nc + c];
        W[e] = F(0.5) * F(P.V[(cp & 15) * 16 + (c & 15)]) + F(0.25) * acc;
    }
}

// ------------------------------------------------------- ring intermediates ----
// One thread per (a, i) = (particle momentum, s_a) x (hole momentum, s_i):
//   R[s_c s_k] = sum_{k_k} t2[a, (k_k + k_i - k_a, s_c), i, (k_k, s_k)]
//   G[s_b s_j] = - sum V[s_b s_k s_c s_j] R[s_c s_k]        (dgram_bkcj_acik, ccDgrams.py:253-264)
//   U[s_d s_l] = sum V[s_c s_d s_k s_l] R[s_c s_k]          (dgram_cdkl_acik_dblj, ccDgrams.py:279-290)
template <typename F>
__global__ void k_pw_R(nlb_pw_problem P, const F* __restrict__ t2, F* __restrict__ R,
                       F* __restrict__ U, F* __restrict__ G) {
    __shared__ F Vs[256];
    for (int q = threadIdx.x; q < 256; q += blockDim.x) Vs[q] = P.V[q];
    __syncthreads();
    const int L = P.L, L3 = L * L * L;
    const int nps = 4 * P.n_pmom, nhs = 4 * P.n_hmom;
    const int64_t n = (int64_t)nps * nhs;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const int al = (int)(e / nhs), il = (int)(e % nhs);
        const int ma = al >> 2, sa = al & 3, mi = il >> 2, si = il & 3;
        const int ka = P.pmom[ma], ki = P.hmom[mi];
        F r[16];
#pragma unroll
        for (int q = 0; q < 16; ++q) r[q] = 0.0;
        for (int mk = 0; mk < P.n_hmom; ++mk) {
            const int kk = P.hmom[mk];
            const int kc = msub(madd(kk, ki, L), ka, L);
            if (P.pinv[kc] < 0) continue;
            const int b = P.kblk[madd(ka, kc, L)];
            const int pa = P.ppos[(int64_t)b * L3 + ka];
            const int pi = P.hpos[(int64_t)b * L3 + ki];
            const int nc = P.blk_nc[b];
            const F* T = t2 + P.blk_off[b] + (int64_t)(pa * 16 + sa * 4) * nc + pi * 16 + si * 4;
#pragma unroll
            for (int sc = 0; sc < 4; ++sc)
#pragma unroll
                for (int sk = 0; sk < 4; ++sk) r[sc * 4 + sk] += T[(int64_t)sc * nc + sk];
        }
        F* Ro = R + e * 16;
        F* Uo = U + e * 16;
        F* Go = G + e * 16;
#pragma unroll
        for (int q = 0; q < 16; ++q) Ro[q] = r[q];
        for (int x = 0; x < 4; ++x)
            for (int y = 0; y < 4; ++y) {
                F g = 0.0, u = 0.0;
#pragma unroll
                for (int sc = 0; sc < 4; ++sc)
#pragma unroll
                    for (int sk = 0; sk < 4; ++sk) {
                        g += Vs[((x * 4 + sk) * 4 + sc) * 4 + y] * r[sc * 4 + sk];
                        u += Vs[((sc * 4 + x) * 4 + sk) * 4 + y] * r[sc * 4 + sk];
                    }
                Go[x * 4 + y] = -g;
                Uo[x * 4 + y] = u;
            }
    }
}

template <typename F>
__device__ __forceinline__ F dot16(const F* __restrict__ x, const F* __restrict__ y) {
    F s = 0;
    if constexpr (sizeof(F) == 8) {
#pragma unroll
        for (int q = 0; q < 16; q += 2) {
            const double2 a = *reinterpret_cast<const double2*>(x + q);
            const double2 c = *reinterpret_cast<const double2*>(y + q);
            s += a.x * c.x;
            s += a.y * c.y;
        }
    } else {
#pragma unroll
        for (int q = 0; q < 16; q += 4) {
            const float4 a = *reinterpret_cast<const float4*>(x + q);
            const float4 c = *reinterpret_cast<const float4*>(y + q);
            s += a.x * c.x;
            s += a.y * c.y;
            s += a.z * c.z;
            s += a.w * c.w;
        }
    }
    return s;
}

// ------------------------------------------------------------- residual ----
// One CTA per tile of 64 rows (four whole row groups pa) x 16 columns (one
// column group pi) of one block: T_K W_K for the tile through shared memory,
// then every other term of the residual per amplitude.  The tile's own T
// values (all the X_pp / X_hh terms need), V and the momenta of the tile's
// row and column groups sit in shared memory.  The quadratic ring term uses
// Z(ai, bj) = R_ai V R_bj = Z(bj, ai) (V[c d k l] = V[d c l k]), so its four
// images reduce to 2 (Z(ai, bj) - Z(bi, aj)).
constexpr int kTR = 64, kTC = 16;

template <typename F>
__global__ void __launch_bounds__(256) k_pw_residual(nlb_pw_problem P, const F* __restrict__ t2,
                                                     const F* __restrict__ M, const F* __restrict__ W,
                                                     const F* __restrict__ Xpp, const F* __restrict__ Xhh,
                                                     const F* __restrict__ R, const F* __restrict__ U,
                                                     const F* __restrict__ G, F* __restrict__ H) {
    __shared__ F Ts[kTR][kTC + 1];
    __shared__ F Town[kTR][kTC + 1];
    __shared__ F Ws[kTC][kTC + 1];
    __shared__ F Vs[256];
    __shared__ int s_ma[4], s_mb[4], s_mi, s_mj;
    const int tid = threadIdx.x;
    const int cc = tid & 15, rr = tid >> 4;
    const int nhs = 4 * P.n_hmom;
    const int L = P.L;
    Vs[tid] = P.V[tid];
    for (int tile = blockIdx.x; tile < P.n_tiles; tile += gridDim.x) {
        const int b = P.tiles[3 * tile], r0 = P.tiles[3 * tile + 1], c0 = P.tiles[3 * tile + 2];
        const int nr = P.blk_nr[b], nc = P.blk_nc[b], K = P.blk_K[b];
        __syncthreads();   // the previous tile's epilogue is done with the shared tables
        if (tid < 4) {
            const int pa = (r0 >> 4) + tid;
            int ma = 0, mb = 0;
            if (pa * 16 < nr) {
                ma = P.pm_list[P.blk_pm0[b] + pa];
                mb = P.pinv[msub(K, P.pmom[ma], L)];
            }
            s_ma[tid] = ma;
            s_mb[tid] = mb;
        } else if (tid == 4) {
            const int mi = P.hm_list[P.blk_hm0[b] + (c0 >> 4)];
            s_mi = mi;
            s_mj = P.hinv[msub(K, P.hmom[mi], L)];
        }
        const F* T = t2 + P.blk_off[b];
        const F* Wb = W + P.w_off[b];
        F acc[4] = {0.0, 0.0, 0.0, 0.0};
        for (int k0 = 0; k0 < nc; k0 += kTC) {
            __syncthreads();
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int e = tid + 256 * q;
                const int rrow = e >> 4, kk = e & 15;
                const int r = r0 + rrow;
                const F x = (r < nr) ? T[(int64_t)r * nc + k0 + kk] : 0.0;
                Ts[rrow][kk] = x;
                if (k0 == c0) Town[rrow][kk] = x;
            }
            Ws[rr][cc] = Wb[(int64_t)(k0 + rr) * nc + c0 + cc];
            __syncthreads();
#pragma unroll
            for (int kk = 0; kk < kTC; ++kk) {
                const F w = Ws[kk][cc];
#pragma unroll
                for (int q = 0; q < 4; ++q) acc[q] += Ts[rr + 16 * q][kk] * w;
            }
        }
        const F* Mb = M + P.m_off[b];
        const int c = c0 + cc;
        const int si = (cc >> 2) & 3, sj = cc & 3, sa = (rr >> 2) & 3, sb = rr & 3;
        const int sab = sa * 4 + sb, sij = si * 4 + sj;
        const int mi = s_mi, mj = s_mj;
        // 1/2 v_pppp t2 through M: the same 16 M values for the four rows
        F lad = 0.0;
#pragma unroll
        for (int sg = 0; sg < 16; ++sg) lad += Vs[sab * 16 + sg] * Mb[(int64_t)sg * nc + c];
        F xhh_j[4], xhh_i[4];
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            xhh_j[s] = Xhh[mj * 16 + s * 4 + sj];
            xhh_i[s] = Xhh[mi * 16 + s * 4 + si];
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int rl = rr + 16 * q;
            const int r = r0 + rl;
            if (r >= nr) continue;
            const int ma = s_ma[q], mb = s_mb[q];
            // v_pphh, 1/2 v_pppp t2 (ccDgrams.py:215-237), hole-hole ladders
            F h = Vs[sab * 16 + sij] + F(0.5) * lad + acc[q];
            // P(ab) X_pp t2 and P(ij) X_hh t2 (coupled_cluster.py:536)
            F xp = 0.0, xh = 0.0;
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                xp += Xpp[mb * 16 + sb * 4 + s] * Town[q * 16 + sa * 4 + s][cc];
                xp += Xpp[ma * 16 + sa * 4 + s] * Town[q * 16 + s * 4 + sb][cc];
                xh += xhh_j[s] * Town[rl][si * 4 + s];
                xh += xhh_i[s] * Town[rl][s * 4 + sj];
            }
            h += xp + xh;
            // rings (four images of G) and the quadratic ring term
            const int64_t a = ma * 4 + sa, bb = mb * 4 + sb;
            const int64_t i = mi * 4 + si, j = mj * 4 + sj;
            const int64_t ai = (a * nhs + i) * 16, bi = (bb * nhs + i) * 16;
            const int64_t aj = (a * nhs + j) * 16, bj = (bb * nhs + j) * 16;
            const F ring = ((G[ai + sb * 4 + sj] - G[bi + sa * 4 + sj]) -
                                 (G[aj + sb * 4 + si] - G[bj + sa * 4 + si]));
            const F quad = dot16(U + ai, R + bj) - dot16(U + bi, R + aj);
            h += ring + quad;
            H[P.blk_off[b] + (int64_t)r * nc + c] = h;
        }
    }
}

// --------------------------------------------------------------- Jacobi ----
// Exact antisymmetric projection over the orbit {abij, baij, abji, baji} (the
// four images sit in the same block), Jacobi step with the dressed diagonal
// denominators and mixing (coupled_cluster.py:538-545, 614-620).
template <typename F>
__global__ void k_pw_jacobi(nlb_pw_problem P, const F* __restrict__ t2, const F* __restrict__ H,
                            const F* __restrict__ Xpp, const F* __restrict__ Xhh, double mixing,
                            F* __restrict__ out, F* __restrict__ err) {
    // grid (chunks, momentum blocks): blockIdx.y is the block of t2
    const int L = P.L, L3 = L * L * L;
    const int b = blockIdx.y;
    const int64_t boff = P.blk_off[b], bn = P.blk_off[b + 1] - boff;
    const int nc = P.blk_nc[b];
    for (int64_t loc = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; loc < bn;
         loc += (int64_t)gridDim.x * blockDim.x) {
        const int64_t e = boff + loc;
        const Amp A = decode_amp(P, b, (int)(loc / nc), (int)(loc % nc));
        const int rb = P.ppos[(int64_t)b * L3 + P.pmom[A.mb]] * 16 + A.sb * 4 + A.sa;
        const int cj = P.hpos[(int64_t)b * L3 + P.hmom[A.mj]] * 16 + A.sj * 4 + A.si;
        const F* Hb = H + A.off;
        const F x_abij = Hb[loc], x_baij = Hb[(int64_t)rb * nc + A.c];
        const F x_abji = Hb[(int64_t)A.r * nc + cj], x_baji = Hb[(int64_t)rb * nc + cj];
        const F v = F(0.25) * ((x_abij - x_baij) - (x_abji - x_baji));
        const F den = -((Xpp[A.ma * 16 + A.sa * 5] + Xpp[A.mb * 16 + A.sb * 5]) +
                             (Xhh[A.mi * 16 + A.si * 5] + Xhh[A.mj * 16 + A.sj * 5]));
        const F t = t2[e];
        const F tn = t + v / den;
        const F o = F(mixing) * t + F(1.0 - mixing) * tn;
        out[e] = o;
        if (err) err[e] = o - t;
    }
}

bool pw_ok(const nlb_pw_problem* P) {
    return P && P->L > 0 && P->n_blocks > 0 && P->n_pmom > 0 && P->n_hmom > 0 && P->n_t2 > 0 && P->n_m > 0 &&
           P->n_w > 0 && P->n_rows > 0 && P->blk_off &&
           P->m_off && P->w_off && P->row_off && P->blk_nr && P->blk_nc && P->blk_K && P->blk_pm0 && P->blk_hm0 &&
           P->pm_list && P->hm_list && P->ppos && P->hpos && P->kblk && P->pmom && P->hmom && P->pinv && P->hinv &&
           P->V && P->fpp && P->fhh && (P->n_tiles == 0 || P->tiles);
}

// The energy and step entry points for amplitudes and intermediates of type
// F (every buffer of S except `energy`, which is FP64, holds F values).
template <typename F>
int pw_energy(const nlb_pw_problem* P, const F* t2, nlb_pw_state* S, cudaStream_t st, const char* name) {
    if (!pw_ok(P) || !t2 || !S || !S->M || !S->Y || !S->energy) return pfail(NLB_ERR_ARG, name);
    F* M = static_cast<F*>(S->M);
    k_pw_M<F><<<pgrid(32 * P->n_m), 256, 0, st>>>(*P, t2, M);
    // the FP64 partial sums go to S->Y (rebuilt from t2 by every step
    // before use): 4 * n_rows values of F hold 4 * n_rows * sizeof(F) / 8
    int64_t nparts = 4 * P->n_rows * (int64_t)sizeof(F) / 8;
    if (nparts > kPwEnergyParts) nparts = kPwEnergyParts;
    if (nparts > P->n_m) nparts = P->n_m;
    if (nparts < 1) nparts = 1;
    double* part = static_cast<double*>(S->Y);
    k_pw_energy_part<F><<<(unsigned)nparts, 256, 0, st>>>(*P, M, part);
    k_pw_energy_sum<<<1, 256, 0, st>>>(part, (int)nparts, S->energy);
    return pcheck(name);
}

template <typename F>
int pw_step(const nlb_pw_problem* P, const F* t2, F* t2_out, F* err, double mixing, nlb_pw_state* S, cudaStream_t st,
            const char* name) {
    if (!pw_ok(P) || !t2 || !t2_out || t2 == t2_out || !S || !S->M || !S->W || !S->Y || !S->Xpp || !S->Xhh || !S->R ||
        !S->U || !S->G || !S->H)
        return pfail(NLB_ERR_ARG, name);
    if (P->n_blocks > 65535) return pfail(NLB_ERR_SIZE, "momentum step: more than 65535 momentum blocks");
    F *M = static_cast<F*>(S->M), *W = static_cast<F*>(S->W), *Y = static_cast<F*>(S->Y);
    F *Xpp = static_cast<F*>(S->Xpp), *Xhh = static_cast<F*>(S->Xhh), *R = static_cast<F*>(S->R);
    F *U = static_cast<F*>(S->U), *G = static_cast<F*>(S->G), *H = static_cast<F*>(S->H);
    const int64_t nph = (int64_t)(4 * P->n_pmom) * (4 * P->n_hmom);
    k_pw_xrow<F><<<pgrid(32 * P->n_rows), 256, 0, st>>>(*P, t2, Y);
    k_pw_X<F><<<pgrid(32 * 16 * (int64_t)(P->n_pmom + P->n_hmom)), 256, 0, st>>>(*P, Y, M, Xpp, Xhh);
    k_pw_W<F><<<pgrid(P->n_w), 256, 0, st>>>(*P, M, W);
    k_pw_R<F><<<pgrid(nph), 256, 0, st>>>(*P, t2, R, U, G);
    int rc = pcheck(name);
    if (rc != NLB_OK) return rc;
    if (P->n_tiles > 0)
        k_pw_residual<F><<<P->n_tiles < 65535 ? P->n_tiles : 65535, 256, 0, st>>>(*P, t2, M, W, Xpp, Xhh, R, U, G, H);
    int64_t gx = 2 * ((P->n_t2 / P->n_blocks + 255) / 256);
    gx = gx < 1 ? 1 : (gx > 64 ? 64 : gx);
    k_pw_jacobi<F><<<dim3((unsigned)gx, (unsigned)P->n_blocks), 256, 0, st>>>(*P, t2, H, Xpp, Xhh, mixing, t2_out,
                                                                            err);
    return pcheck(name);
}

}  // namespace

extern "C" {

int nlb_pw_init(const nlb_pw_problem* P, double* t2, double delta, nlb_stream_t stream) {
    if (!pw_ok(P) || !t2) return pfail(NLB_ERR_ARG, "nlb_pw_init: bad argument");
    k_pw_init<<<pgrid(P->n_t2), 256, 0, (cudaStream_t)stream>>>(*P, t2, delta);
    return pcheck("nlb_pw_init");
}

int nlb_pw_energy(const nlb_pw_problem* P, const double* t2, nlb_pw_state* S, nlb_stream_t stream) {
    return pw_energy<double>(P, t2, S, (cudaStream_t)stream, "nlb_pw_energy");
}

int nlb_pw_step(const nlb_pw_problem* P, const double* t2, double* t2_out, double* err, double mixing,
                nlb_pw_state* S, nlb_stream_t stream) {
    return pw_step<double>(P, t2, t2_out, err, mixing, S, (cudaStream_t)stream, "nlb_pw_step");
}

int nlb_pw_energy_f32(const nlb_pw_problem* P, const float* t2, nlb_pw_state* S, nlb_stream_t stream) {
    return pw_energy<float>(P, t2, S, (cudaStream_t)stream, "nlb_pw_energy_f32");
}

int nlb_pw_step_f32(const nlb_pw_problem* P, const float* t2, float* t2_out, float* err, double mixing,
                    nlb_pw_state* S, nlb_stream_t stream) {
    return pw_step<float>(P, t2, t2_out, err, mixing, S, (cudaStream_t)stream, "nlb_pw_step_f32");
}

}  // extern "C"
