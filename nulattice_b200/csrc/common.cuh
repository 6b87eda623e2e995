// Device helpers shared by the structured kernels (ccsd_struct.cu) and the
// adjoint kernels (lambda.cu).  Included inside an anonymous namespace.
#pragma once

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
// Layout of the prep scratch (doubles), see nlb_struct_prep_len:
//   Q[h*h]   Q[k,j] = sum_c f_ck t1_cj
//   Xh2[h*h] X_hh of the T2 equation, -f_hh - Q      (coupled_cluster.py:505-513)
//   Xh1[h*h] X_hh of the T1 equation, -f_hh - Q/2    (coupled_cluster.py:388-393)
//   dXp2[p], dXp1[p]  diagonals of X_pp: f_aa - S_a, f_aa - S_a/2, S_a = sum_k f_ak t1_ak
//   t1c[n_t1c]  t1[P_g[a'], H_g[k']] per label (a' major)
//   xc[n_xc]    Xh2[H_g[k'], H_g[i']] per label (k' major)
//   dpc[p]      dXp2 in label order
//   dhc[h]      diag Xh2 in label order
//   red[kRedLen] per-block partial sums of the reductions of a step (below)
//
// Reductions are deterministic: a kernel that reduces over the grid writes
// one partial per block into its own slot range of `red`, and the kernel that
// consumes the total (k_finish, k_l_finish, the DIIS Gram reduction) adds the
// partials in slot order.  No floating-point atomics, so a solve repeats bit
// for bit and its stopping step does not depend on block scheduling.
constexpr int kRedSlots = 2048;            // most blocks of a reducing launch
constexpr int kRedKinds = 4;               // partial arrays of kRedSlots each
constexpr int kGramSlots = 512;            // most blocks of the DIIS Gram launch
constexpr int kGramPairs = 55;             // pairs (s <= t) of at most 10 vectors
constexpr int64_t kRedLen = (int64_t)kRedKinds * kRedSlots + (int64_t)kGramSlots * kGramPairs;
// slot ranges of `red`: the forward step uses E, DT1, DT2; the Lambda step
// uses NRM1 (|lam1|^2), DT1, DT2 and NRM2 (|Lam|^2)
enum { kRedE = 0, kRedNrm1 = 0, kRedDt1 = 1, kRedDt2 = 2, kRedNrm2 = 3 };

struct PrepView {
    double *Q, *Xh2, *Xh1, *dXp2, *dXp1, *t1c, *xc, *dpc, *dhc, *red;
    __host__ __device__ double* slots(int kind) const { return red + (int64_t)kind * kRedSlots; }
    __host__ __device__ double* gram_slots() const { return red + (int64_t)kRedKinds * kRedSlots; }
};

__host__ __device__ inline PrepView prep_view(double* base, const nlb_struct_problem& P) {
    const int64_t hh = (int64_t)P.h * P.h;
    PrepView v;
    v.Q = base;
    v.Xh2 = v.Q + hh;
    v.Xh1 = v.Xh2 + hh;
    v.dXp2 = v.Xh1 + hh;
    v.dXp1 = v.dXp2 + P.p;
    v.t1c = v.dXp1 + P.p;
    v.xc = v.t1c + P.n_t1c;
    v.dpc = v.xc + P.n_xc;
    v.dhc = v.dpc + P.p;
    v.red = v.dhc + P.h;
    return v;
}

// Sum of the first n partials at `part` in a fixed order: lane-strided
// sums, then a fixed butterfly.  Every lane of the (full) warp must call it
// with the same n; all lanes return the same value.
__device__ __forceinline__ double warp_sum_slots(const double* part, int n) {
    double s = 0.0;
    for (int b = (int)(threadIdx.x & 31); b < n; b += 32) s += part[b];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    return s;
}

__device__ __forceinline__ int find_label(const int32_t* base, int G, int64_t u) {
    int lo = 0, hi = G - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (u >= base[mid]) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// Q[k,i] = sum_c f_ck t1_ci using the f_ph column list of hole k.
__device__ __forceinline__ double q_entry(const nlb_struct_problem& P, const double* t1, int k, int i) {
    // entries in batches of eight whose loads go out together (a lattice
    // hole has at most six particle neighbours); the sum keeps their order
    double q = 0.0;
    if (P.h_row && P.fph_prow) {
        const int row = P.h_row[k];
        const int e0 = P.fph_ptr[row], e1 = P.fph_ptr[row + 1];
        for (int b = e0; b < e1; b += 8) {
            double tv[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) tv[u] = (b + u < e1) ? t1[(int64_t)P.fph_prow[b + u] * P.h + i] : 0.0;
#pragma unroll
            for (int u = 0; u < 8; ++u)
                if (b + u < e1) q += P.fph_val[b + u] * tv[u];
        }
        return q;
    }
    const int g = P.h_label[k];
    const int row = P.h_base[g] + P.h_loc[k];
    const int pb = P.p_base[g];
    const int e0 = P.fph_ptr[row], e1 = P.fph_ptr[row + 1];
    for (int b = e0; b < e1; b += 8) {
        double tv[8];
#pragma unroll
        for (int u = 0; u < 8; ++u)
            tv[u] = (b + u < e1) ? t1[(int64_t)P.p_ord[pb + P.fph_col[b + u]] * P.h + i] : 0.0;
#pragma unroll
        for (int u = 0; u < 8; ++u)
            if (b + u < e1) q += P.fph_val[b + u] * tv[u];
    }
    return q;
}

__device__ __forceinline__ double s_entry(const nlb_struct_problem& P, const double* t1, int a) {
    // loads in batches of eight that go out together; the sum keeps the order
    const double* f = P.f_ph + (int64_t)a * P.h;
    const double* t = t1 + (int64_t)a * P.h;
    double s = 0.0;
    for (int k = 0; k < P.h; k += 8) {
        double fv[8], tv[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            fv[u] = (k + u < P.h) ? f[k + u] : 0.0;
            tv[u] = (k + u < P.h) ? t[k + u] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 8; ++u)
            if (k + u < P.h) s += fv[u] * tv[u];
    }
    return s;
}

// One thread of the prep tables (layout above) at amplitudes t1.
__device__ void prep_body(const nlb_struct_problem& P, const double* t1, double* prep, int64_t u) {
    const int h = P.h, p = P.p, G = P.n_labels;
    const PrepView V = prep_view(prep, P);
    const int64_t hh = (int64_t)h * h;
    if (u < hh) {
        const int k = (int)(u / h), j = (int)(u % h);
        const double q = q_entry(P, t1, k, j);
        V.Q[u] = q;
        V.Xh2[u] = -P.f_hh[u] - q;
        V.Xh1[u] = -P.f_hh[u] - 0.5 * q;
        return;
    }
    u -= hh;
    if (u < p) {
        const double s = s_entry(P, t1, (int)u);
        V.dXp2[u] = P.fpp_diag[u] - s;
        V.dXp1[u] = P.fpp_diag[u] - 0.5 * s;
        return;
    }
    u -= p;
    if (u < P.n_t1c) {
        if (P.t1c_idx) {
            V.t1c[u] = t1[P.t1c_idx[u]];
            return;
        }
        const int g = find_label(P.t1c_base, G, u);
        const int nh = P.h_base[g + 1] - P.h_base[g];
        const int loc = (int)(u - P.t1c_base[g]);
        const int ap = loc / nh, kq = loc - ap * nh;
        V.t1c[u] = t1[(int64_t)P.p_ord[P.p_base[g] + ap] * h + P.h_ord[P.h_base[g] + kq]];
        return;
    }
    u -= P.n_t1c;
    if (u < P.n_xc) {
        if (P.xc_ki) {
            const int ki = P.xc_ki[u];
            const int k = ki / h, i = ki - k * h;
            V.xc[u] = -P.f_hh[ki] - q_entry(P, t1, k, i);
            return;
        }
        const int g = find_label(P.xc_base, G, u);
        const int nh = P.h_base[g + 1] - P.h_base[g];
        const int loc = (int)(u - P.xc_base[g]);
        const int kq = loc / nh, iq = loc - kq * nh;
        const int k = P.h_ord[P.h_base[g] + kq], i = P.h_ord[P.h_base[g] + iq];
        V.xc[u] = -P.f_hh[(int64_t)k * h + i] - q_entry(P, t1, k, i);
        return;
    }
    u -= P.n_xc;
    if (u < p) {
        const int a = P.p_ord[u];
        V.dpc[u] = P.fpp_diag[a] - s_entry(P, t1, a);
        return;
    }
    u -= p;
    if (u < h) {
        const int i = P.h_ord[u];
        V.dhc[u] = -P.f_hh[(int64_t)i * h + i] - q_entry(P, t1, i, i);
    }
}


// Ga[k'][b'][i'j'] = sum_c f_ck B[c'][b'][i'j'] (k = hole k' of label g1) at
// flat index e of the Ga array: the f_ph^T t2 half-contraction along the
// first particle index.  With t1 it gives the rank-h part of X_pp t2 along a,
// and it holds the T1 Fock term f_ck t2_acik for particles of label g2.
template <typename T>
__device__ __forceinline__ T ga_element(const nlb_struct_problem& P, const T* B, int64_t e) {
    const int ci = find_seg(P.g_end, P.n_channels, e);
    const nlb_channel& ch = P.chan[ci];
    const int rowlen = ch.np2 * ch.nh1 * ch.nh2;
    const int loc = (int)(e - ch.ga_off);
    const int kq = loc / rowlen, rem = loc - kq * rowlen;
    const int row = ch.hb1 + kq;
    const T* Bc = B + ch.offset + rem;
    T acc = T(0);
    for (int q = P.fph_ptr[row]; q < P.fph_ptr[row + 1]; ++q) acc += (T)P.fph_val[q] * Bc[(int64_t)P.fph_col[q] * rowlen];
    return acc;
}

__host__ __device__ inline int64_t lat_round16(int64_t b) { return (b + 15) & ~int64_t(15); }

// Work units of channel cc for the row kernels that split rows by b'
// columns: max(np2, 1) per row (a row with no columns still is one unit, so
// that its per-row outputs get a writer).
__device__ __forceinline__ int64_t lat_units(const nlb_struct_problem& P, int cc) {
    const nlb_channel& c = P.chan[cc];
    return (int64_t)c.np1 * (c.np2 > 0 ? c.np2 : 1);
}

// Asynchronous global -> shared copies (cp.async) and vector loads of
// 16-byte aligned shared-memory records.
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}

template <int N>
__device__ __forceinline__ void cp_async_el(void* dst, const void* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(d), "l"(src), "n"(N) : "memory");
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Eight consecutive shared-memory values (16-byte aligned) with vector loads.
__device__ __forceinline__ void lds8(const float* p, float (&v)[8]) {
    const float4 a = reinterpret_cast<const float4*>(p)[0], b = reinterpret_cast<const float4*>(p)[1];
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w; v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
}
__device__ __forceinline__ void lds8(const double* p, double (&v)[8]) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const double2 a = reinterpret_cast<const double2*>(p)[k];
        v[2 * k] = a.x; v[2 * k + 1] = a.y;
    }
}
__device__ __forceinline__ void lds8(const int32_t* p, int (&v)[8]) {
    const int4 a = reinterpret_cast<const int4*>(p)[0], b = reinterpret_cast<const int4*>(p)[1];
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w; v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
}


// Jacobi quotient R / D.  FP32 amplitudes: the approximate reciprocal (the
// denominators only set the step length, the fixed point R = 0 does not
// depend on them); FP64: IEEE division.
__device__ __forceinline__ float lat_div(float r, float d) { return __fdividef(r, d); }
__device__ __forceinline__ double lat_div(double r, double d) { return r / d; }

