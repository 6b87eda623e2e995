// Tensor-core contraction for the general (dense) engine, sm_100a.
//
// The ring, quadratic and dense-ladder diagrams of CCM/ccDgrams.py
// (dgram_bkcj_acik :253-264, dgram_cdkl_acik_dblj :279-290, dgram_cdkl_cdij_abkl
// :292-303, dgram_acik_bcjk :359-370, dgram_cdkl_ci_bl_adkj :474-487, and the
// v_pppp ladders of a rotated basis) are pairwise contractions that the
// general engine gathers into row-major panels (nlb_contract_gemm_f64).  In
// the mixed-precision phase of a solve they run here instead of the FP64
// library GEMM:
//
//   C = A B  with  A ~ A_hi + A_lo, B ~ B_hi + B_lo (TF32 parts of the FP32
//   values) and  C ~ A_hi B_hi + A_hi B_lo + A_lo B_hi  (3xTF32),
//
// accumulated in FP32 in tensor memory.  One CTA computes a 128 x 128 tile of
// C: one thread issues the TMA loads of the four operand panels (SWIZZLE_128B,
// K-major, 32 TF32 values per row), one thread issues the tcgen05.mma
// instructions (kind::tf32, M=128, N=128, K=8) and commits each stage back to
// the loader, and the four warps read the accumulator out of tensor memory
// with tcgen05.ld.  The operand tensor maps cover this GPU's own work buffer
// only; no load is multicast.
//
// Every wait on an mbarrier is bounded (2 s of the global timer): a wait that
// runs out records an error in the work buffer's flag word, the CTA stops
// issuing work, waits (bounded) for the copies it already issued, frees its
// tensor memory and returns; the write-back then fills the output with NaN.

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include "nulattice_b200.h"

void nlb_internal_set_error(const char* msg);

namespace {

constexpr int kBM = 128, kBN = 128, kBK = 32;     // tile; kBK TF32 values = one 128-byte row
constexpr int kStages = 3;
constexpr int kPanelBytes = kBM * kBK * 4;         // one operand panel of a stage (16 KB)
constexpr int kStageBytes = 4 * kPanelBytes;       // A_hi, A_lo, B_hi, B_lo
constexpr int kThreads = 128;
constexpr uint64_t kWaitNs = 2000000000ull;        // bound of every mbarrier wait (2 s)

// ------------------------------------------------------------ PTX wrappers --
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// Wait for the phase of the given parity to complete; false when it has not
// completed within kWaitNs (a bound on wall time, so that threads that wait
// through a long product loop are not cut short).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    const uint32_t a = smem_u32(bar);
    const uint64_t t0 = global_ns();
    for (uint32_t it = 0;; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
        if ((it & 255) == 255 && global_ns() - t0 > kWaitNs) return false;
    }
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
        ::"r"(smem_u32(dst)), "l"(map), "r"(smem_u32(bar)), "r"(x), "r"(y)
        : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Shared-memory matrix descriptor of a K-major operand panel loaded by TMA
// with SWIZZLE_128B: rows of 128 bytes, groups of eight rows 1024 bytes
// apart (stride byte offset), leading byte offset unused for this layout,
// descriptor version 1, layout type 2 = SWIZZLE_128B.
__device__ __forceinline__ uint64_t panel_desc(uint32_t addr) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);          // start address, bits [0,14)
    d |= (uint64_t)1 << 16;                          // leading byte offset (16 B units)
    d |= (uint64_t)(1024 >> 4) << 32;                // stride byte offset, bits [32,46)
    d |= (uint64_t)1 << 46;                          // version
    d |= (uint64_t)2 << 61;                          // SWIZZLE_128B
    return d;
}

// Instruction descriptor of tcgen05.mma kind::tf32: FP32 accumulator, TF32
// A and B, both K-major, N = kBN, M = kBM.
constexpr uint32_t kIdesc = (1u << 4)                 // c_format F32
                            | (2u << 7)               // a_format TF32
                            | (2u << 10)              // b_format TF32
                            | ((uint32_t)(kBN >> 3) << 17)
                            | ((uint32_t)(kBM >> 4) << 24);

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(tmem_d), "l"(da), "l"(db), "r"(kIdesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// 32 consecutive accumulator columns of this warp's 32 lanes (one row per lane).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
}

__device__ __forceinline__ float to_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

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

// Gather one operand of the contraction into the padded K-major panels the
// tensor cores read, split into TF32 parts: hi = tf32(x), lo = tf32(x - hi)
// with x the FP32 value.  which = 0: A[m][k] (rows m); 1: B as [n][k].
// Rows beyond the operand and columns beyond K are zero.
// 32 x 32 tiles through shared memory: the row and column offsets are
// decoded once per tile, and the strided side is read (or written) along
// its contiguous index.  `*_fast`: the row index (pack: m or n; write-back:
// m) is the contiguous one of the strided side.
constexpr int kPT = 32;
constexpr int kGroupM = 8;   // tile rows per group of the GEMM's tile order

__global__ void __launch_bounds__(256) k_split_pack_t(const double* __restrict__ src, float* __restrict__ hi,
                                                      float* __restrict__ lo, int64_t rows, int64_t rows_pad,
                                                      int64_t cols, int64_t cols_pad, nlb_contract_desc d,
                                                      int which, int rows_fast) {
    __shared__ int64_t roff[kPT], coff[kPT];
    __shared__ float tile[kPT][kPT + 1];
    const int64_t r0 = (int64_t)blockIdx.y * kPT, c0 = (int64_t)blockIdx.x * kPT;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    if (threadIdx.x < kPT) {
        const int64_t r = r0 + threadIdx.x;
        roff[threadIdx.x] = r < rows ? (which == 0 ? decode(r, d.ext_m, d.sa_m, d.nm) : decode(r, d.ext_n, d.sb_n, d.nn))
                                     : 0;
    } else if (threadIdx.x < 2 * kPT) {
        const int q = threadIdx.x - kPT;
        const int64_t c = c0 + q;
        coff[q] = c < cols ? (which == 0 ? decode(c, d.ext_k, d.sa_k, d.nk) : decode(c, d.ext_k, d.sb_k, d.nk)) : 0;
    }
    __syncthreads();
    for (int i = ty; i < kPT; i += 8) {
        const int rr = rows_fast ? tx : i, cc = rows_fast ? i : tx;
        const int64_t r = r0 + rr, c = c0 + cc;
        tile[rr][cc] = (r < rows && c < cols) ? (float)src[roff[rr] + coff[cc]] : 0.f;
    }
    __syncthreads();
    for (int i = ty; i < kPT; i += 8) {
        const int64_t r = r0 + i, c = c0 + tx;
        if (r < rows_pad && c < cols_pad) {
            const float x = tile[i][tx];
            const float h = to_tf32(x);
            hi[r * cols_pad + c] = h;
            lo[r * cols_pad + c] = to_tf32(x - h);
        }
    }
}

// C = alpha * P + beta * C with the tile results written back into the
// strided output; P holds `splits` partial slices [M_pad][N_pad] (split-K),
// added in slice order in FP64.  When a tile reported a failed wait (*err)
// every output entry becomes NaN, so the failure cannot pass unnoticed.
__global__ void __launch_bounds__(256) k_unpack_tile_t(const float* __restrict__ P, int64_t m_pad, int64_t n_pad,
                                                       int splits, double* __restrict__ C, nlb_contract_desc d,
                                                       double alpha, double beta, const int* err, int m_fast) {
    __shared__ int64_t moff[kPT], noff[kPT];
    __shared__ double tile[kPT][kPT + 1];
    const int64_t m0 = (int64_t)blockIdx.y * kPT, n0 = (int64_t)blockIdx.x * kPT;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const bool bad = *err != 0;
    if (threadIdx.x < kPT) {
        const int64_t m = m0 + threadIdx.x;
        moff[threadIdx.x] = m < d.M ? decode(m, d.ext_m, d.sc_m, d.nm) : 0;
    } else if (threadIdx.x < 2 * kPT) {
        const int q = threadIdx.x - kPT;
        const int64_t n = n0 + q;
        noff[q] = n < d.N ? decode(n, d.ext_n, d.sc_n, d.nn) : 0;
    }
    for (int i = ty; i < kPT; i += 8) {
        const int64_t m = m0 + i, n = n0 + tx;
        double acc = 0.0;
        if (m < d.M && n < d.N)
            for (int s = 0; s < splits; ++s) acc += (double)P[(int64_t)s * m_pad * n_pad + m * n_pad + n];
        tile[i][tx] = alpha * acc;
    }
    __syncthreads();
    for (int i = ty; i < kPT; i += 8) {
        const int mm = m_fast ? tx : i, nn = m_fast ? i : tx;
        const int64_t m = m0 + mm, n = n0 + nn;
        if (m < d.M && n < d.N) {
            const int64_t off = moff[mm] + noff[nn];
            const double v = tile[mm][nn];
            C[off] = bad ? __longlong_as_double(0x7ff8000000000000LL) : ((beta == 0.0) ? v : v + beta * C[off]);
        }
    }
}

// One 128 x 128 tile of P = A B^T (A: [M_pad][K_pad], B: [N_pad][K_pad],
// both as TF32 hi/lo panels), over K blocks [kb0, kb0 + n_kblocks) of split
// blockIdx.z, into that split's slice of P.  Warp 0 allocates tensor memory
// and its lane 0 loads; warp 1 lane 0 issues the products; all four warps
// drain the accumulator.  *err receives 1 when a bounded wait ran out.
__global__ void __launch_bounds__(kThreads, 1)
    k_gemm_tf32x3(const __grid_constant__ CUtensorMap mAh, const __grid_constant__ CUtensorMap mAl,
                  const __grid_constant__ CUtensorMap mBh, const __grid_constant__ CUtensorMap mBl, int kb_total,
                  int kb_per_split, float* __restrict__ P, int64_t m_pad, int64_t n_pad, int* err) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    // 1024-byte alignment of the stage panels (SWIZZLE_128B pattern repeat)
    unsigned char* base = reinterpret_cast<unsigned char*>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    __shared__ __align__(8) uint64_t full[kStages], empty[kStages], accum;
    __shared__ uint32_t tmem_base;
    __shared__ int failed;
    __shared__ int n_issued, n_consumed;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // tile order: groups of kGroupM tile rows, the tile columns of a group
    // in turn, so that a wave of CTAs shares a few A panels and B panels
    // that stay in L2 (the plain raster order streams every B panel per row)
    int tm, tn;
    {
        const int tiles_m = gridDim.x, tiles_n = gridDim.y;
        const int lin = blockIdx.y * tiles_m + blockIdx.x;
        const int per_group = kGroupM * tiles_n;
        const int first_m = (lin / per_group) * kGroupM;
        const int gsize = min(tiles_m - first_m, kGroupM);
        const int in_group = lin % per_group;
        tm = first_m + in_group % gsize;
        tn = in_group / gsize;
    }
    const int m0 = tm * kBM, n0 = tn * kBN;
    const int kb0 = blockIdx.z * kb_per_split;
    const int n_kblocks = min(kb_per_split, kb_total - kb0);
    P += (int64_t)blockIdx.z * m_pad * n_pad;
    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(&accum, 1);
        failed = 0;
        n_issued = 0;
        n_consumed = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                     "r"(kBN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base;

    if (warp == 0 && lane == 0) {
        // loader: stage s = kb % kStages, reused once the products of its
        // previous use have completed (empty[s])
        int kb = 0;
        for (; kb < n_kblocks; ++kb) {
            const int s = kb % kStages;
            if (kb >= kStages && !mbar_wait(&empty[s], ((kb / kStages) - 1) & 1)) {
                atomicExch(&failed, 1);
                break;
            }
            if (*(volatile int*)&failed) break;
            unsigned char* st = base + s * kStageBytes;
            mbar_expect_tx(&full[s], kStageBytes);
            const int k0 = (kb0 + kb) * kBK;
            tma_load_2d(st, &mAh, &full[s], k0, m0);
            tma_load_2d(st + kPanelBytes, &mAl, &full[s], k0, m0);
            tma_load_2d(st + 2 * kPanelBytes, &mBh, &full[s], k0, n0);
            tma_load_2d(st + 3 * kPanelBytes, &mBl, &full[s], k0, n0);
        }
        n_issued = kb;
    } else if (warp == 1 && lane == 0) {
        // products: per stage 4 K-steps of 8 TF32 values x 3 products
        int kb = 0;
        for (; kb < n_kblocks; ++kb) {
            const int s = kb % kStages;
            if (!mbar_wait(&full[s], (kb / kStages) & 1)) {
                atomicExch(&failed, 1);
                break;
            }
            tc_fence_after();
            const uint32_t st = smem_u32(base + s * kStageBytes);
#pragma unroll
            for (int k = 0; k < kBK / 8; ++k) {
                // K-step k: 8 TF32 values = 32 bytes along the 128-byte rows
                const uint64_t ah = panel_desc(st + k * 32), al = panel_desc(st + kPanelBytes + k * 32);
                const uint64_t bh = panel_desc(st + 2 * kPanelBytes + k * 32);
                const uint64_t bl = panel_desc(st + 3 * kPanelBytes + k * 32);
                const uint32_t acc0 = (kb > 0 || k > 0) ? 1u : 0u;
                mma_tf32(tmem, al, bh, acc0);   // small terms first
                mma_tf32(tmem, ah, bl, 1u);
                mma_tf32(tmem, ah, bh, 1u);
            }
            mma_commit(&empty[s]);        // the stage is free once these products have read it
        }
        n_consumed = kb;
        mma_commit(&accum);               // every product issued so far has completed
    }
    __syncthreads();
    // epilogue: warp w holds accumulator lanes (rows) 32w .. 32w + 31
    bool ok = mbar_wait(&accum, 0);
    if (!ok) atomicExch(&failed, 1);
    tc_fence_after();
    if (ok && !*(volatile int*)&failed) {
        const int row = m0 + warp * 32 + lane;
        float* prow = P + (int64_t)row * n_pad + n0;
#pragma unroll 1
        for (int c = 0; c < kBN / 32; ++c) {
            float v[32];
            tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(c * 32), v);
#pragma unroll
            for (int j = 0; j < 32; j += 4)
                *reinterpret_cast<float4*>(prow + c * 32 + j) = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0 && failed) {
        // copies issued but never consumed: let them land before the CTA
        // (and its shared memory) goes away
        for (int kb = n_consumed; kb < n_issued; ++kb) mbar_wait(&full[kb % kStages], (kb / kStages) & 1);
        atomicExch(err, 1);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kBN));
}

int gfail(int code, const char* msg) {
    nlb_internal_set_error(msg);
    return code;
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

// Tensor map of a K-major panel [rows][k_pad] FP32, box kBK x 128 rows, SWIZZLE_128B.
bool panel_map(CUtensorMap* m, float* base, int64_t rows, int64_t k_pad) {
    auto fn = encode_fn();
    if (!fn) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)k_pad, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)(k_pad * 4)};
    const cuuint32_t box[2] = {(cuuint32_t)kBK, (cuuint32_t)kBM};
    const cuuint32_t estr[2] = {1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
              CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

int64_t round_up(int64_t x, int64_t q) { return (x + q - 1) / q * q; }

int sm_count() {
    static int n = 0;
    if (n == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 148;
    }
    return n;
}

struct GemmLayout {
    int64_t mp, np, kp;
    int splits, kb_per_split;
    int64_t ah, al, bh, bl, p, err, total;   // byte offsets in the work buffer
};

// Tiles of 128 x 128; when they are fewer than the SMs, K is split so that
// about one CTA runs per SM (each split at least four K blocks).
GemmLayout gemm_layout(const nlb_contract_desc* d) {
    GemmLayout g;
    g.mp = round_up(d->M, kBM);
    g.np = round_up(d->N, kBN);
    g.kp = round_up(d->K, kBK);
    const int64_t tiles = (g.mp / kBM) * (g.np / kBN);
    const int64_t kblocks = g.kp / kBK;
    int64_t splits = sm_count() / (tiles > 0 ? tiles : 1);
    if (splits > kblocks / 4) splits = kblocks / 4;
    if (splits > 64) splits = 64;
    if (splits < 1) splits = 1;
    g.kb_per_split = (int)((kblocks + splits - 1) / splits);
    g.splits = (int)((kblocks + g.kb_per_split - 1) / g.kb_per_split);
    g.ah = 0;
    g.al = g.ah + g.mp * g.kp * 4;
    g.bh = g.al + g.mp * g.kp * 4;
    g.bl = g.bh + g.np * g.kp * 4;
    g.p = g.bl + g.np * g.kp * 4;
    g.err = g.p + (int64_t)g.splits * g.mp * g.np * 4;
    g.total = g.err + 256;
    return g;
}

}  // namespace

extern "C" {

int64_t nlb_contract_gemm_tc_work(const nlb_contract_desc* d) {
    if (!d || d->M <= 0 || d->N <= 0 || d->K <= 0) return 0;
    return gemm_layout(d).total;
}

int nlb_contract_gemm_tf32x3(const nlb_contract_desc* d, const double* A, const double* B, double* C, double alpha,
                             double beta, void* work, int64_t work_bytes, nlb_stream_t stream) {
    if (!d || !A || !B || !C || !work) return gfail(NLB_ERR_ARG, "nlb_contract_gemm_tf32x3: null argument");
    if (d->nm > 4 || d->nn > 4 || d->nk > 4 || d->nm < 0 || d->nn < 0 || d->nk < 0 || d->nb != 0 || d->B != 1)
        return gfail(NLB_ERR_ARG, "nlb_contract_gemm_tf32x3: no batch indices, at most 4 indices per group");
    if (d->M <= 0 || d->N <= 0 || d->K <= 0) return gfail(NLB_ERR_SIZE, "nlb_contract_gemm_tf32x3: empty GEMM");
    if (((uintptr_t)work & 255) != 0) return gfail(NLB_ERR_ARG, "nlb_contract_gemm_tf32x3: work not 256-byte aligned");
    const GemmLayout g = gemm_layout(d);
    if (work_bytes < g.total) return gfail(NLB_ERR_SIZE, "nlb_contract_gemm_tf32x3: workspace too small");
    if (g.mp / kBM > 0x7fffffff || g.np / kBN > 65535 || g.kp > 0x7fffffff)
        return gfail(NLB_ERR_SIZE, "nlb_contract_gemm_tf32x3: GEMM too large");
    unsigned char* w = static_cast<unsigned char*>(work);
    float *ah = reinterpret_cast<float*>(w + g.ah), *al = reinterpret_cast<float*>(w + g.al);
    float *bh = reinterpret_cast<float*>(w + g.bh), *bl = reinterpret_cast<float*>(w + g.bl);
    float* P = reinterpret_cast<float*>(w + g.p);
    int* err = reinterpret_cast<int*>(w + g.err);
    cudaStream_t st = (cudaStream_t)stream;
    CUtensorMap maps[4];
    if (!panel_map(&maps[0], ah, g.mp, g.kp) || !panel_map(&maps[1], al, g.mp, g.kp) ||
        !panel_map(&maps[2], bh, g.np, g.kp) || !panel_map(&maps[3], bl, g.np, g.kp))
        return gfail(NLB_ERR_CUDA, "nlb_contract_gemm_tf32x3: cuTensorMapEncodeTiled failed");
    const int smem = kStages * kStageBytes + 1024;
    static bool attr[64] = {};   // once per device
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64 || !attr[dev]) {
        if (cudaFuncSetAttribute(k_gemm_tf32x3, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess)
            return gfail(NLB_ERR_CUDA, "nlb_contract_gemm_tf32x3: shared-memory attribute");
        if (dev >= 0 && dev < 64) attr[dev] = true;
    }
    cudaMemsetAsync(err, 0, sizeof(int), st);
    // the contiguous (innermost) index of each group: last in the decode order
    auto unit = [](const int64_t* str, int nd) { return nd > 0 && str[nd - 1] == 1; };
    const int a_rows_fast = unit(d->sa_m, d->nm) && !unit(d->sa_k, d->nk);
    const int b_rows_fast = unit(d->sb_n, d->nn) && !unit(d->sb_k, d->nk);
    const int c_m_fast = unit(d->sc_m, d->nm) && !unit(d->sc_n, d->nn);
    if (g.mp / kPT > 65535 || g.np / kPT > 65535 || (d->M + kPT - 1) / kPT > 65535)
        return gfail(NLB_ERR_SIZE, "nlb_contract_gemm_tf32x3: too many row tiles");
    k_split_pack_t<<<dim3((unsigned)(g.kp / kPT), (unsigned)(g.mp / kPT)), 256, 0, st>>>(A, ah, al, d->M, g.mp, d->K,
                                                                                      g.kp, *d, 0, a_rows_fast);
    k_split_pack_t<<<dim3((unsigned)(g.kp / kPT), (unsigned)(g.np / kPT)), 256, 0, st>>>(B, bh, bl, d->N, g.np, d->K,
                                                                                      g.kp, *d, 1, b_rows_fast);
    const dim3 grid((unsigned)(g.mp / kBM), (unsigned)(g.np / kBN), (unsigned)g.splits);
    k_gemm_tf32x3<<<grid, kThreads, smem, st>>>(maps[0], maps[1], maps[2], maps[3], (int)(g.kp / kBK),
                                                 g.kb_per_split, P, g.mp, g.np, err);
    k_unpack_tile_t<<<dim3((unsigned)((d->N + kPT - 1) / kPT), (unsigned)((d->M + kPT - 1) / kPT)), 256, 0, st>>>(
        P, g.mp, g.np, g.splits, C, *d, alpha, beta, err, c_m_fast);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        char buf[256];
        snprintf(buf, sizeof(buf), "nlb_contract_gemm_tf32x3: %s", cudaGetErrorString(e));
        nlb_internal_set_error(buf);
        return NLB_ERR_LAUNCH;
    }
    return NLB_OK;
}

}  // extern "C"
