/*
 * nulattice_b200 -- C ABI of the B200 CCSD kernels.
 *
 * The reference (NuLattice) is pure Python and has no FFI: its CCSD entry
 * point is the Python function `ccsd_solver` (CCM/coupled_cluster.py:547-687,
 * torch twin CCM/soa/coupled_cluster.py:440-575).  The Python package
 * `nulattice_b200` mirrors that function and calls the entry points below
 * through ctypes; every comment names the reference code whose work the
 * entry point takes over.
 *
 * Conventions
 *  - Every pointer is a device pointer unless its name ends in `_host`.
 *  - No entry point allocates device memory: the caller owns every buffer
 *    (sizes from the *_bytes queries).  The stream is the caller's.
 *  - Return value: NLB_OK (0) or a positive NLB_ERR_* code; launches are
 *    asynchronous, so a kernel fault surfaces at the caller's next sync.
 *  - Amplitudes are stored either as FP64 or FP32 (`dtype` = NLB_F64 /
 *    NLB_F32); T1, the energy, norms and the DIIS algebra are always FP64.
 */
#ifndef NULATTICE_B200_H
#define NULATTICE_B200_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef void *nlb_stream_t; /* a cudaStream_t */

enum { NLB_OK = 0, NLB_ERR_ARG = 1, NLB_ERR_LAUNCH = 2, NLB_ERR_SIZE = 3, NLB_ERR_CUDA = 4 };
enum { NLB_F64 = 0, NLB_F32 = 1 };
enum { NLB_RUNNING = 0, NLB_CONVERGED = 1, NLB_MAX_ITER = 2, NLB_DIVERGED = 3 };
enum { NLB_CRIT_SOA = 0, NLB_CRIT_NUMPY = 1 };
/* Stages of one step (nlb_struct_stage): PREP forms the dressed-Fock tables
 * and the Ga intermediates in one launch, GTERMS is kept for compatibility
 * and launches nothing, T2 and T1 update the amplitudes, FINISH tests
 * convergence. */
enum { NLB_STAGE_PREP = 0, NLB_STAGE_GTERMS = 1, NLB_STAGE_T2 = 2, NLB_STAGE_T1 = 3, NLB_STAGE_FINISH = 4 };

/* One channel (label pair g1 < g2) of the compact T2: a dense block
 * B[a'][b'][i'][j'] of np1*np2*nh1*nh2 numbers at element `offset`.  A "row"
 * is B[a'][:][:] (np2*nh1*nh2 numbers). */
typedef struct {
    int32_t g1, g2, np1, np2, nh1, nh2;
    int32_t pb1, pb2, hb1, hb2;   /* label bases into p_ord / h_ord */
    int64_t offset;               /* element offset in compact T2 */
    int64_t ga_off;               /* offset of Ga[k'][b'][i'j'] (nh1*np2*nh1*nh2) */
    int64_t f2_off;               /* offset of the T1 Fock term F2[a'][i'] (np1*nh1) */
    int64_t hh_ptr_off, hh_col_off, pp_ptr_off, pp_col_off;
} nlb_channel;

/* Structured problem description (closed-site, label-conserving inputs).
 * Built on the host by nulattice_b200.structure; all arrays on the device. */
typedef struct {
    int32_t p, h, n_labels, n_channels;
    int64_t n_t2;                 /* compact T2 length */
    int64_t n_g;                  /* Ga length (sum over channels) */
    int64_t n_f2;                 /* F2 length (sum of np1*nh1) */
    int64_t n_rows;               /* sum of np1: one T2-update task per row */
    int64_t n_t1c, n_xc;          /* compact T1 / X_hh table lengths */
    int32_t max_row;              /* max np2*nh1*nh2 */
    int32_t max_nh;               /* max holes in one label */
    int32_t uniform_nh;           /* every channel has nh1 == nh2 == this (0: not uniform) */
    int32_t diag_ladders;         /* 1: both ladders only couple a pair to itself */
    int32_t max_fpp_offdiag;      /* most off-diagonal entries in one f_pp row */
    int32_t tune;                 /* launch shapes, 0 = defaults (threads x resident blocks/SM):
                                     bits 0-3 lattice T2 kernel, FP32 (0 256x2, 1 512x1, 2 384x1;
                                       packed FP32x2 sums: 3 512x1, 4 384x1; two rows per
                                       pass: 5 256x1, 6 384x1, 7 448x1, 8 512x1);
                                     bits 4-7 lattice Lambda row pass, FP32 (0 256x2, 1 512x1);
                                     bits 8-15 Lambda column-pass row chunks (0: automatic);
                                     bits 16-19 lattice T2 kernel, FP64 (0 512x1, 1 256x1) */
    const nlb_channel *chan;      /* [n_channels] */
    const int64_t *t2_end;        /* [n_channels] cumulative end of each block */
    const int64_t *g_end;         /* [n_channels] cumulative end of Ga blocks */
    const int64_t *row_end;       /* [n_channels] cumulative row count */
    const int32_t *t1c_base;      /* [n_labels+1] offsets of t1[P_g, H_g] tables */
    const int32_t *xc_base;       /* [n_labels+1] offsets of X_hh[H_g, H_g] tables */
    const int32_t *p_ord;         /* [p] particle index of label-ordered row */
    const int32_t *h_ord;         /* [h] */
    const int32_t *p_label, *h_label, *p_loc, *h_loc;   /* [p], [h], [p], [h] */
    const int32_t *p_base, *h_base;                     /* [n_labels+1] */
    const int32_t *fpp_ptr, *fpp_col; const double *fpp_val;  /* f_pp CSR per label */
    const double *fpp_diag;       /* [p] */
    const int32_t *fph_ptr, *fph_col; const double *fph_val;  /* f_ph per hole */
    const double *f_ph;           /* [p*h] dense */
    const double *f_hh;           /* [h*h] dense */
    const int32_t *hh_ptr, *hh_col; const double *hh_val;     /* hole-hole ladder CSR */
    const int32_t *pp_ptr, *pp_col; const double *pp_val;     /* particle-particle ladder CSR */
    /* Optional index tables that shorten the chains of dependent loads in
       the step kernels; NULL: the same indices are derived from the tables
       above. */
    const int32_t *h_row;         /* [h] label-ordered f_ph row of hole k: h_base[h_label[k]] + h_loc[k] */
    const int32_t *fph_prow;      /* [nnz f_ph] particle index of each f_ph entry: p_ord[p_base[g] + fph_col] */
    const int32_t *fpp_prow;      /* [nnz f_pp] particle index of each f_pp entry: p_ord[p_base[g] + fpp_col] */
    const int32_t *t1c_idx;       /* [n_t1c] flat t1 index a * h + i of each t1c entry */
    const int32_t *xc_ki;         /* [n_xc] k * h + i (global holes) of each X_hh entry */
} nlb_struct_problem;

/* Device-resident solver state shared by the kernels of one solve. */
typedef struct {
    double e_acc;       /* energy of the amplitudes being written */
    double dt1_sq;      /* ||t1_new - t1||^2 */
    double dt2_sq;      /* ||t2_new - t2||^2 (dense weight applied) */
    double e_prev;      /* energy of the previous step */
    double e_last;      /* energy of the last finished step */
    double eps;
    double mixing;
    double gram[121];   /* DIIS Gram matrix (max_diis <= 10), then coefficients */
    int32_t parity;     /* which amplitude buffer is current */
    int32_t iter;
    int32_t status;
    int32_t max_steps;
    int32_t criterion;  /* NLB_CRIT_SOA / NLB_CRIT_NUMPY */
    int32_t max_diis;
    int32_t diis_count; /* error vectors stored since the last extrapolation */
    int32_t diis_pulse; /* 1 when the step just finished must extrapolate */
    int32_t diis_applied;
    int32_t ccs;
} nlb_ctrl;

/* Per-solve buffers (all caller-allocated). */
typedef struct {
    double *t1[2];      /* [p*h] double-buffered T1 */
    void *t2[2];        /* [n_t2] double-buffered compact T2 (dtype) */
    void *g;            /* [n_g] Ga intermediates (dtype) */
    void *f2;           /* [n_f2] T1 Fock-term partial sums (dtype) */
    double *prep;       /* [nlb_struct_prep_len(prob)] dressed-Fock scratch */
    double *diis_t1;    /* [max_diis * p*h] T1 error ring (may be NULL) */
    void *diis_t2;      /* [max_diis * n_t2] T2 error ring (dtype, may be NULL) */
    nlb_ctrl *ctrl;
    int32_t dtype;
} nlb_struct_state;

int nlb_version(void);
/* human-readable text of the last error set on the calling host thread */
const char *nlb_last_error(void);

/* Length (doubles) of the dressed-Fock scratch: Q, X_hh (T2 eq), X_hh (T1 eq)
 * as h*h each, the particle diagonals of X_pp for both equations, the
 * per-label compact tables t1[P_g,H_g], X_hh[H_g,H_g], diag X_pp, diag X_hh,
 * and the per-block partial sums of the step's reductions (energy, norms,
 * DIIS Gram matrix), which the consuming kernel adds in a fixed order so that
 * every solve repeats bit for bit. */
int64_t nlb_struct_prep_len(const nlb_struct_problem *prob);

/* Dynamic shared memory (bytes) the T2-update kernel needs per block for
 * this problem and dtype; 0 when it exceeds the device limit. */
int64_t nlb_struct_smem_bytes(const nlb_struct_problem *prob, int32_t dtype);

/* Reset `ctrl` on the device and load the solver parameters. */
int nlb_struct_ctrl_init(nlb_ctrl *ctrl, double eps, double mixing, int32_t max_steps,
                         int32_t criterion, int32_t max_diis, int32_t ccs, double e0,
                         nlb_stream_t stream);

/* One CCSD Jacobi step on the compact layout, replacing the reference's
 * t1Iter + t2Iter + mixing + ccsd_energy (CCM/coupled_cluster.py:342-545,
 * 614-623; ccDgrams.py terms that survive for closed-site inputs), followed by
 * the convergence test (coupled_cluster.py:629 / soa/coupled_cluster.py:517).
 * Reads the current buffers (ctrl->parity), writes the other ones, stores the
 * DIIS error vectors when max_diis > 0 and flips ctrl->parity.  Kernels do
 * nothing once ctrl->status != NLB_RUNNING, so steps may be queued ahead. */
int nlb_struct_step(const nlb_struct_problem *prob, const nlb_struct_state *st,
                    nlb_stream_t stream);

/* The five launches of nlb_struct_step one at a time (NLB_STAGE_*), so a
 * caller can bracket a single kernel with events.  Running the stages
 * PREP..FINISH in order is exactly one nlb_struct_step. */
int nlb_struct_stage(const nlb_struct_problem *prob, const nlb_struct_state *st, int32_t stage,
                     nlb_stream_t stream);

/* No counterpart in the reference.  The same step as nlb_struct_step for
 * callers that cannot allocate device memory -- for example an application
 * whose memory manager has already reserved the whole of HBM, or a
 * latency-critical loop where cudaMalloc/cudaFree would synchronise the
 * device.  The caller passes t1, t2, ctrl (and the optional DIIS rings) as
 * usual; st->g, st->f2 and st->prep are ignored.  The step's scratch comes
 * from a fixed 8 MiB array in device memory that every GPU loading this
 * library holds until exit; a problem that needs more (see
 * nlb_struct_noalloc_scratch_bytes) is rejected with NLB_ERR_SIZE, and so is
 * a problem with negative sizes.  The first call on a device looks up the
 * array's device address, so make it before any stream capture.  All calls
 * share the array: calls that overlap on the GPU (other streams, other
 * threads) race and must not be issued.  Nothing is allocated or freed.
 * The step fills the DIIS rings when they are given; the extrapolation
 * (nlb_struct_diis) needs st->prep for its partial sums, while
 * nlb_struct_energy needs no scratch. */
int nlb_struct_step_noalloc(const nlb_struct_problem *prob, const nlb_struct_state *st,
                            nlb_stream_t stream);
/* Bytes of the static scratch nlb_struct_step_noalloc needs for this problem
 * and dtype (-1 on bad arguments). */
int64_t nlb_struct_noalloc_scratch_bytes(const nlb_struct_problem *prob, int32_t dtype);

/* Pulsed DIIS of the torch solver (CCM/soa/coupled_cluster.py:522-567): when
 * ctrl->diis_pulse is set, build the Gram matrix of the stored error vectors
 * (FP64), solve the bordered system in FP64 on the device and extrapolate the
 * current amplitudes in place.  No-op otherwise.  `max_diis` must equal the
 * value given to nlb_struct_ctrl_init (it selects the compiled kernel).
 * Reads t1, t2, the rings, ctrl and the partial-sum area of st->prep; st->g
 * and st->f2 are not used. */
int nlb_struct_diis(const nlb_struct_problem *prob, const nlb_struct_state *st, int32_t max_diis,
                    nlb_stream_t stream);

/* Energy of the current amplitudes, sum_ai f_ai t1_ai (ccsd_energy,
 * coupled_cluster.py:265-286, with v_pphh = 0), written to *e_out (device).
 * Reads t1, f_ph and ctrl only (no scratch). */
int nlb_struct_energy(const nlb_struct_problem *prob, const nlb_struct_state *st,
                      double *e_out, nlb_stream_t stream);

/* Copy between compact T2 of one dtype and another (FP32 <-> FP64). */
int nlb_convert(const void *src, int32_t src_dtype, void *dst, int32_t dst_dtype,
                int64_t n, nlb_stream_t stream);

/* Scatter the compact T2 into the dense reference layout t2[a,b,i,j]
 * (FP64, p*p*h*h, zero-filled by the caller) with all four antisymmetric
 * images, and gather dense -> compact. */
int nlb_struct_unpack_t2(const nlb_struct_problem *prob, const void *t2c, int32_t dtype,
                         double *t2_dense, nlb_stream_t stream);
int nlb_struct_pack_t2(const nlb_struct_problem *prob, const double *t2_dense, void *t2c,
                       int32_t dtype, nlb_stream_t stream);

/* ---------------------------------------------------------------------
 * Adjoint of the structured engine (no counterpart in the reference, which
 * has no gradients): CC Lambda equations at converged amplitudes.
 *
 * Seven holes per label with diagonal ladders (closed-site lattice inputs)
 * take the lattice path: FP32 or FP64 multipliers (dtype), pulsed DIIS on
 * the Jacobi iteration.  Other inputs take the general path (FP64 only).
 * --------------------------------------------------------------------- */
typedef struct {
    double *lam1[2];    /* [p*h] multipliers of the T1 equation (double-buffered, FP64) */
    void *lam2[2];      /* [n_t2] multipliers of the compact T2 equation (dtype) */
    const double *t1;   /* converged t1 [p*h] */
    const void *t2;     /* converged compact t2 [n_t2] (dtype) */
    double *prep;       /* [nlb_struct_prep_len] tables at the converged t1 (filled by init) */
    void *ga;           /* [n_g] Ga of the converged t2 (dtype, filled by init) */
    void *ha;           /* [nlb_lambda_ha_len] scratch (dtype) */
    double *acc;        /* [nlb_lambda_acc_len] scratch; after a step it holds Y1, U, T */
    nlb_ctrl *ctrl;
    void *gb;           /* [nlb_lambda_gb_len] Gb of every row of the converged t2 (dtype, lattice path) */
    double *diis_t1;    /* [max_diis*p*h] DIIS error ring, or NULL without DIIS */
    void *diis_t2;      /* [max_diis*n_t2] (dtype), or NULL */
    int32_t dtype;      /* NLB_F32 or NLB_F64 */
    int32_t reserved;   /* 0 */
} nlb_lambda_state;

#define NLB_LAMBDA_KEEP 1   /* nlb_lambda_init: start from lam1[0], lam2[0] instead of zero */

int64_t nlb_lambda_acc_len(const nlb_struct_problem *prob);
/* Length (elements of the state's dtype) of the `ha` scratch: on the lattice
 * path one slice of n_g per row chunk of the column pass (each slice has one
 * writer per element; the slices are added in chunk order), else n_g. */
int64_t nlb_lambda_ha_len(const nlb_struct_problem *prob);
int64_t nlb_lambda_gb_len(const nlb_struct_problem *prob);
/* 1 when the lattice path applies to prob (FP32 and DIIS available). */
int32_t nlb_lambda_lattice(const nlb_struct_problem *prob);
/* Build the tables at (t1, t2), reset ctrl and zero the multipliers (unless
 * flags has NLB_LAMBDA_KEEP); tol is the relative step size of the
 * multipliers that ends the iteration, max_diis the DIIS subspace (0: none). */
int nlb_lambda_init(const nlb_struct_problem *prob, const nlb_lambda_state *st, double tol,
                    double mixing, int32_t max_steps, int32_t max_diis, int32_t flags, nlb_stream_t stream);
/* One Jacobi step of the Lambda equations; does nothing once ctrl->status is
 * not NLB_RUNNING, so the accumulators keep U = t1^T lam1 and T of the last
 * step that ran.  With DIIS the step stores its error vector. */
int nlb_lambda_step(const nlb_struct_problem *prob, const nlb_lambda_state *st, nlb_stream_t stream);
/* DIIS extrapolation of the multipliers when the last step filled the
 * subspace (a no-op otherwise); call after every max_diis-th step. */
int nlb_lambda_diis(const nlb_struct_problem *prob, const nlb_lambda_state *st, int32_t max_diis,
                    nlb_stream_t stream);
/* *out = <lam2, (dW + dV) tau> for diagonal derivative ladders
 * dw[hh_ptr_off + hp], dv[pp_ptr_off + ab] (tau = t2 + t1 t1); FP64 state. */
int nlb_lambda_coupling(const nlb_struct_problem *prob, const nlb_lambda_state *st, const double *dw,
                        const double *dv, double *out, nlb_stream_t stream);

/* ---------------------------------------------------------------------
 * Batched scan (no counterpart in the reference): many structured problems
 * of uneven size solved, with their coupling derivatives, in ONE CUDA graph
 * launch (one instance and the forward phases alone give a whole solve as
 * one launch, no host round trips).  The graph holds four device-side loops (conditional WHILE nodes):
 * forward FP32 to mixed_eps, forward FP64 to eps, Lambda FP32 to
 * lambda_tol_fp32 (lattice instances) and Lambda FP64 to lambda_tol; each
 * loop body is one branch per instance (chunk steps, DIIS pulses included).
 * --------------------------------------------------------------------- */
typedef struct {
    const nlb_struct_problem *prob;   /* the instance (host struct, device tables) */
    nlb_struct_state f32, f64;        /* forward buffers (dtype F32 / F64) */
    nlb_lambda_state l32, l64;        /* Lambda buffers; l32.dtype 0: no FP32 Lambda phase.
                                         l64.t1/t2 (and l32.t1) must be f64.t1[0]/f64.t2[0];
                                         l32.t2 receives the converged t2 in FP32 */
    const double *t1_init;            /* [p*h] start amplitudes (MP2 t1) */
    double e0;                        /* energy of t1_init */
    const double *dw[2], *dv[2];      /* diagonal derivative ladders of two couplings (FP64) */
    double *out;                      /* [8]: E_corr, coupling term 0, coupling term 1, forward status,
                                         forward iterations, Lambda status, Lambda iterations,
                                         FP32 forward iterations; without a Lambda phase [1] is the
                                         parity of the last forward phase and [2] the FP32 energy */
} nlb_batch_item;

enum { NLB_PHASE_FWD32 = 1, NLB_PHASE_FWD64 = 2, NLB_PHASE_LAMBDA = 4 };

typedef struct {
    double mixing, mixed_eps, eps, lambda_tol_fp32, lambda_tol;
    int32_t max_steps, max_diis, lambda_max_steps;
    int32_t chunk;                    /* steps per loop iteration; a multiple of max_diis */
    int32_t phases;                   /* NLB_PHASE_* bits: forward FP32 (to mixed_eps), forward FP64 (to eps,
                                         from the FP32 result when both), Lambda (needs FP64 forward) */
    int32_t criterion;                /* NLB_CRIT_SOA / NLB_CRIT_NUMPY for the forward phases */
} nlb_batch_config;

/* Capture and instantiate the batch graph (buffers stay caller-owned). */
int nlb_batch_create(const nlb_batch_item *items, int32_t n, const nlb_batch_config *cfg, void **handle);
/* Launch the whole batch on `stream` (one cudaGraphLaunch). */
int nlb_batch_launch(void *handle, nlb_stream_t stream);
int nlb_batch_destroy(void *handle);

/* ---------------------------------------------------------------------
 * General (dense) engine: the full factorised equation set of
 * CCM/coupled_cluster.py:342-545 on dense FP64 tensors in the reference's
 * layouts, for inputs without the closed-site label structure.
 * --------------------------------------------------------------------- */

/* C[m,n] = alpha * sum_k A[m,k] B[k,n] + beta * C[m,n], where m, n, k and the
 * batch index b are multi-indices of up to four dimensions each with their
 * own strides in A, B and C (every pairwise einsum of ccDgrams.py). */
typedef struct {
    int32_t nm, nn, nk, nb;
    int64_t M, N, K, B;                      /* products of the extents */
    int64_t ext_m[4], ext_n[4], ext_k[4], ext_b[4];
    int64_t sa_m[4], sc_m[4];                /* strides of the m dims in A and C */
    int64_t sb_n[4], sc_n[4];                /* n dims in B and C */
    int64_t sa_k[4], sb_k[4];                /* k dims in A and B */
    int64_t sa_b[4], sb_b[4], sc_b[4];       /* batch dims in A, B and C */
} nlb_contract_desc;

int nlb_contract_f64(const nlb_contract_desc *d, const double *A, const double *B, double *C,
                     double alpha, double beta, nlb_stream_t stream);

/* The same contraction (no batch indices) as one library GEMM: A and B are
 * gathered into row-major [M][K] and [K][N] panels in `work`, multiplied by
 * cublasDgemm on `stream` and written back into the strided C (alpha, beta as
 * above).  `work` holds nlb_contract_gemm_work(d) bytes. */
int64_t nlb_contract_gemm_work(const nlb_contract_desc *d);
int nlb_contract_gemm_f64(const nlb_contract_desc *d, const double *A, const double *B, double *C,
                          double alpha, double beta, double *work, int64_t work_bytes, nlb_stream_t stream);

/* The same contraction on the tensor cores (mixed-precision phase of the
 * general engine): the operands are split into TF32 parts, A ~ A_hi + A_lo,
 * B ~ B_hi + B_lo, and C ~ alpha (A_hi B_hi + A_hi B_lo + A_lo B_hi) + beta C
 * with FP32 accumulation in tensor memory (tcgen05.mma kind::tf32, 128x128
 * tiles, TMA-staged operands, split-K when the tiles are fewer than the SMs;
 * the split partials are added in a fixed order).  Relative accuracy is that
 * of FP32 (about 1e-6 of the largest product).  `work` holds
 * nlb_contract_gemm_tc_work(d) bytes and starts on a 256-byte boundary.  A
 * tile whose bounded waits ran out turns every output entry into NaN.
 * Replaces, in the mixed phase, the library GEMM that evaluates the ring,
 * quadratic and dense-ladder diagrams (ccDgrams.py:253-303, 359-385,
 * 474-500). */
int64_t nlb_contract_gemm_tc_work(const nlb_contract_desc *d);
int nlb_contract_gemm_tf32x3(const nlb_contract_desc *d, const double *A, const double *B, double *C,
                             double alpha, double beta, void *work, int64_t work_bytes, nlb_stream_t stream);

/* H += alpha * P(Z) on (p,p,h,h) tensors, P = 1, pAB, pIJ or pIJ pAB
 * (perm 0..3; ccDgrams.py:193-213). */
int nlb_antisym_acc_f64(const double *Z, double *H, int64_t p, int64_t h, int32_t perm,
                        double alpha, nlb_stream_t stream);

/* In place: H_abij <- ((H_abij - H_baij) - (H_abji - H_baji)) / 4, exact
 * antisymmetry in floating point; identity on exactly antisymmetric H. */
int nlb_antisym_project_f64(double *H, int64_t p, int64_t h, nlb_stream_t stream);

/* Row list of v_ppph, idx[q] = (c,d,a,k) with value val[q] (repeated keys
 * add up), with the orders its intermediates are gathered in.  perm_* list
 * the rows sorted by the named key (a stable sort, so rows with equal keys
 * keep their list order); seg_*[s] .. seg_*[s+1] is the range of key s in that
 * order (n_* keys, seg_* has n_* + 1 entries).  perm_adk sorts by (a, d, k),
 * and seg_a, seg_ad and seg_adk all index it.  Built once per problem on the
 * host; every output entry is then the sum of its rows in a fixed order. */
typedef struct {
    int64_t nnz;
    const int64_t *idx;          /* [nnz][4] (c, d, a, k) */
    const double *val;           /* [nnz] */
    const int32_t *perm_adk, *perm_ak, *perm_cdk;
    int64_t n_a, n_ad, n_adk, n_ak, n_cdk;
    const int64_t *seg_a, *seg_ad, *seg_adk, *seg_ak, *seg_cdk;
} nlb_ppph_plan;

/* Row list of v_pppp, idx[q] = (a,b,c,d), sorted by (a, b) through perm_ab
 * with the n_ab key ranges seg_ab (as above). */
typedef struct {
    int64_t nnz;
    const int64_t *idx;
    const double *val;
    const int32_t *perm_ab;
    int64_t n_ab;
    const int64_t *seg_ab;
} nlb_pppp_plan;

/* v_ppph_dgrams (ccDgrams.py:13-45): r[0..6] zero-filled by the caller. */
int nlb_ppph_intermediates_f64(const nlb_ppph_plan *plan, const double *t1, const double *t2, int64_t p,
                               int64_t h, double *const *r, nlb_stream_t stream);

/* v_pppp_dgrams (ccDgrams.py:215-237): l1 += v t2[c,d], l2 += v t1[c] t1[d]. */
int nlb_pppp_ladders_f64(const nlb_pppp_plan *plan, const double *t1, const double *t2, int64_t p, int64_t h,
                         double *l1, double *l2, nlb_stream_t stream);

/* Jacobi steps with mixing for T1 and T2 (coupled_cluster.py:410-414,
 * 538-545, 614-620); e1/e2 (optional) receive new - old. */
int nlb_jacobi_f64(const double *t1, const double *H1, const double *t2, const double *H2,
                   const double *xpp1, const double *xhh1, const double *xpp2, const double *xhh2,
                   int64_t p, int64_t h, double mixing, double *t1_out, double *t2_out, double *e1,
                   double *e2, nlb_stream_t stream);

/* Doubles of the `work` buffer of nlb_dense_energy_f64 and nlb_vec_diis_f64
 * (per-block partial sums, added in a fixed order). */
#define NLB_DENSE_WORK_DOUBLES 57344

/* ccsd_energy (coupled_cluster.py:265-286) into *out (device); v_pphh may be
 * NULL when it is zero.  work holds NLB_DENSE_WORK_DOUBLES doubles. */
int nlb_dense_energy_f64(const double *f_ph, const double *t1, const double *v_pphh,
                         const double *t2, int64_t p, int64_t h, double *out, double *work,
                         nlb_stream_t stream);

/* Pulsed DIIS on concatenated amplitude vectors (soa/coupled_cluster.py:
 * 533-561): Gram of m error vectors err[m][n], FP64 bordered solve, and
 * out = sum_s c_s hist[s] (out untouched when the solve fails).  work holds
 * NLB_DENSE_WORK_DOUBLES doubles. */
int nlb_vec_diis_f64(const double *err, const double *hist, int64_t n, int32_t m, double *work,
                     double *out, nlb_stream_t stream);
/* The same on FP32 vectors (FP64 Gram, solve and sums; out rounded once). */
int nlb_vec_diis_f32(const float *err, const float *hist, int64_t n, int32_t m, double *work,
                     float *out, nlb_stream_t stream);

/* ------------------------------------------------------------------------
 * Momentum-block path: closed-shell plane-wave inputs with a contact
 * interaction (the input family of planewave.py, fed to the reference's
 * ccsd_solver at CCM/coupled_cluster.py:547-687).  Every hole momentum holds
 * all four spin-isospin states, so t1 vanishes by momentum conservation and
 * t2[a,b,i,j] lives in blocks of total momentum K = k_a + k_b = k_i + k_j:
 * block b is a row-major [nr x nc] matrix, row = pa*16 + s_a*4 + s_b (pa the
 * position of k_a among the block's particle momenta), col = pi*16 + s_i*4 +
 * s_j.  The interaction is <pq||rs> = V[s_p s_q s_r s_s] delta(K).  The
 * residual is the T2 equation of coupled_cluster.py:476-536 at t1 = 0
 * (ccDgrams.py:215-303, 502-527), the step its Jacobi update with mixing.
 * ---------------------------------------------------------------------- */
typedef struct {
    int32_t L;                 /* momenta n = (nx*L + ny)*L + nz, n < L^3 */
    int32_t n_blocks;          /* total momenta carried by hole pairs */
    int32_t n_pmom, n_hmom;    /* particle / hole momenta (4 states each) */
    int64_t n_t2;              /* blocked amplitudes = blk_off[n_blocks] */
    int64_t n_m, n_w, n_rows;  /* m_off[n_blocks], w_off[n_blocks], row_off[n_blocks] */
    int32_t n_tiles;           /* residual tiles (64 rows x 16 columns) */
    int32_t pad0;
    const int64_t *blk_off;    /* [n_blocks + 1] first amplitude of each block */
    const int64_t *m_off;      /* [n_blocks + 1] M blocks [16][nc] */
    const int64_t *w_off;      /* [n_blocks + 1] W blocks [nc][nc] */
    const int64_t *row_off;    /* [n_blocks + 1] first row of each block (Y rows) */
    const int32_t *blk_nr, *blk_nc, *blk_K;
    const int32_t *blk_pm0, *blk_hm0; /* start of the block's lists in pm_list / hm_list */
    const int32_t *pm_list;    /* particle-momentum index of each row group */
    const int32_t *hm_list;    /* hole-momentum index of each column group */
    const int32_t *ppos, *hpos; /* [n_blocks * L^3] row / column group of a momentum, or -1 */
    const int32_t *kblk;       /* [L^3] block of a total momentum, or -1 */
    const int32_t *pmom, *hmom; /* momentum of each particle / hole momentum index */
    const int32_t *pinv, *hinv; /* [L^3] particle / hole momentum index, or -1 */
    const int32_t *tiles;      /* [n_tiles * 3] (block, row0, col0) */
    const double *V;           /* [256] V[s_p s_q s_r s_s] (antisymmetric pairs) */
    const double *fpp;         /* [n_pmom * 16] Fock block of each particle momentum */
    const double *fhh;         /* [n_hmom * 16] Fock block of each hole momentum */
} nlb_pw_problem;

/* Intermediates of the momentum-block step, all of the amplitude type of the
 * entry point they are passed to (FP64: nlb_pw_energy / nlb_pw_step; FP32:
 * the _f32 entry points), except `energy`, which is FP64 in both. */
typedef struct {
    void *M;        /* [m_off[n]]   M_K[s_c s_d][col] = sum over k_c of t2 */
    void *W;        /* [w_off[n]]   dressed hole-hole ladder */
    void *Y;        /* [rows * 4]   row dots for X_pp */
    void *Xpp;      /* [n_pmom * 16] */
    void *Xhh;      /* [n_hmom * 16] */
    void *R, *U, *G; /* [4 n_pmom * 4 n_hmom * 16] particle-hole intermediates */
    void *H;        /* [n_t2] residual */
    double *energy; /* [1] */
} nlb_pw_state;

/* MP2 start t2 = V / (e_i + e_j - e_a - e_b + delta) (coupled_cluster.py:416-439). */
int nlb_pw_init(const nlb_pw_problem *P, double *t2, double delta, nlb_stream_t stream);
/* M of t2 and E = 1/4 sum v_pphh t2 into S->energy (coupled_cluster.py:265-286).
 * S->Y holds the energy's partial sums afterwards (nlb_pw_step rebuilds Y
 * from t2 before it reads it). */
int nlb_pw_energy(const nlb_pw_problem *P, const double *t2, nlb_pw_state *S, nlb_stream_t stream);
/* One Jacobi step with mixing (S->M must hold M of t2): t2_out, and
 * err = t2_out - t2 when err is not NULL. */
int nlb_pw_step(const nlb_pw_problem *P, const double *t2, double *t2_out, double *err, double mixing,
                nlb_pw_state *S, nlb_stream_t stream);
/* The same in FP32 (amplitudes and intermediates FP32, the energy's sums
 * FP64): the first phase of a mixed-precision plane-wave solve, which then
 * continues in FP64 from the converted amplitudes. */
int nlb_pw_energy_f32(const nlb_pw_problem *P, const float *t2, nlb_pw_state *S, nlb_stream_t stream);
int nlb_pw_step_f32(const nlb_pw_problem *P, const float *t2, float *t2_out, float *err, double mixing,
                    nlb_pw_state *S, nlb_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* NULATTICE_B200_H */
