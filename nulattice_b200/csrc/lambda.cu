// Adjoint (CC Lambda) kernels of the structured engine, sm_100a.
//
// At converged amplitudes (t1, t2) the coupling derivative of the CCSD energy
// is dE/dc = dE_ref/dc + <lam1, R1(t; dH)> + <Lam, R2(t; dH)>, where the
// multipliers solve the Lambda equations
//   Z1 = dE/dt1 + (dR/dt1)^T lam = 0,   Z2 = (dR/dt2)^T lam = 0,
// R being the residual of t1Iter / t2Iter (CCM/coupled_cluster.py:342-545)
// on the compact channel layout and dH the derivative Hamiltonian (the
// residual is linear in the Hamiltonian).  The reference has no adjoint; the
// transposed terms below mirror the forward kernels of ccsd_struct.cu one by
// one (stencils and ladders are symmetric, the X_hh mixing is transposed, the
// rank-h parts swap the roles of t1 and f_ph).  The equations are iterated
// with the forward Jacobi denominators and mixing, optionally with the same
// pulsed DIIS as the forward solve (the Lambda equations are linear, so the
// extrapolation pays off quickly).
//
// Two paths:
// * general (any hole counts, FP64): one block per row task, every
//   contraction of the row in shared memory (k_l_rows);
// * lattice (seven holes per label, diagonal ladders, short f_pp rows; FP32
//   or FP64): a column pass over the multipliers (k_l_cols: Ha, the Z1
//   contributions of the particles b' and the hole-hole contractions T) and
//   a row pass laid out like the forward k_t2_lat (k_l_lat: Z2, the Jacobi
//   update and the Z1 contributions of the particles a').

#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>

#include "nulattice_b200.h"

void nlb_internal_set_error(const char* msg);

namespace {

constexpr int kThreads = 256;

#include "common.cuh"

int lfail(int code, const char* msg) {
    nlb_internal_set_error(msg);
    return code;
}

int lcheck(const char* where) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        char buf[512];
        snprintf(buf, sizeof(buf), "%s: %s", where, cudaGetErrorString(e));
        nlb_internal_set_error(buf);
        return NLB_ERR_LAUNCH;
    }
    return NLB_OK;
}

// scratch layout (doubles): Y1[p*h] Z1 contributions gathered from T2 rows
// (general path), U[h*h] = t1^T lam1, T[h*h] X_hh contractions, fc[n_t1c]
// f_ph per label, and the lattice path's per-writer slots: Y1r[n_f2] (the Z1
// contribution of row a' of each channel, [a'][k'], from the block holding
// the row's first b' column), Y1q[n_f2] (the part of the row's b' columns
// that the next block holds, zero when one block holds the whole row),
// Y1c[kMaxColChunks][n_f2]
// (of column b' and one row chunk of the column pass, [b'][k']) and
// Tp[col items][2][49] (the X_hh contractions of one column-pass block, g1
// side then g2 side).  Every slot has exactly one writer; k_l_t1 and
// k_l_treduce add them in a fixed order, so the lattice path's Lambda solve
// repeats bit for bit.
constexpr int kMaxColChunks = 8;       // row chunks of the column pass
constexpr int kLHP_ = 49;              // hole pairs per channel block on the lattice path
constexpr int kColNB = 256 / kLHP_;    // column-pass b' per block (kColThreads / 49)

__host__ __device__ inline int64_t col_items_max(const nlb_struct_problem& P) {
    const int64_t np = P.max_row / kLHP_;
    return (int64_t)P.n_channels * ((np + kColNB - 1) / kColNB) * kMaxColChunks;
}

// General path (FP64, any hole counts): the row kernel writes, per row task,
// its Z1 contributions of particle a' into Y1r (as on the lattice path), its
// contributions to the particles b' of label g2 into Yg (the row's own
// [b'][k'] slice at the channel's T2 offset: n_t2 doubles cover every
// channel), and its X_hh contractions into Tg[row][side][k'][m'] (max_nh^2
// per side); k_l_rows_reduce adds them in a fixed order into Y1 and T.
struct LView {
    double *Y1, *U, *T, *fc, *Y1r, *Y1q, *Y1c, *Tp, *Yg, *Tg;
};

__host__ __device__ inline LView lview(double* acc, const nlb_struct_problem& P) {
    LView v;
    v.Y1 = acc;
    v.U = v.Y1 + (int64_t)P.p * P.h;
    v.T = v.U + (int64_t)P.h * P.h;
    v.fc = v.T + (int64_t)P.h * P.h;
    v.Y1r = v.fc + P.n_t1c;
    v.Y1q = v.Y1r + P.n_f2;
    v.Y1c = v.Y1q + P.n_f2;
    v.Tp = v.Y1c + (int64_t)kMaxColChunks * P.n_f2;
    v.Yg = v.Tp + col_items_max(P) * 2 * kLHP_;   // general path only
    v.Tg = v.Yg + P.n_t2;
    return v;
}

// f_ph[P_g[a'], H_g[k']] for entry q of the label-ordered t1 tables.
__device__ __forceinline__ double fc_entry(const nlb_struct_problem& P, int64_t q) {
    const int g = find_label(P.t1c_base, P.n_labels, q);
    const int nh = P.h_base[g + 1] - P.h_base[g];
    const int loc = (int)(q - P.t1c_base[g]);
    const int ap = loc / nh, kq = loc - ap * nh;
    return P.f_ph[(int64_t)P.p_ord[P.p_base[g] + ap] * P.h + P.h_ord[P.h_base[g] + kq]];
}

// =================================================== general path (FP64) ==

// Tables at the converged amplitudes: prep, Ga, and the per-label f_ph copy.
__global__ void k_l_setup(nlb_struct_problem P, nlb_lambda_state S) {
    const int64_t nprep = (int64_t)P.h * P.h + 2 * (int64_t)P.p + P.n_t1c + P.n_xc + P.h;
    const LView V = lview(S.acc, P);
    const double* t2 = static_cast<const double*>(S.t2);
    double* ga = static_cast<double*>(S.ga);
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < nprep + P.n_g + P.n_t1c; u += stride) {
        if (u < nprep) prep_body(P, S.t1, S.prep, u);
        else if (u < nprep + P.n_g) ga[u - nprep] = ga_element(P, t2, u - nprep);
        else V.fc[u - nprep - P.n_g] = fc_entry(P, u - nprep - P.n_g);
    }
}

// Ha[k'][e] = sum_a' t1[a,k] Lam[a'][e] (k in H_g1), laid out like Ga.
__global__ void k_l_ha(nlb_struct_problem P, nlb_lambda_state S) {
    const nlb_ctrl* c = S.ctrl;
    if (c->status != NLB_RUNNING) return;
    const double* Lm = static_cast<const double*>(S.lam2[c->parity]);
    double* ha = static_cast<double*>(S.ha);
    const PrepView PV = prep_view(S.prep, P);
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < P.n_g; u += stride) {
        const int ci = find_seg(P.g_end, P.n_channels, u);
        const nlb_channel& ch = P.chan[ci];
        const int rowlen = ch.np2 * ch.nh1 * ch.nh2;
        const int loc = (int)(u - ch.ga_off);
        const int kq = loc / rowlen, e = loc - kq * rowlen;
        const double* t1a = PV.t1c + P.t1c_base[ch.g1] + kq;
        const double* col = Lm + ch.offset + e;
        double acc = 0.0;
        for (int ap = 0; ap < ch.np1; ++ap) acc += t1a[ap * ch.nh1] * col[(int64_t)ap * rowlen];
        ha[u] = acc;
    }
}

// One block per row task (channel, a'): Z2 and the Jacobi update of the row,
// and the row's contributions to Z1 (through Y1) and to T.
__global__ void __launch_bounds__(kThreads) k_l_rows(nlb_struct_problem P, nlb_lambda_state S) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const nlb_ctrl* c = S.ctrl;
    if (c->status != NLB_RUNNING) return;
    const int par = c->parity;
    const double* __restrict__ Lm = static_cast<const double*>(S.lam2[par]);
    double* __restrict__ Lo = static_cast<double*>(S.lam2[par ^ 1]);
    const double* __restrict__ l1 = S.lam1[par];
    const double* __restrict__ B = static_cast<const double*>(S.t2);
    const double* __restrict__ ga = static_cast<const double*>(S.ga);
    const double* __restrict__ ha = static_cast<const double*>(S.ha);
    double* E2 = (S.diis_t2 != nullptr && c->max_diis > 0 && c->diis_count < c->max_diis)
                     ? static_cast<double*>(S.diis_t2) + (int64_t)c->diis_count * P.n_t2 : nullptr;
    const PrepView PV = prep_view(S.prep, P);
    const LView V = lview(S.acc, P);
    const double m = c->mixing;
    const int mh = P.max_nh, h = P.h;
    double* lrow = reinterpret_cast<double*>(smem_raw);  // [max_row] Lam row
    double* brow = lrow + P.max_row;                      // [max_row] t2 row
    double* shb = brow + P.max_row;                       // [mh^3] Hb
    double* sgb = shb + mh * mh * mh;                     // [mh^3] Gb of t2
    double* sx1 = sgb + mh * mh * mh;                     // [mh^2]
    double* sx2 = sx1 + mh * mh;                          // [mh^2]
    double* st1a = sx2 + mh * mh;                         // [mh]
    double* sf1a = st1a + mh;                             // [mh]
    double* sl1a = sf1a + mh;                             // [mh]
    double* shh = sl1a + mh;                              // [mh^2]
    double dnrm = 0.0, lnrm = 0.0;
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int64_t task = blockIdx.x; task < P.n_rows; task += gridDim.x) {
        const int ci = find_seg(P.row_end, P.n_channels, task);
        const nlb_channel& ch = P.chan[ci];
        const int ap = (int)(task - (ci ? P.row_end[ci - 1] : 0));
        const int nh1 = ch.nh1, nh2 = ch.nh2, np2 = ch.np2;
        const int nhp = nh1 * nh2;
        const int rowlen = np2 * nhp;
        const int64_t rbase = ch.offset + (int64_t)ap * rowlen;
        const int a = P.p_ord[ch.pb1 + ap];
        const int32_t* hptr = P.hh_ptr + ch.hh_ptr_off;
        const double* hval = P.hh_val + ch.hh_col_off;
        const int32_t* pptr = P.pp_ptr + ch.pp_ptr_off;
        const double* pval = P.pp_val + ch.pp_col_off;
        const double* t1b = PV.t1c + P.t1c_base[ch.g2];
        const double* f2c = V.fc + P.t1c_base[ch.g2];
        for (int e = tid; e < rowlen; e += nt) {
            lrow[e] = Lm[rbase + e];
            brow[e] = B[rbase + e];
        }
        for (int e = tid; e < nh1 * nh1; e += nt) sx1[e] = PV.xc[P.xc_base[ch.g1] + e];
        for (int e = tid; e < nh2 * nh2; e += nt) sx2[e] = PV.xc[P.xc_base[ch.g2] + e];
        for (int e = tid; e < nh1; e += nt) {
            st1a[e] = PV.t1c[P.t1c_base[ch.g1] + ap * nh1 + e];
            sf1a[e] = V.fc[P.t1c_base[ch.g1] + ap * nh1 + e];
            sl1a[e] = l1[(int64_t)a * h + P.h_ord[ch.hb1 + e]];
        }
        for (int e = tid; e < nhp; e += nt) shh[e] = (hptr[e + 1] > hptr[e]) ? hval[hptr[e]] : 0.0;
        __syncthreads();
        for (int e = tid; e < nh2 * nhp; e += nt) {
            const int kq = e / nhp, hp = e - kq * nhp;
            double acc = 0.0;
            for (int cq = 0; cq < np2; ++cq) acc += t1b[cq * nh2 + kq] * lrow[cq * nhp + hp];
            shb[e] = acc;
            const int row = ch.hb2 + kq;
            double g = 0.0;
            for (int q = P.fph_ptr[row]; q < P.fph_ptr[row + 1]; ++q) g += P.fph_val[q] * brow[P.fph_col[q] * nhp + hp];
            sgb[e] = g;
        }
        __syncthreads();
        const double da = PV.dpc[ch.pb1 + ap];
        const int ra0 = P.fpp_ptr[ch.pb1 + ap], ra1 = P.fpp_ptr[ch.pb1 + ap + 1];
        for (int e = tid; e < rowlen; e += nt) {
            const int bp = e / nhp, hp = e - bp * nhp;
            const int ip = hp / nh2, jp = hp - ip * nh2;
            const double x = lrow[e];
            double Z = 0.0;
            const int rb = ch.pb2 + bp;
            for (int q = P.fpp_ptr[rb]; q < P.fpp_ptr[rb + 1]; ++q) Z += P.fpp_val[q] * lrow[P.fpp_col[q] * nhp + hp];
            for (int q = ra0; q < ra1; ++q) {
                const int col = P.fpp_col[q];
                Z += P.fpp_val[q] * ((col == ap) ? x : Lm[ch.offset + (int64_t)col * rowlen + e]);
            }
            for (int k = 0; k < nh2; ++k) Z -= f2c[bp * nh2 + k] * shb[k * nhp + hp];
            for (int k = 0; k < nh1; ++k) Z -= sf1a[k] * ha[ch.ga_off + (int64_t)k * rowlen + e];
            for (int k = 0; k < nh1; ++k) Z += sx1[ip * nh1 + k] * lrow[bp * nhp + k * nh2 + jp];
            for (int k = 0; k < nh2; ++k) Z += sx2[jp * nh2 + k] * lrow[bp * nhp + ip * nh2 + k];
            const int ab = ap * np2 + bp;
            const double cpp = (pptr[ab + 1] > pptr[ab]) ? pval[pptr[ab]] : 0.0;
            Z += (shh[hp] + cpp) * x;
            Z += sl1a[ip] * f2c[bp * nh2 + jp];
            Z += l1[(int64_t)P.p_ord[ch.pb2 + bp] * h + P.h_ord[ch.hb2 + jp]] * sf1a[ip];
            const double D = -((da + PV.dpc[ch.pb2 + bp]) + (PV.dhc[ch.hb1 + ip] + PV.dhc[ch.hb2 + jp]));
            const double out = x + (1.0 - m) * Z / D;
            Lo[rbase + e] = out;
            if (E2) E2[rbase + e] = out - x;
            dnrm += (out - x) * (out - x);
            lnrm += out * out;
        }
        // row contributions to Z1 for particles b' of label g2
        for (int w = tid; w < np2 * nh2; w += nt) {
            const int bp = w / nh2, kq = w - bp * nh2;
            double s = 0.0;
            for (int hp = 0; hp < nhp; ++hp) s += lrow[bp * nhp + hp] * sgb[kq * nhp + hp];
            const int ab = ap * np2 + bp;
            const double cpp = (pptr[ab + 1] > pptr[ab]) ? pval[pptr[ab]] : 0.0;
            double lt = 0.0;
            for (int ip = 0; ip < nh1; ++ip) {
                const int hp = ip * nh2 + kq;
                lt += lrow[bp * nhp + hp] * (shh[hp] + cpp) * st1a[ip];
            }
            // (a channel without holes on the a side has no T2 block, adds
            // nothing and owns no slots)
            if (nh1 > 0) V.Yg[ch.offset + ((int64_t)ap * np2 + bp) * nh2 + kq] = lt - s;
        }
        // X_hh contractions T along i (g1) and along j (g2)
        for (int w = tid; w < nh1 * nh1 + nh2 * nh2; w += nt) {
            double s = 0.0;
            if (w < nh1 * nh1) {
                const int kq = w / nh1, iq = w - kq * nh1;
                for (int bp = 0; bp < np2; ++bp)
                    for (int jq = 0; jq < nh2; ++jq)
                        s += lrow[bp * nhp + iq * nh2 + jq] * brow[bp * nhp + kq * nh2 + jq];
                V.Tg[((int64_t)task * 2 + 0) * mh * mh + kq * mh + iq] = s;
            } else {
                const int w2 = w - nh1 * nh1;
                const int kq = w2 / nh2, jq = w2 - kq * nh2;
                for (int bp = 0; bp < np2; ++bp)
                    for (int iq = 0; iq < nh1; ++iq)
                        s += lrow[bp * nhp + iq * nh2 + jq] * brow[bp * nhp + iq * nh2 + kq];
                V.Tg[((int64_t)task * 2 + 1) * mh * mh + kq * mh + jq] = s;
            }
        }
        // particle a' of label g1: -sum_e Lam Ga[k'] and the ladder t1 term
        for (int q = 0; q < 2 * nh1; ++q) {
            double part = 0.0;
            if (q < nh1) {
                for (int e = tid; e < rowlen; e += nt) part += lrow[e] * ga[ch.ga_off + (int64_t)q * rowlen + e];
                part = -part;
            } else {
                const int iq = q - nh1;
                for (int w = tid; w < np2 * nh2; w += nt) {
                    const int bp = w / nh2, jq = w - bp * nh2;
                    const int hp = iq * nh2 + jq, ab = ap * np2 + bp;
                    const double cpp = (pptr[ab + 1] > pptr[ab]) ? pval[pptr[ab]] : 0.0;
                    part += lrow[bp * nhp + hp] * (shh[hp] + cpp) * t1b[bp * nh2 + jq];
                }
            }
            const double tot = block_sum(part);
            if (tid == 0) {
                double* y = V.Y1r + ch.f2_off + (int64_t)ap * nh1 + (q % nh1);
                *y = q < nh1 ? tot : *y + tot;   // the two parts of (a', k') in a fixed order
            }
        }
        __syncthreads();
    }
    const double s1 = block_sum(dnrm);
    const double s2 = block_sum(lnrm);
    if (tid == 0) {
        PV.slots(kRedDt2)[blockIdx.x] = 4.0 * s1;
        PV.slots(kRedNrm2)[blockIdx.x] = 4.0 * s2;
    }
}

// ========================================================== both paths ==

// U = t1^T lam1 (one warp per hole pair of one label; pairs of different
// labels vanish) and zeroed accumulators Y1, T.
__global__ void k_l_u(nlb_struct_problem P, nlb_lambda_state S) {
    const nlb_ctrl* c = S.ctrl;
    if (c->status != NLB_RUNNING) return;
    const double* l1 = S.lam1[c->parity];
    const LView V = lview(S.acc, P);
    const int h = P.h;
    const int64_t hh = (int64_t)h * h, ph = (int64_t)P.p * h;
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t u = warp; u < hh; u += nwarps) {
        const int k = (int)(u / h), mm = (int)(u % h);
        const int g = P.h_label[k];
        double s = 0.0;
        if (P.h_label[mm] == g)
            for (int i = P.p_base[g] + lane; i < P.p_base[g + 1]; i += 32) {
                const int64_t a = P.p_ord[i];
                s += S.t1[a * h + k] * l1[a * h + mm];
            }
        s = warp_sum(s);
        if (lane == 0) V.U[u] = s;
    }
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < hh + ph; u += stride) {
        if (u < hh) V.T[u] = 0.0;
        else V.Y1[u - hh] = 0.0;
    }
}

// General path: Y1 and T from the row kernel's slots.  Thread per entry of
// Y1 (p*h) or T (h*h); the channels in order, the rows of a channel in order.
__global__ void k_l_rows_reduce(nlb_struct_problem P, nlb_lambda_state S) {
    const nlb_ctrl* c = S.ctrl;
    if (c->status != NLB_RUNNING) return;
    const LView V = lview(S.acc, P);
    const int h = P.h, mh = P.max_nh;
    const int64_t ph = (int64_t)P.p * h, hh = (int64_t)h * h;
    for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < ph + hh;
         idx += (int64_t)gridDim.x * blockDim.x) {
        if (idx < ph) {
            const int x = (int)(idx / h), mm = (int)(idx % h);
            const int g = P.p_label[x];
            double y = 0.0;
            if (P.h_label[mm] == g) {
                const int xl = P.p_loc[x], ml = P.h_loc[mm];
                for (int ci = 0; ci < P.n_channels; ++ci) {
                    const nlb_channel& ch = P.chan[ci];
                    if (ch.g1 == g) y += V.Y1r[ch.f2_off + (int64_t)xl * ch.nh1 + ml];
                    if (ch.g2 == g && ch.nh1 > 0)
                        for (int ap = 0; ap < ch.np1; ++ap)
                            y += V.Yg[ch.offset + ((int64_t)ap * ch.np2 + xl) * ch.nh2 + ml];
                }
            }
            V.Y1[idx] = y;
        } else {
            const int64_t u = idx - ph;
            const int k = (int)(u / h), mm = (int)(u % h);
            const int g = P.h_label[k];
            double t = 0.0;
            if (P.h_label[mm] == g) {
                const int kl = P.h_loc[k], ml = P.h_loc[mm];
                for (int ci = 0; ci < P.n_channels; ++ci) {
                    const nlb_channel& ch = P.chan[ci];
                    const int64_t t0 = ci ? P.row_end[ci - 1] : 0;
                    for (int side = 0; side < 2; ++side) {
                        if ((side ? ch.g2 : ch.g1) != g) continue;
                        for (int ap = 0; ap < ch.np1; ++ap)
                            t += V.Tg[((t0 + ap) * 2 + side) * mh * mh + kl * mh + ml];
                    }
                }
            }
            V.T[u] = t;
        }
    }
}

// Z1 and the Jacobi update of lam1.  nchunk > 0 (lattice path): the Z1
// contributions come from the row and column slots (Y1r, Y1c), added in
// channel order; 0 (general path): from the Y1 accumulator.
__global__ void k_l_t1(nlb_struct_problem P, nlb_lambda_state S, int nchunk) {
    nlb_ctrl* c = S.ctrl;
    if (c->status != NLB_RUNNING) return;
    const int par = c->parity;
    const double* l1 = S.lam1[par];
    double* lo = S.lam1[par ^ 1];
    const PrepView PV = prep_view(S.prep, P);
    const LView V = lview(S.acc, P);
    const int h = P.h, p = P.p;
    const double m = c->mixing;
    double* E1 = (S.diis_t1 != nullptr && c->max_diis > 0 && c->diis_count < c->max_diis)
                     ? S.diis_t1 + (int64_t)c->diis_count * p * h : nullptr;
    double dn = 0.0, ln = 0.0;
    for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < (int64_t)p * h;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(idx / h), mm = (int)(idx % h);
        const int g = P.p_label[x];
        if (P.h_label[mm] != g) {
            lo[idx] = 0.0;
            if (E1) E1[idx] = 0.0;
            continue;
        }
        double y1 = 0.0;
        if (nchunk > 0) {
            const int xl = P.p_loc[x], ml = P.h_loc[mm];
            for (int ci = 0; ci < P.n_channels; ++ci) {
                const nlb_channel& ch = P.chan[ci];
                const int64_t o = ch.f2_off + (int64_t)xl * ch.nh1 + ml;
                if (ch.g1 == g) y1 += V.Y1r[o] + V.Y1q[o];
                if (ch.g2 == g)
                    for (int cq = 0; cq < nchunk; ++cq) y1 += V.Y1c[(int64_t)cq * P.n_f2 + o];
            }
        } else {
            y1 = V.Y1[idx];
        }
        double Z = P.f_ph[idx] + y1;
        const int pb = P.p_base[g];
        const int r = pb + P.p_loc[x];
        for (int q = P.fpp_ptr[r]; q < P.fpp_ptr[r + 1]; ++q)
            Z += P.fpp_val[q] * l1[(int64_t)P.p_ord[pb + P.fpp_col[q]] * h + mm];
        for (int i = 0; i < h; ++i) {
            const double li = l1[(int64_t)x * h + i];
            if (li != 0.0) Z -= li * (P.f_hh[(int64_t)mm * h + i] + PV.Q[(int64_t)mm * h + i]);
        }
        for (int k = 0; k < h; ++k) {
            const double fk = P.f_ph[(int64_t)x * h + k];
            if (fk != 0.0) Z -= fk * (V.U[(int64_t)k * h + mm] + V.T[(int64_t)k * h + mm]);
        }
        const double D1 = -(PV.dXp1[x] + PV.Xh1[(int64_t)mm * h + mm]);
        const double out = l1[idx] + (1.0 - m) * Z / D1;
        lo[idx] = out;
        if (E1) E1[idx] = out - l1[idx];
        dn += (out - l1[idx]) * (out - l1[idx]);
        ln += out * out;
    }
    const double s1 = block_sum(dn);
    const double s2 = block_sum(ln);
    if (threadIdx.x == 0) {
        PV.slots(kRedDt1)[blockIdx.x] = s1;
        PV.slots(kRedNrm1)[blockIdx.x] = s2;
    }
}

// Convergence on the relative step of the multipliers; DIIS bookkeeping as
// in the forward k_finish (a pulse when max_diis error vectors are stored).
// One warp: the norms from the per-block partials of the T1 (n1 blocks) and
// row (n2 blocks) launches, added in slot order.
// Launched with four warps, one per partial-sum array, each added in the
// fixed order of warp_sum_slots.
__global__ void k_l_finish(nlb_ctrl* c, const double* red, int n1, int n2) {
    __shared__ double sums[4];
    if (blockIdx.x != 0 || c->status != NLB_RUNNING) return;
    const int w = threadIdx.x >> 5;
    const int kind[4] = {kRedDt1, kRedNrm1, kRedDt2, kRedNrm2};
    if (w < 4) sums[w] = warp_sum_slots(red + (int64_t)kind[w] * kRedSlots, w < 2 ? n1 : n2);
    __syncthreads();
    if (threadIdx.x != 0) return;
    const double d1 = sums[0], l1 = sums[1], d2 = sums[2], l2 = sums[3];
    c->dt1_sq = d1;
    c->dt2_sq = d2;
    c->e_acc = l1 + l2;
    c->iter += 1;
    c->parity ^= 1;
    c->diis_pulse = 0;
    const double step = sqrt(c->dt1_sq + c->dt2_sq), size = sqrt(c->e_acc);
    c->e_last = step;
    if (step < c->eps * fmax(1.0, size)) {
        c->status = NLB_CONVERGED;
    } else if (!(step == step) || step > 1e12) {
        c->status = NLB_DIVERGED;
    } else {
        if (c->max_diis > 0) {
            c->diis_count += 1;
            if (c->diis_count == c->max_diis) {
                c->diis_pulse = 1;
                for (int k = 0; k < 121; ++k) c->gram[k] = 0.0;
            }
        }
        if (c->iter >= c->max_steps) c->status = NLB_MAX_ITER;
    }
}

__global__ void k_l_init(nlb_ctrl* c, double tol, double mixing, int max_steps, int max_diis) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    c->e_acc = 0.0; c->dt1_sq = 0.0; c->dt2_sq = 0.0; c->e_prev = 0.0; c->e_last = 0.0;
    c->eps = tol; c->mixing = mixing;
    c->parity = 0; c->iter = 0; c->status = max_steps > 0 ? NLB_RUNNING : NLB_MAX_ITER; c->max_steps = max_steps;
    c->criterion = NLB_CRIT_SOA; c->max_diis = max_diis; c->diis_count = 0; c->diis_pulse = 0;
    c->diis_applied = 0; c->ccs = 0;
    for (int k = 0; k < 121; ++k) c->gram[k] = 0.0;
}

// <Lam, (dW + dV) tau> over the compact layout for a derivative Hamiltonian
// whose ladders are diagonal: dw[hh_ptr_off + hp], dv[pp_ptr_off + ab].
__global__ void k_l_coupling(nlb_struct_problem P, nlb_lambda_state S, const double* dw, const double* dv,
                             double* out) {
    const double* Lm = static_cast<const double*>(S.lam2[S.ctrl->parity]);
    const double* t2 = static_cast<const double*>(S.t2);
    const PrepView PV = prep_view(S.prep, P);
    double acc = 0.0;
    // the block's contiguous range [u0, u1) of the compact amplitudes; a
    // thread walks it at stride blockDim.x, tracking its channel, row a' and
    // element e of the row (no per-element search or 64-bit division)
    const int64_t u0 = (int64_t)blockIdx.x * P.n_t2 / gridDim.x;
    const int64_t u1 = (int64_t)(blockIdx.x + 1) * P.n_t2 / gridDim.x;
    int64_t u = u0 + threadIdx.x;
    if (u < u1) {
        int ci = find_seg(P.t2_end, P.n_channels, u);
        const nlb_channel* ch = &P.chan[ci];
        int nhp = ch->nh1 * ch->nh2, rowlen = ch->np2 * nhp;
        int ap = (int)((u - ch->offset) / rowlen);
        int e = (int)(u - ch->offset - (int64_t)ap * rowlen);
        for (; u < u1; u += blockDim.x, e += blockDim.x) {
            while (e >= rowlen) {   // next row, or the first row of a later channel
                e -= rowlen;
                if (++ap >= ch->np1) {
                    do {
                        ch = &P.chan[++ci];
                    } while ((int64_t)ch->np1 * ch->np2 * ch->nh1 * ch->nh2 == 0);   // channels hold
                    // their amplitudes back to back, so u is the first one of this channel
                    nhp = ch->nh1 * ch->nh2;
                    rowlen = ch->np2 * nhp;
                    ap = 0;
                }
            }
            const int bp = e / nhp, hp = e - bp * nhp;
            const int ip = hp / ch->nh2, jp = hp - ip * ch->nh2;
            const double tau = t2[u] + PV.t1c[P.t1c_base[ch->g1] + ap * ch->nh1 + ip] *
                                           PV.t1c[P.t1c_base[ch->g2] + bp * ch->nh2 + jp];
            acc += Lm[u] * (dw[ch->hh_ptr_off + hp] + dv[ch->pp_ptr_off + ap * ch->np2 + bp]) * tau;
        }
    }
    const double s = block_sum(acc);
    if (threadIdx.x == 0) PV.slots(0)[blockIdx.x] = s;
}

// *out = the n per-block partials at `part`, added in slot order (one warp).
__global__ void k_l_sum_slots(const double* part, int n, double* out) {
    const double s = warp_sum_slots(part, n);
    if (threadIdx.x == 0) *out = s;
}

// ======================================================== lattice path ==
constexpr int kLH = 7;                 // holes per label on the lattice path
constexpr int kLHP = kLH * kLH;
constexpr int kLNa = 6;                // off-diagonal f_pp entries of a' in registers
constexpr int kLNb = 8;                // staged f_pp slots of b' (at most 7 used)
constexpr int kLRec = 24;              // record of b': f_ph[7], flag | lam1[7], pp ladder | t1[7], denominator

// Tables at the converged amplitudes: prep, f_ph per label, Ga and the Gb of
// every row, both in the multipliers' type.
template <typename T>
__global__ void k_l_setup_lat(nlb_struct_problem P, nlb_lambda_state S) {
    const int64_t nprep = (int64_t)P.h * P.h + 2 * (int64_t)P.p + P.n_t1c + P.n_xc + P.h;
    const int64_t n_gb = P.n_rows * kLH * kLHP;
    const LView V = lview(S.acc, P);
    const T* t2 = static_cast<const T*>(S.t2);
    T* ga = static_cast<T*>(S.ga);
    T* gb = static_cast<T*>(S.gb);
    const int64_t total = nprep + P.n_g + P.n_t1c + n_gb;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < total; u += stride) {
        if (u < nprep) {
            prep_body(P, S.t1, S.prep, u);
        } else if (u < nprep + P.n_g) {
            ga[u - nprep] = ga_element(P, t2, u - nprep);
        } else if (u < nprep + P.n_g + P.n_t1c) {
            V.fc[u - nprep - P.n_g] = fc_entry(P, u - nprep - P.n_g);
        } else {
            // Gb[row][k'][hp] = sum_c f_ck B[a'][c'][hp], holes k of label g2
            const int64_t v = u - nprep - P.n_g - P.n_t1c;
            const int64_t task = v / (kLH * kLHP);
            const int rem = (int)(v - task * (kLH * kLHP));
            const int kq = rem / kLHP, hp = rem - kq * kLHP;
            const int ci = find_seg(P.row_end, P.n_channels, task);
            const nlb_channel& ch = P.chan[ci];
            const int ap = (int)(task - (ci ? P.row_end[ci - 1] : 0));
            const int64_t rowlen = (int64_t)ch.np2 * kLHP;
            const T* Brow = t2 + ch.offset + ap * rowlen;
            const int row = ch.hb2 + kq;
            T acc = T(0);
            for (int q = P.fph_ptr[row]; q < P.fph_ptr[row + 1]; ++q)
                acc += (T)P.fph_val[q] * Brow[P.fph_col[q] * kLHP + hp];
            gb[v] = acc;
        }
    }
}

// Column pass over the multipliers Lam (current parity).  A block owns NB
// consecutive b' of one channel (a group of NH^2 threads per b', a thread per
// hole pair) and a chunk of the rows a'; per row it accumulates
//   Ha[k'][b'][hp]  += t1[a', k'] Lam[a'][b'][hp]                       (k' in H_g1)
//   Y1[b', k']      += Lam[a'][b'][(i', k')] (v_hh + v_pp) t1[a', i'] - Lam[a'][b'][hp] Gb[a'][k'][hp]
//   T[k', i'] (g1)  += Lam[a'][b'][i', j'] B[a'][b'][k', j']
//   T[k', j'] (g2)  += Lam[a'][b'][i', j'] B[a'][b'][i', k']
// and writes its partial sums into slots with one writer each (Ha per row
// chunk, Y1 per chunk, T per block), added in a fixed order afterwards.
constexpr int kColRows = 256;          // most rows in one chunk of the column pass

template <typename T, int NT>
__global__ void __launch_bounds__(NT, 2) k_l_cols(nlb_struct_problem P, nlb_lambda_state S, int nchunk) {
    constexpr int NB = NT / kLHP;
    __shared__ double sv[NT][kLH + 1];    // per-thread partial sums, one kind at a time
    __shared__ __align__(16) unsigned char smem_raw[kColRows * (8 + NB) * sizeof(T)];
    const nlb_ctrl* c = S.ctrl;
    if (c->status != NLB_RUNNING) return;
    const T* __restrict__ Lm = static_cast<const T*>(S.lam2[c->parity]);
    const T* __restrict__ B = static_cast<const T*>(S.t2);
    const T* __restrict__ gb = static_cast<const T*>(S.gb);
    T* __restrict__ ha = static_cast<T*>(S.ha);
    const PrepView PV = prep_view(S.prep, P);
    const LView V = lview(S.acc, P);
    const int tid = threadIdx.x;
    const int grp = tid / kLHP, hp = tid - grp * kLHP;
    const int ip = hp / kLH, jp = hp - ip * kLH;
    // work item -> (channel, b' block, row chunk)
    int64_t item = blockIdx.x;
    int ci = 0;
    for (; ci < P.n_channels; ++ci) {
        const int64_t nit = (int64_t)((P.chan[ci].np2 + NB - 1) / NB) * nchunk;
        if (item < nit) break;
        item -= nit;
    }
    if (ci >= P.n_channels) return;   // uniform over the block
    const nlb_channel& ch = P.chan[ci];
    const int bb = (int)(item / nchunk), chunk = (int)(item - (int64_t)bb * nchunk);
    const int a0 = (int)((int64_t)chunk * ch.np1 / nchunk), a1 = (int)((int64_t)(chunk + 1) * ch.np1 / nchunk);
    const int bp = bb * NB + grp;
    const bool act = grp < NB && bp < ch.np2;
    const int rowlen = ch.np2 * kLHP;
    T hak[kLH], ys[kLH], tt1[kLH], tt2[kLH];
    T ylt = T(0);
#pragma unroll
    for (int k = 0; k < kLH; ++k) { hak[k] = T(0); ys[k] = T(0); tt1[k] = T(0); tt2[k] = T(0); }
    const int64_t col = (int64_t)bp * kLHP + hp;   // element offset of (b', hp) in a row
    // the chunk's t1[a', H_g1] rows (8-padded) and pp ladder entries (a', b'),
    // staged once per block
    T* st1 = reinterpret_cast<T*>(smem_raw);                 // [nr][8]
    T* scpp = st1 + kColRows * 8;                            // [nr][NB]
    const int nr = a1 - a0;
    {
        const double* t1a = PV.t1c + P.t1c_base[ch.g1];
        const int32_t* pptr = P.pp_ptr + ch.pp_ptr_off;
        const double* pval = P.pp_val + ch.pp_col_off;
        for (int w = tid; w < nr * 8; w += NT) {
            const int r = w >> 3, k = w & 7;
            st1[w] = k < kLH ? (T)t1a[(a0 + r) * kLH + k] : T(0);
        }
        for (int w = tid; w < nr * NB; w += NT) {
            const int r = w / NB, g = w - r * NB;
            const int b2 = bb * NB + g;
            T v = T(0);
            if (b2 < ch.np2) {
                const int ab = (a0 + r) * ch.np2 + b2;
                if (pptr[ab + 1] > pptr[ab]) v = (T)pval[pptr[ab]];
            }
            scpp[w] = v;
        }
    }
    __syncthreads();
    if (act) {
        const int32_t* hptr = P.hh_ptr + ch.hh_ptr_off;
        const T shh = (hptr[hp + 1] > hptr[hp]) ? (T)P.hh_val[ch.hh_col_off + hptr[hp]] : T(0);
        const T* gbr = gb + (ci ? P.row_end[ci - 1] : 0) * (int64_t)(kLH * kLHP) + hp;
        const T* Lc = Lm + ch.offset + col;
        const T* Bb = B + ch.offset + (int64_t)bp * kLHP;   // block (a', b') of t2 at + a' rowlen
        // no barrier in the loop: every operand is an independent load (the
        // t2 block values come from L1 after the first touch); two rows per
        // step keep twice the loads in flight
        auto row = [&](int r, T x, const T (&bc)[kLH], const T (&br)[kLH], const T (&g)[kLH]) {
            T ta[8];
            lds8(st1 + r * 8, ta);
            const T cpp = scpp[r * NB + grp];
#pragma unroll
            for (int k = 0; k < kLH; ++k) {
                hak[k] += ta[k] * x;
                ys[k] += x * g[k];
                tt1[k] += x * bc[k];
                tt2[k] += x * br[k];
            }
            T tai = ta[0];
#pragma unroll
            for (int k = 1; k < kLH; ++k) tai = (ip == k) ? ta[k] : tai;
            ylt += x * (shh + cpp) * tai;
        };
        int r = 0;
        for (; r + 1 < nr; r += 2) {
            const int64_t ro0 = (int64_t)(a0 + r) * rowlen, ro1 = ro0 + rowlen;
            const T x0 = Lc[ro0], x1 = Lc[ro1];
            T bc0[kLH], br0[kLH], g0[kLH], bc1[kLH], br1[kLH], g1[kLH];
#pragma unroll
            for (int k = 0; k < kLH; ++k) {
                bc0[k] = __ldg(Bb + ro0 + k * kLH + jp);
                br0[k] = __ldg(Bb + ro0 + ip * kLH + k);
                g0[k] = __ldg(gbr + (int64_t)(a0 + r) * (kLH * kLHP) + k * kLHP);
                bc1[k] = __ldg(Bb + ro1 + k * kLH + jp);
                br1[k] = __ldg(Bb + ro1 + ip * kLH + k);
                g1[k] = __ldg(gbr + (int64_t)(a0 + r + 1) * (kLH * kLHP) + k * kLHP);
            }
            row(r, x0, bc0, br0, g0);
            row(r + 1, x1, bc1, br1, g1);
        }
        if (r < nr) {
            const int64_t ro0 = (int64_t)(a0 + r) * rowlen;
            const T x0 = Lc[ro0];
            T bc0[kLH], br0[kLH], g0[kLH];
#pragma unroll
            for (int k = 0; k < kLH; ++k) {
                bc0[k] = __ldg(Bb + ro0 + k * kLH + jp);
                br0[k] = __ldg(Bb + ro0 + ip * kLH + k);
                g0[k] = __ldg(gbr + (int64_t)(a0 + r) * (kLH * kLHP) + k * kLHP);
            }
            row(r, x0, bc0, br0, g0);
        }
        // this chunk's slice of Ha (one writer per element: no zeroing, no atomics)
        T* hc = ha + (int64_t)chunk * P.n_g + ch.ga_off;
#pragma unroll
        for (int k = 0; k < kLH; ++k) hc[(int64_t)k * rowlen + col] = hak[k];
    }
    // Y1[b', k'] of this chunk = sum over the group's hole pairs of -ys[k'] +
    // (k' == j') ylt, into the chunk's slot (the lattice path's uniform
    // channels give the column side the [b'][k'] layout of F2)
#pragma unroll
    for (int k = 0; k < kLH; ++k) sv[tid][k] = act ? (double)(-ys[k]) + (k == jp ? (double)ylt : 0.0) : 0.0;
    __syncthreads();
    for (int w = tid; w < NB * kLH; w += NT) {
        const int g2 = w / kLH, k = w % kLH;
        const int b2 = bb * NB + g2;
        if (b2 < ch.np2) {
            double s = 0.0;
            for (int q = 0; q < kLHP; ++q) s += sv[g2 * kLHP + q][k];
            V.Y1c[(int64_t)chunk * P.n_f2 + ch.f2_off + (int64_t)b2 * kLH + k] = s;
        }
    }
    __syncthreads();
    // T[k', i'] (g1) = sum over threads with that i'; then T[k', j'] (g2)
    // likewise, into this block's slot (k_l_treduce adds the blocks)
    double* tp = V.Tp + (int64_t)blockIdx.x * 2 * kLHP;
    for (int side = 0; side < 2; ++side) {
#pragma unroll
        for (int k = 0; k < kLH; ++k) sv[tid][k] = act ? (double)(side ? tt2[k] : tt1[k]) : 0.0;
        __syncthreads();
        for (int w = tid; w < kLHP; w += NT) {
            const int k = w / kLH, i = w % kLH;
            double s = 0.0;
            for (int g2 = 0; g2 < NB; ++g2)
                for (int o = 0; o < kLH; ++o) s += sv[g2 * kLHP + (side ? o * kLH + i : i * kLH + o)][k];
            tp[side * kLHP + w] = s;
        }
        __syncthreads();
    }
}

// The column pass's slots, added in a fixed order.  Blocks 0 ..
// n_labels * 49 - 1: T[k, m] for one (label g, local holes k', i'); the
// threads take the column-pass blocks strided (their g1 side and g2 side
// values), the block tree adds them.  The remaining blocks add the Ha chunk
// slices into slice 0, element by element in chunk order, for the row pass.
__global__ void k_l_treduce(nlb_struct_problem P, nlb_lambda_state S, int nchunk, int n_items, int elsize) {
    const nlb_ctrl* c = S.ctrl;
    if (c->status != NLB_RUNNING) return;
    const LView V = lview(S.acc, P);
    const int nt_out = P.n_labels * kLHP;
    if ((int)blockIdx.x < nt_out) {
        const int g = blockIdx.x / kLHP, w = blockIdx.x - g * kLHP;
        double s = 0.0;
        for (int it = threadIdx.x; it < n_items; it += blockDim.x) {
            // the channel of column-pass block `it` (numbered channel by channel)
            int64_t item0 = 0;
            int ci = 0;
            for (; ci < P.n_channels - 1; ++ci) {
                const int64_t nit = (int64_t)((P.chan[ci].np2 + kColNB - 1) / kColNB) * nchunk;
                if (it < item0 + nit) break;
                item0 += nit;
            }
            const nlb_channel& ch = P.chan[ci];
            if (ch.g1 == g) s += V.Tp[(int64_t)it * 2 * kLHP + w];
            if (ch.g2 == g) s += V.Tp[(int64_t)it * 2 * kLHP + kLHP + w];
        }
        s = block_sum(s);
        if (threadIdx.x == 0) {
            const int hb = P.h_base[g];
            V.T[(int64_t)P.h_ord[hb + w / kLH] * P.h + P.h_ord[hb + w % kLH]] = s;
        }
        return;
    }
    if (nchunk < 2) return;
    const int64_t nb = (int64_t)gridDim.x - nt_out;
    for (int64_t e = ((int64_t)blockIdx.x - nt_out) * blockDim.x + threadIdx.x; e < P.n_g; e += nb * blockDim.x) {
        if (elsize == 4) {
            float* ha = static_cast<float*>(S.ha);
            float v = ha[e];
            for (int cq = 1; cq < nchunk; ++cq) v += ha[(int64_t)cq * P.n_g + e];
            ha[e] = v;
        } else {
            double* ha = static_cast<double*>(S.ha);
            double v = ha[e];
            for (int cq = 1; cq < nchunk; ++cq) v += ha[(int64_t)cq * P.n_g + e];
            ha[e] = v;
        }
    }
}

// Shared-memory layout of k_l_lat for element size el and nb hole-pair groups.
struct LLat {
    int64_t row, hbp, rec, off, val, total;
};

__host__ __device__ inline LLat llat_smem(int64_t max_row, int nb, int64_t el) {
    const int64_t np2 = max_row / kLHP;
    LLat s;
    s.row = 0;
    s.hbp = lat_round16(el * (max_row + 16 / el + 4));
    s.rec = s.hbp + lat_round16(el * nb * kLH * kLHP);
    s.off = s.rec + lat_round16(el * np2 * kLRec);
    s.val = s.off + lat_round16(4 * np2 * kLNb);
    s.total = s.val + lat_round16(el * np2 * kLNb);
    return s;
}

// Row pass (after k_l_cols of the same step): Z2 of row a' and its Jacobi
// update, and the row's Z1 contributions of particle a'
//   Y1[a', k'] += -sum_e Lam[a'][e] Ga[k'][e] + sum_{b', j'} Lam[a'][b'][(k', j')] (v_hh + v_pp) t1[b', j'],
// laid out like the forward k_t2_lat: a thread keeps one hole pair for the
// whole row, the row sits in shared memory, the terms along a come from L2.
template <typename T, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_l_lat(nlb_struct_problem P, nlb_lambda_state S) {
    constexpr int NB = NT / kLHP;
    constexpr int VEC = 16 / (int)sizeof(T);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double sred[NT / 32][kLH];
    const nlb_ctrl* c = S.ctrl;
    if (c->status != NLB_RUNNING) return;
    const int par = c->parity;
    const T* __restrict__ Lm = static_cast<const T*>(S.lam2[par]);
    T* __restrict__ Lo = static_cast<T*>(S.lam2[par ^ 1]);
    const double* __restrict__ l1 = S.lam1[par];
    const T* __restrict__ Ga = static_cast<const T*>(S.ga);
    const T* __restrict__ Ha = static_cast<const T*>(S.ha);
    T* E2 = (S.diis_t2 != nullptr && c->max_diis > 0 && c->diis_count < c->max_diis)
                ? static_cast<T*>(S.diis_t2) + (int64_t)c->diis_count * P.n_t2 : nullptr;
    const PrepView PV = prep_view(S.prep, P);
    const LView V = lview(S.acc, P);
    const T om = (T)(1.0 - c->mixing);
    const LLat L = llat_smem(P.max_row, NB, sizeof(T));
    T* srow = reinterpret_cast<T*>(smem_raw + L.row);
    T* hbp = reinterpret_cast<T*>(smem_raw + L.hbp);       // [NB][k'][hp] partial Hb
    T* srec = reinterpret_cast<T*>(smem_raw + L.rec);      // [b'][kLRec]
    int32_t* soff = reinterpret_cast<int32_t*>(smem_raw + L.off);
    T* sval = reinterpret_cast<T*>(smem_raw + L.val);

    const int tid = threadIdx.x, h = P.h;
    const bool active = tid < NB * kLHP;
    const int grp = tid / kLHP, hp = tid - grp * kLHP;
    const int ip = hp / kLH, jp = hp - ip * kLH;
    const int lane = tid & 31, wid = tid >> 5;
    double dnrm = 0.0, lnrm = 0.0;
    int cur_ci = -1;
    T x1t[kLH], x2t[kLH], shh = T(0), dh = T(0);
    // work units: np2 b' columns per row, rows in channel order, cut into
    // gridDim.x equal contiguous ranges [w0, w1).  Every channel has np2 =
    // np1 = np and the grid is at most the row count, so a range is at
    // least np units long and a row lies in one block or in two consecutive
    // ones: the first writes the row's Z1 part to Y1r, the second to Y1q.
    int64_t W = 0;
    for (int cc = 0; cc < P.n_channels; ++cc) W += lat_units(P, cc);
    const int w0 = (int)((int64_t)blockIdx.x * W / gridDim.x);
    const int w1 = (int)((int64_t)(blockIdx.x + 1) * W / gridDim.x);
    int ci = 0, ap = 0, blo = 0, wc = 0;
    if (w0 < w1) {
        while (wc + lat_units(P, ci) <= w0) wc += (int)lat_units(P, ci++);
        const int u = P.chan[ci].np2 > 0 ? P.chan[ci].np2 : 1;
        ap = (w0 - wc) / u;
        blo = w0 - wc - ap * u;
    }
    while (w0 < w1) {
        const nlb_channel& ch = P.chan[ci];
        const int np2 = ch.np2;
        const int rowlen = np2 * kLHP;
        const int upp = np2 > 0 ? np2 : 1;                      // units per row
        const int wp = wc + ap * upp;                           // first unit of this row
        const int bhi = w1 - wp < np2 ? w1 - wp : np2;          // b' columns [blo, bhi)
        const int64_t rbase = ch.offset + (int64_t)ap * rowlen;
        const int a = P.p_ord[ch.pb1 + ap];
        // the row, asynchronously (ragged head, 16-byte middle, ragged tail)
        const T* Lrow = Lm + rbase;
        const int mis = (int)((reinterpret_cast<uintptr_t>(Lrow) / sizeof(T)) & (VEC - 1));
        T* sr = srow + mis;
        {
            const int head = min((VEC - mis) & (VEC - 1), rowlen);
            const int nvec = (rowlen - head) / VEC;
            const int tail0 = head + nvec * VEC;
            for (int e = tid; e < head; e += NT) cp_async_el<sizeof(T)>(sr + e, Lrow + e);
            for (int v = tid; v < nvec; v += NT) cp_async16(sr + head + v * VEC, Lrow + head + v * VEC);
            for (int e = tail0 + tid; e < rowlen; e += NT) cp_async_el<sizeof(T)>(sr + e, Lrow + e);
            cp_async_commit();
        }
        if (ci != cur_ci) {
            cur_ci = ci;
            const int x1b = P.xc_base[ch.g1], x2b = P.xc_base[ch.g2];
#pragma unroll
            for (int k = 0; k < kLH; ++k) {
                x1t[k] = (T)PV.xc[x1b + ip * kLH + k];
                x2t[k] = (T)PV.xc[x2b + jp * kLH + k];
            }
            const int32_t* hptr = P.hh_ptr + ch.hh_ptr_off;
            shh = (hptr[hp + 1] > hptr[hp]) ? (T)P.hh_val[ch.hh_col_off + hptr[hp]] : T(0);
            dh = (T)(PV.dhc[ch.hb1 + ip] + PV.dhc[ch.hb2 + jp]);
            const int t1b_b = P.t1c_base[ch.g2];
            for (int w = tid; w < np2 * kLNb; w += NT) {
                const int bq = w / kLNb, k = w - bq * kLNb;
                const int r0 = P.fpp_ptr[ch.pb2 + bq], r1 = P.fpp_ptr[ch.pb2 + bq + 1];
                soff[w] = ((k < r1 - r0) ? P.fpp_col[r0 + k] : bq) * kLHP;
                sval[w] = (k < r1 - r0) ? (T)P.fpp_val[r0 + k] : T(0);
                T* rec = srec + bq * kLRec;
                if (k < kLH) {
                    rec[k] = (T)V.fc[t1b_b + bq * kLH + k];
                    rec[8 + k] = (T)l1[(int64_t)P.p_ord[ch.pb2 + bq] * h + P.h_ord[ch.hb2 + k]];
                    rec[16 + k] = (T)PV.t1c[t1b_b + bq * kLH + k];
                } else {
                    bool nz = false;
                    for (int kk = 0; kk < kLH; ++kk) nz |= V.fc[t1b_b + bq * kLH + kk] != 0.0;
                    rec[7] = nz ? T(1) : T(0);   // f_ph row of b' not all zero
                }
            }
        }
        // per row: f_pp of a' (unused slots point at the row itself with
        // weight 0), f_ph and lam1 of a', pp ladder entries and denominators
        const int ra0 = P.fpp_ptr[ch.pb1 + ap], ra1 = P.fpp_ptr[ch.pb1 + ap + 1];
        T adiag = T(0);
        int aoff[kLNa];
        T aval[kLNa];
        {
            int q = ra0;
#pragma unroll
            for (int s = 0; s < kLNa; ++s) {
                aoff[s] = ap * rowlen;
                aval[s] = T(0);
                for (; q < ra1; ++q) {
                    const int colq = P.fpp_col[q];
                    if (colq == ap) { adiag += (T)P.fpp_val[q]; continue; }
                    aoff[s] = colq * rowlen;
                    aval[s] = (T)P.fpp_val[q];
                    ++q;
                    break;
                }
            }
            for (; q < ra1; ++q)
                if (P.fpp_col[q] == ap) adiag += (T)P.fpp_val[q];
        }
        const int fa_b = P.t1c_base[ch.g1] + ap * kLH;
        T sf1a[kLH];
        bool near = false;
#pragma unroll
        for (int k = 0; k < kLH; ++k) {
            sf1a[k] = (T)V.fc[fa_b + k];
            near |= sf1a[k] != T(0);
        }
        const T sf1ai = (T)V.fc[fa_b + ip];
        const T sl1a = (T)l1[(int64_t)a * h + P.h_ord[ch.hb1 + ip]];
        const double da = PV.dpc[ch.pb1 + ap];
        const int32_t* pptr = P.pp_ptr + ch.pp_ptr_off;
        const double* pval = P.pp_val + ch.pp_col_off;
        for (int bq = blo + tid; bq < bhi; bq += NT) {
            const int ab = ap * np2 + bq;
            srec[bq * kLRec + 15] = (pptr[ab + 1] > pptr[ab]) ? (T)pval[pptr[ab]] : T(0);
            srec[bq * kLRec + 23] = (T)(da + PV.dpc[ch.pb2 + bq]);
        }
        cp_async_wait_all();
        __syncthreads();
        // Hb[k'][hp] = sum_c t1[c, k'] Lam[a'][c][hp] (c in P_g2): group g takes c = g mod NB
        T hb[kLH];
        if (active) {
            T part[kLH];
#pragma unroll
            for (int k = 0; k < kLH; ++k) part[k] = T(0);
            for (int cq = grp; cq < np2; cq += NB) {
                const T v = sr[cq * kLHP + hp];
                T t[8];
                lds8(srec + cq * kLRec + 16, t);
#pragma unroll
                for (int k = 0; k < kLH; ++k) part[k] += t[k] * v;
            }
#pragma unroll
            for (int k = 0; k < kLH; ++k) hbp[(grp * kLH + k) * kLHP + hp] = part[k];
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < kLH; ++k) hb[k] = T(0);
        if (active) {
#pragma unroll
            for (int k = 0; k < kLH; ++k) {
                T s = T(0);
                for (int g = 0; g < NB; ++g) s += hbp[(g * kLH + k) * kLHP + hp];
                hb[k] = s;
            }
        }
        T acc_ga[kLH];
        T acc3 = T(0);
#pragma unroll
        for (int k = 0; k < kLH; ++k) acc_ga[k] = T(0);
        if (active && blo + grp < bhi) {
            const T* __restrict__ gL = Lm + ch.offset + hp;
            const T* __restrict__ gG = Ga + ch.ga_off + hp;
            const T* __restrict__ gH = Ha + ch.ga_off + hp;
            T* __restrict__ Lout = Lo + rbase + hp;
            T* __restrict__ Eout = E2 ? E2 + rbase + hp : nullptr;
            const T* s_hp = sr + hp;
            const T* s_col = sr + jp;            // Lam[a'][b'][k'][j'] at eb + k' NH
            const T* s_row = sr + ip * kLH;      // Lam[a'][b'][i'][k'] at eb + k'
            T nrm_d = T(0), nrm_l = T(0);
            for (int bq = blo + grp; bq < bhi; bq += NB) {
                const int eb = bq * kLHP;
                T nb[kLNa], gv[kLH];
#pragma unroll
                for (int q = 0; q < kLNa; ++q) nb[q] = __ldg(gL + aoff[q] + eb);
#pragma unroll
                for (int k = 0; k < kLH; ++k) gv[k] = __ldg(gG + k * rowlen + eb);
                const T x = s_hp[eb];
                const T* rec = srec + bq * kLRec;
                T f2[8], sv[8];
                int so[8];
                lds8(rec, f2);
                lds8(soff + bq * kLNb, so);
                lds8(sval + bq * kLNb, sv);
                // f_pp along b
                T zb = T(0);
#pragma unroll
                for (int q = 0; q < kLNb - 1; ++q) zb += sv[q] * s_hp[so[q]];
                // X_hh along i and j (transposed)
                T zx = T(0), zy = T(0);
#pragma unroll
                for (int k = 0; k < kLH; ++k) {
                    zx += x1t[k] * s_col[eb + k * kLH];
                    zy += x2t[k] * s_row[eb + k];
                }
                // rank-h parts: -f_ph[b', k'] Hb[k'] and -f_ph[a', k'] Ha[k'] (sparse f_ph)
                T zh = T(0);
                if (f2[7] != T(0)) {
#pragma unroll
                    for (int k = 0; k < kLH; ++k) zh += f2[k] * hb[k];
                }
                if (near) {
#pragma unroll
                    for (int k = 0; k < kLH; ++k) zh += sf1a[k] * __ldg(gH + k * rowlen + eb);
                }
                // f_pp along a
                T za = adiag * x;
#pragma unroll
                for (int q = 0; q < kLNa; ++q) za += aval[q] * nb[q];
                const T lad = shh + rec[15];
                const T f2j = rec[jp], l1bj = rec[8 + jp], t1bj = rec[16 + jp];
                const T Z = ((za + zb) - zh) + ((zx + zy) + lad * x) + (sl1a * f2j + l1bj * sf1ai);
                const T D = -(rec[23] + dh);
                const T out = x + lat_div(om * Z, D);
                __stcg(Lout + eb, out);
                const T d = out - x;
                if (Eout) __stcg(Eout + eb, d);
                nrm_d += d * d;
                nrm_l += out * out;
#pragma unroll
                for (int k = 0; k < kLH; ++k) acc_ga[k] += x * gv[k];
                acc3 += x * lad * t1bj;
            }
            dnrm += (double)nrm_d;
            lnrm += (double)nrm_l;
        }
        // Y1 of particle a': block sums of -acc_ga[k'] + (k' == i') acc3
#pragma unroll
        for (int k = 0; k < kLH; ++k) {
            double v = -(double)acc_ga[k] + ((active && k == ip) ? (double)acc3 : 0.0);
            v = warp_sum(v);
            if (lane == 0) sred[wid][k] = v;
        }
        __syncthreads();
        if (tid < kLH) {
            double s = 0.0;
            for (int w = 0; w < NT / 32; ++w) s += sred[w][tid];
            const int64_t o = ch.f2_off + (int64_t)ap * kLH + tid;
            if (blo > 0) {
                V.Y1q[o] = s;             // the rest of a row that the block before began
            } else {
                V.Y1r[o] = s;
                if (bhi == np2) V.Y1q[o] = 0.0;   // the whole row is this block's
            }
        }
        __syncthreads();
        if (wp + upp >= w1) break;
        ++ap;
        while (ap >= P.chan[ci].np1) {   // past the channel's last row
            wc += (int)lat_units(P, ci++);
            ap = 0;
        }
        blo = 0;
    }
    const double s1 = block_sum(dnrm);
    const double s2 = block_sum(lnrm);
    if (tid == 0) {
        PV.slots(kRedDt2)[blockIdx.x] = 4.0 * s1;
        PV.slots(kRedNrm2)[blockIdx.x] = 4.0 * s2;
    }
}

// =============================================================== host ==
int num_sms_l() {
    static int n = 0;
    if (n == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 148;
    }
    return n;
}

int optin_smem() {
    static int v = 0;
    if (v == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        if (v <= 0) v = 227 * 1024;
    }
    return v;
}

int grid_l(int64_t work) {
    const int64_t g = (work + kThreads - 1) / kThreads;
    const int64_t cap = (int64_t)num_sms_l() * 8;
    return (int)(g < 1 ? 1 : (g < cap ? g : cap));
}

int64_t l_smem(const nlb_struct_problem* P) {
    const int64_t mh = P->max_nh;
    return 8 * (2 * (int64_t)P->max_row + 2 * mh * mh * mh + 3 * mh * mh + 3 * mh);
}

constexpr int kLatThreads = 256;            // 5 hole-pair groups per block
constexpr int kColThreads = 256;

bool lattice(const nlb_struct_problem* P) {
    if (P->uniform_nh != kLH || !P->diag_ladders || P->max_fpp_offdiag > kLNa || P->n_t2 <= 0) return false;
    // every channel np1 = np2 = max_row / 49 (the column-side slots share the
    // row side's [particle][hole] layout): the row count and the amplitude
    // count reach their maxima only then
    const int64_t np = P->max_row / kLHP;
    if (P->n_rows != (int64_t)P->n_channels * np || P->n_t2 != (int64_t)P->n_channels * np * np * kLHP) return false;
    return llat_smem(P->max_row, kLatThreads / kLHP, 8).total + 1024 <= optin_smem();
}

int64_t gb_len(const nlb_struct_problem* P) { return P->n_rows * (int64_t)kLH * kLHP; }

// Blocks per SM of a kernel at a dynamic shared-memory size, queried once.
int lat_bps(const void* fn, int64_t smem, int threads) {
    static const void* fns[16] = {};
    static int64_t sms[16] = {};
    static int vals[16] = {};
    for (int k = 0; k < 16; ++k)
        if (fns[k] == fn && sms[k] == smem) return vals[k];
    // raise the limit to the device maximum (less the kernel's static shared
    // memory) for every kernel that takes dynamic shared memory: the 48 KB
    // default counts static shared memory too, and lowering the limit for a
    // smaller problem would break launches (and captured graphs) of a larger one
    if (smem > 0) {
        cudaFuncAttributes fa;
        if (cudaFuncGetAttributes(&fa, fn) == cudaSuccess)
            cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(optin_smem() - (int64_t)fa.sharedSizeBytes));
    }
    int bps = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, fn, threads, (size_t)smem) != cudaSuccess || bps < 1)
        bps = 1;
    for (int k = 0; k < 16; ++k)
        if (fns[k] == nullptr) { fns[k] = fn; sms[k] = smem; vals[k] = bps; break; }
    return bps;
}

// Row chunks of the column pass: about sixteen blocks per SM, at least
// eight rows per chunk.
int col_chunks(const nlb_struct_problem* P) {
    constexpr int NB = kColThreads / kLHP;
    const int64_t np = P->max_row / kLHP;
    const int64_t per = (np + NB - 1) / NB * P->n_channels;
    const int64_t want = (int64_t)num_sms_l() * 16;
    int64_t n = (want + per - 1) / (per > 0 ? per : 1);
    if (n > np / 8) n = np / 8;
    return (int)(n < 1 ? 1 : n);
}

template <typename T, int NT, int MINB>
int launch_llat(const nlb_struct_problem* P, const nlb_lambda_state* S, cudaStream_t s) {
    const int64_t sm = llat_smem(P->max_row, NT / kLHP, sizeof(T)).total;
    auto kern = k_l_lat<T, NT, MINB>;
    const int bps = lat_bps(reinterpret_cast<const void*>(kern), sm, NT);
    int64_t grid = (int64_t)num_sms_l() * bps;
    if (grid > P->n_rows) grid = P->n_rows;
    if (grid > kRedSlots) grid = kRedSlots;
    if (grid < 1) grid = 1;
    kern<<<(unsigned)grid, NT, (size_t)sm, s>>>(*P, *S);
    return (int)grid;
}

template <typename T>
int lat_step(const nlb_struct_problem* P, const nlb_lambda_state* S, cudaStream_t s) {
    constexpr int MINB = sizeof(T) == 4 ? 2 : 1;
    const int64_t hh = (int64_t)P->h * P->h;
    k_l_u<<<grid_l(32 * hh + (int64_t)P->p * P->h), kThreads, 0, s>>>(*P, *S);
    // every label has the same particle count on the lattice path; row
    // chunks from the tuning word (bits 8-15, 0: automatic), at most
    // kMaxColChunks (the slots of the column pass)
    constexpr int NB = kColThreads / kLHP;
    static_assert(NB == kColNB, "column-pass blocks");
    const int tuned = (P->tune >> 8) & 255;
    const int64_t np1 = P->max_row / kLHP;
    int nchunk = tuned > 0 ? (int)(tuned < np1 ? tuned : np1) : col_chunks(P);
    const int need = (int)((np1 + kColRows - 1) / kColRows);   // rows of a chunk fit the staging
    if (nchunk < need) nchunk = need;
    if (nchunk > kMaxColChunks) nchunk = kMaxColChunks;
    if (nchunk < need) return lfail(NLB_ERR_SIZE, "nlb_lambda_step: rows too long for the column pass");
    {
        const int64_t np2 = P->max_row / kLHP;
        const int64_t items = (np2 + NB - 1) / NB * nchunk * P->n_channels;
        k_l_cols<T, kColThreads><<<(unsigned)items, kColThreads, 0, s>>>(*P, *S, nchunk);
        const int hblocks = nchunk > 1 ? grid_l(P->n_g) : 0;
        k_l_treduce<<<P->n_labels * kLHP + hblocks, 128, 0, s>>>(*P, *S, nchunk, (int)items, (int)sizeof(T));
    }
    // row-pass launch shape from the tuning word (bits 4-7)
    int n2 = 0;
    if constexpr (sizeof(T) == 4) {
        if (((P->tune >> 4) & 15) == 1) n2 = launch_llat<T, 512, 1>(P, S, s);
        else n2 = launch_llat<T, kLatThreads, MINB>(P, S, s);
    } else {
        n2 = launch_llat<T, kLatThreads, MINB>(P, S, s);
    }
    if (cudaPeekAtLastError() != cudaSuccess) return lcheck("nlb_lambda_step");
    const int n1 = grid_l((int64_t)P->p * P->h);
    k_l_t1<<<n1, kThreads, 0, s>>>(*P, *S, nchunk);
    k_l_finish<<<1, 128, 0, s>>>(S->ctrl, prep_view(S->prep, *P).red, n1, n2);
    return lcheck("nlb_lambda_step");
}

}  // namespace

extern "C" {

int64_t nlb_lambda_acc_len(const nlb_struct_problem* prob) {
    if (!prob) return 0;
    const int64_t common = (int64_t)prob->p * prob->h + 2 * (int64_t)prob->h * prob->h + prob->n_t1c +
                           (int64_t)(2 + kMaxColChunks) * prob->n_f2 + col_items_max(*prob) * 2 * kLHP;
    if (lattice(prob)) return common;
    // general path: the row kernel's Yg and Tg slots
    return common + prob->n_t2 + prob->n_rows * 2 * (int64_t)prob->max_nh * prob->max_nh;
}

int64_t nlb_lambda_ha_len(const nlb_struct_problem* prob) {
    if (!prob) return 0;
    return lattice(prob) ? (int64_t)kMaxColChunks * prob->n_g : prob->n_g;
}

int64_t nlb_lambda_gb_len(const nlb_struct_problem* prob) {
    if (!prob || !lattice(prob)) return 0;
    return gb_len(prob);
}

int32_t nlb_lambda_lattice(const nlb_struct_problem* prob) { return (prob && lattice(prob)) ? 1 : 0; }

int nlb_lambda_init(const nlb_struct_problem* prob, const nlb_lambda_state* st, double tol, double mixing,
                    int32_t max_steps, int32_t max_diis, int32_t flags, nlb_stream_t stream) {
    if (!prob || !st || !st->ctrl || !st->t1 || !st->t2 || !st->prep || !st->ga || !st->ha || !st->acc)
        return lfail(NLB_ERR_ARG, "nlb_lambda_init: null argument");
    if (!st->lam1[0] || !st->lam1[1] || !st->lam2[0] || !st->lam2[1])
        return lfail(NLB_ERR_ARG, "nlb_lambda_init: null multiplier buffer");
    if (prob->diag_ladders != 1) return lfail(NLB_ERR_ARG, "nlb_lambda_init: ladders must be diagonal");
    if (st->dtype != NLB_F64 && st->dtype != NLB_F32) return lfail(NLB_ERR_ARG, "nlb_lambda_init: bad dtype");
    if (max_diis < 0 || max_diis > 10) return lfail(NLB_ERR_ARG, "nlb_lambda_init: max_diis must be in [0, 10]");
    if (max_diis > 0 && (!st->diis_t1 || !st->diis_t2)) return lfail(NLB_ERR_ARG, "nlb_lambda_init: null DIIS ring");
    const bool lat = lattice(prob);
    if (!lat) {
        if (st->dtype != NLB_F64) return lfail(NLB_ERR_ARG, "nlb_lambda_init: FP32 needs the lattice path");
        cudaFuncAttributes fa;
        cudaFuncGetAttributes(&fa, k_l_rows);
        if (l_smem(prob) + (int64_t)fa.sharedSizeBytes > optin_smem())
            return lfail(NLB_ERR_SIZE, "nlb_lambda_init: a row does not fit in shared memory");
    } else if (!st->gb) {
        return lfail(NLB_ERR_ARG, "nlb_lambda_init: null Gb table");
    }
    cudaStream_t s = (cudaStream_t)stream;
    const size_t el = st->dtype == NLB_F64 ? 8 : 4;
    if (!(flags & NLB_LAMBDA_KEEP)) {
        cudaMemsetAsync(st->lam1[0], 0, sizeof(double) * prob->p * prob->h, s);
        cudaMemsetAsync(st->lam2[0], 0, el * prob->n_t2, s);
    }
    cudaMemsetAsync(st->lam1[1], 0, sizeof(double) * prob->p * prob->h, s);
    cudaMemsetAsync(st->lam2[1], 0, el * prob->n_t2, s);
    const int64_t nprep = (int64_t)prob->h * prob->h + 2 * (int64_t)prob->p + prob->n_t1c + prob->n_xc + prob->h;
    if (lat) {
        const int64_t tot = nprep + prob->n_g + prob->n_t1c + gb_len(prob);
        if (st->dtype == NLB_F64) k_l_setup_lat<double><<<grid_l(tot), kThreads, 0, s>>>(*prob, *st);
        else k_l_setup_lat<float><<<grid_l(tot), kThreads, 0, s>>>(*prob, *st);
    } else {
        k_l_setup<<<grid_l(nprep + prob->n_g + prob->n_t1c), kThreads, 0, s>>>(*prob, *st);
    }
    k_l_init<<<1, 32, 0, s>>>(st->ctrl, tol, mixing, max_steps, max_diis);
    return lcheck("nlb_lambda_init");
}

int nlb_lambda_step(const nlb_struct_problem* prob, const nlb_lambda_state* st, nlb_stream_t stream) {
    if (!prob || !st || !st->ctrl) return lfail(NLB_ERR_ARG, "nlb_lambda_step: null argument");
    cudaStream_t s = (cudaStream_t)stream;
    if (lattice(prob)) return st->dtype == NLB_F64 ? lat_step<double>(prob, st, s) : lat_step<float>(prob, st, s);
    if (st->dtype != NLB_F64) return lfail(NLB_ERR_ARG, "nlb_lambda_step: FP32 needs the lattice path");
    const int64_t hh = (int64_t)prob->h * prob->h;
    k_l_u<<<grid_l(32 * hh + (int64_t)prob->p * prob->h), kThreads, 0, s>>>(*prob, *st);
    k_l_ha<<<grid_l(prob->n_g), kThreads, 0, s>>>(*prob, *st);
    const int64_t sm = l_smem(prob);
    const int bps = lat_bps(reinterpret_cast<const void*>(k_l_rows), sm, kThreads);
    int64_t grid = (int64_t)num_sms_l() * bps;
    if (grid > prob->n_rows) grid = prob->n_rows;
    if (grid > kRedSlots) grid = kRedSlots;
    if (grid < 1) grid = 1;
    k_l_rows<<<(unsigned)grid, kThreads, (size_t)sm, s>>>(*prob, *st);
    k_l_rows_reduce<<<grid_l((int64_t)prob->p * prob->h + hh), kThreads, 0, s>>>(*prob, *st);
    const int n1 = grid_l((int64_t)prob->p * prob->h);
    k_l_t1<<<n1, kThreads, 0, s>>>(*prob, *st, 0);
    k_l_finish<<<1, 128, 0, s>>>(st->ctrl, prep_view(st->prep, *prob).red, n1, (int)grid);
    return lcheck("nlb_lambda_step");
}

int nlb_lambda_diis(const nlb_struct_problem* prob, const nlb_lambda_state* st, int32_t max_diis,
                    nlb_stream_t stream) {
    if (!prob || !st || !st->ctrl) return lfail(NLB_ERR_ARG, "nlb_lambda_diis: null argument");
    // the forward DIIS kernels on a view of the multipliers
    nlb_struct_state v = {};
    v.t1[0] = st->lam1[0];
    v.t1[1] = st->lam1[1];
    v.t2[0] = st->lam2[0];
    v.t2[1] = st->lam2[1];
    v.g = st->ha;
    v.f2 = st->acc;
    v.prep = st->prep;
    v.ctrl = st->ctrl;
    v.diis_t1 = st->diis_t1;
    v.diis_t2 = st->diis_t2;
    v.dtype = st->dtype;
    return nlb_struct_diis(prob, &v, max_diis, stream);
}

int nlb_lambda_coupling(const nlb_struct_problem* prob, const nlb_lambda_state* st, const double* dw,
                        const double* dv, double* out, nlb_stream_t stream) {
    if (!prob || !st || !dw || !dv || !out) return lfail(NLB_ERR_ARG, "nlb_lambda_coupling: null argument");
    if (st->dtype != NLB_F64) return lfail(NLB_ERR_ARG, "nlb_lambda_coupling: needs the FP64 state");
    if (!st->prep) return lfail(NLB_ERR_ARG, "nlb_lambda_coupling: null prep");
    cudaStream_t s = (cudaStream_t)stream;
    const int nb = grid_l(prob->n_t2);
    k_l_coupling<<<nb, kThreads, 0, s>>>(*prob, *st, dw, dv, out);
    k_l_sum_slots<<<1, 32, 0, s>>>(prep_view(st->prep, *prob).slots(0), nb, out);
    return lcheck("nlb_lambda_coupling");
}

}  // extern "C"
