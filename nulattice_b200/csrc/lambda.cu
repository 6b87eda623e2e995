// Adjoint (CC Lambda) kernels of the structured engine, FP64, sm_100a.
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
// with the forward Jacobi denominators and mixing.

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

// scratch layout (doubles): Y1[p*h] Z1 contributions gathered from T2 rows,
// U[h*h] = t1^T lam1, T[h*h] X_hh contractions, fc[n_t1c] f_ph per label.
struct LView {
    double *Y1, *U, *T, *fc;
};

__host__ __device__ inline LView lview(double* acc, const nlb_struct_problem& P) {
    LView v;
    v.Y1 = acc;
    v.U = v.Y1 + (int64_t)P.p * P.h;
    v.T = v.U + (int64_t)P.h * P.h;
    v.fc = v.T + (int64_t)P.h * P.h;
    return v;
}

// Tables at the converged amplitudes: prep, Ga, and the per-label f_ph copy.
__global__ void k_l_setup(nlb_struct_problem P, nlb_lambda_state S) {
    const int64_t nprep = (int64_t)P.h * P.h + 2 * (int64_t)P.p + P.n_t1c + P.n_xc + P.h;
    const LView V = lview(S.acc, P);
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < nprep + P.n_g + P.n_t1c; u += stride) {
        if (u < nprep) {
            prep_body(P, S.t1, S.prep, u);
        } else if (u < nprep + P.n_g) {
            S.ga[u - nprep] = ga_element(P, S.t2, u - nprep);
        } else {
            const int64_t q = u - nprep - P.n_g;
            const int g = find_label(P.t1c_base, P.n_labels, q);
            const int nh = P.h_base[g + 1] - P.h_base[g];
            const int loc = (int)(q - P.t1c_base[g]);
            const int ap = loc / nh, kq = loc - ap * nh;
            V.fc[q] = P.f_ph[(int64_t)P.p_ord[P.p_base[g] + ap] * P.h + P.h_ord[P.h_base[g] + kq]];
        }
    }
}

// U = t1^T lam1 and zeroed accumulators.
__global__ void k_l_prep(nlb_struct_problem P, nlb_lambda_state S) {
    const nlb_ctrl* c = S.ctrl;
    if (c->status != NLB_RUNNING) return;
    const double* l1 = S.lam1[c->parity];
    const LView V = lview(S.acc, P);
    const int h = P.h, p = P.p;
    const int64_t hh = (int64_t)h * h, ph = (int64_t)p * h;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < 2 * hh + ph; u += stride) {
        if (u < hh) {
            const int k = (int)(u / h), m = (int)(u % h);
            double s = 0.0;
            for (int a = 0; a < p; ++a) s += S.t1[(int64_t)a * h + k] * l1[(int64_t)a * h + m];
            V.U[u] = s;
        } else if (u < 2 * hh) {
            V.T[u - hh] = 0.0;
        } else {
            V.Y1[u - 2 * hh] = 0.0;
        }
    }
}

// Ha[k'][e] = sum_a' t1[a,k] Lam[a'][e] (k in H_g1), laid out like Ga.
__global__ void k_l_ha(nlb_struct_problem P, nlb_lambda_state S) {
    const nlb_ctrl* c = S.ctrl;
    if (c->status != NLB_RUNNING) return;
    const double* Lm = S.lam2[c->parity];
    const PrepView PV = prep_view(S.prep, P);
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < P.n_g; u += stride) {
        const int ci = find_seg(P.g_end, P.n_channels, u);
        const nlb_channel ch = P.chan[ci];
        const int rowlen = ch.np2 * ch.nh1 * ch.nh2;
        const int loc = (int)(u - ch.ga_off);
        const int kq = loc / rowlen, e = loc - kq * rowlen;
        const double* t1a = PV.t1c + P.t1c_base[ch.g1] + kq;
        const double* col = Lm + ch.offset + e;
        double acc = 0.0;
        for (int ap = 0; ap < ch.np1; ++ap) acc += t1a[ap * ch.nh1] * col[(int64_t)ap * rowlen];
        S.ha[u] = acc;
    }
}

// One block per row task (channel, a'): Z2 and the Jacobi update of the row,
// and the row's contributions to Z1 (through Y1) and to T.
__global__ void __launch_bounds__(kThreads) k_l_rows(nlb_struct_problem P, nlb_lambda_state S) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const nlb_ctrl* c = S.ctrl;
    if (c->status != NLB_RUNNING) return;
    const int par = c->parity;
    const double* __restrict__ Lm = S.lam2[par];
    double* __restrict__ Lo = S.lam2[par ^ 1];
    const double* __restrict__ l1 = S.lam1[par];
    const double* __restrict__ B = S.t2;
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
        const nlb_channel ch = P.chan[ci];
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
            for (int k = 0; k < nh1; ++k) Z -= sf1a[k] * S.ha[ch.ga_off + (int64_t)k * rowlen + e];
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
            atomicAdd(&V.Y1[(int64_t)P.p_ord[ch.pb2 + bp] * h + P.h_ord[ch.hb2 + kq]], lt - s);
        }
        // X_hh contractions T along i (g1) and along j (g2)
        for (int w = tid; w < nh1 * nh1 + nh2 * nh2; w += nt) {
            double s = 0.0;
            if (w < nh1 * nh1) {
                const int kq = w / nh1, iq = w - kq * nh1;
                for (int bp = 0; bp < np2; ++bp)
                    for (int jq = 0; jq < nh2; ++jq)
                        s += lrow[bp * nhp + iq * nh2 + jq] * brow[bp * nhp + kq * nh2 + jq];
                atomicAdd(&V.T[(int64_t)P.h_ord[ch.hb1 + kq] * h + P.h_ord[ch.hb1 + iq]], s);
            } else {
                const int w2 = w - nh1 * nh1;
                const int kq = w2 / nh2, jq = w2 - kq * nh2;
                for (int bp = 0; bp < np2; ++bp)
                    for (int iq = 0; iq < nh1; ++iq)
                        s += lrow[bp * nhp + iq * nh2 + jq] * brow[bp * nhp + iq * nh2 + kq];
                atomicAdd(&V.T[(int64_t)P.h_ord[ch.hb2 + kq] * h + P.h_ord[ch.hb2 + jq]], s);
            }
        }
        // particle a' of label g1: -sum_e Lam Ga[k'] and the ladder t1 term
        for (int q = 0; q < 2 * nh1; ++q) {
            double part = 0.0;
            if (q < nh1) {
                for (int e = tid; e < rowlen; e += nt) part += lrow[e] * S.ga[ch.ga_off + (int64_t)q * rowlen + e];
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
            if (tid == 0) atomicAdd(&V.Y1[(int64_t)a * h + P.h_ord[ch.hb1 + (q % nh1)]], tot);
        }
        __syncthreads();
    }
    const double s1 = block_sum(dnrm);
    const double s2 = block_sum(lnrm);
    if (tid == 0) {
        atomicAdd(&S.ctrl->dt2_sq, 4.0 * s1);
        atomicAdd(&S.ctrl->e_acc, 4.0 * s2);
    }
}

// Z1 and the Jacobi update of lam1.
__global__ void k_l_t1(nlb_struct_problem P, nlb_lambda_state S) {
    nlb_ctrl* c = S.ctrl;
    if (c->status != NLB_RUNNING) return;
    const int par = c->parity;
    const double* l1 = S.lam1[par];
    double* lo = S.lam1[par ^ 1];
    const PrepView PV = prep_view(S.prep, P);
    const LView V = lview(S.acc, P);
    const int h = P.h, p = P.p;
    const double m = c->mixing;
    double dn = 0.0, ln = 0.0;
    for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < (int64_t)p * h;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(idx / h), mm = (int)(idx % h);
        const int g = P.p_label[x];
        if (P.h_label[mm] != g) {
            lo[idx] = 0.0;
            continue;
        }
        double Z = P.f_ph[idx] + V.Y1[idx];
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
        dn += (out - l1[idx]) * (out - l1[idx]);
        ln += out * out;
    }
    const double s1 = block_sum(dn);
    const double s2 = block_sum(ln);
    if (threadIdx.x == 0) {
        atomicAdd(&c->dt1_sq, s1);
        atomicAdd(&c->e_acc, s2);
    }
}

// convergence on the relative step of the multipliers
__global__ void k_l_finish(nlb_ctrl* c) {
    if (threadIdx.x != 0 || blockIdx.x != 0 || c->status != NLB_RUNNING) return;
    c->iter += 1;
    c->parity ^= 1;
    const double step = sqrt(c->dt1_sq + c->dt2_sq), size = sqrt(c->e_acc);
    c->e_last = step;
    if (step < c->eps * fmax(1.0, size)) c->status = NLB_CONVERGED;
    else if (!(step == step) || step > 1e12) c->status = NLB_DIVERGED;
    else if (c->iter >= c->max_steps) c->status = NLB_MAX_ITER;
    c->dt1_sq = 0.0;
    c->dt2_sq = 0.0;
    c->e_acc = 0.0;
}

__global__ void k_l_init(nlb_ctrl* c, double tol, double mixing, int max_steps) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    c->e_acc = 0.0; c->dt1_sq = 0.0; c->dt2_sq = 0.0; c->e_prev = 0.0; c->e_last = 0.0;
    c->eps = tol; c->mixing = mixing;
    c->parity = 0; c->iter = 0; c->status = max_steps > 0 ? NLB_RUNNING : NLB_MAX_ITER; c->max_steps = max_steps;
    c->criterion = 0; c->max_diis = 0; c->diis_count = 0; c->diis_pulse = 0; c->diis_applied = 0; c->ccs = 0;
}

// <Lam, (dW + dV) tau> over the compact layout for a derivative Hamiltonian
// whose ladders are diagonal: dw[hh_ptr_off + hp], dv[pp_ptr_off + ab].
__global__ void k_l_coupling(nlb_struct_problem P, nlb_lambda_state S, const double* dw, const double* dv,
                             double* out) {
    const double* Lm = S.lam2[S.ctrl->parity];
    const PrepView PV = prep_view(S.prep, P);
    double acc = 0.0;
    for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < P.n_t2; u += (int64_t)gridDim.x * blockDim.x) {
        const int ci = find_seg(P.t2_end, P.n_channels, u);
        const nlb_channel ch = P.chan[ci];
        const int64_t loc = u - ch.offset;
        const int nhp = ch.nh1 * ch.nh2;
        const int hp = (int)(loc % nhp);
        const int ab = (int)(loc / nhp);
        const int ap = ab / ch.np2, bp = ab - ap * ch.np2;
        const int ip = hp / ch.nh2, jp = hp - ip * ch.nh2;
        const double tau = S.t2[u] + PV.t1c[P.t1c_base[ch.g1] + ap * ch.nh1 + ip] *
                                         PV.t1c[P.t1c_base[ch.g2] + bp * ch.nh2 + jp];
        acc += Lm[u] * (dw[ch.hh_ptr_off + hp] + dv[ch.pp_ptr_off + ab]) * tau;
    }
    const double s = block_sum(acc);
    if (threadIdx.x == 0) atomicAdd(out, s);
}

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

int grid_l(int64_t work) {
    const int64_t g = (work + kThreads - 1) / kThreads;
    const int64_t cap = (int64_t)num_sms_l() * 8;
    return (int)(g < 1 ? 1 : (g < cap ? g : cap));
}

int64_t l_smem(const nlb_struct_problem* P) {
    const int64_t mh = P->max_nh;
    return 8 * (2 * (int64_t)P->max_row + 2 * mh * mh * mh + 3 * mh * mh + 3 * mh);
}

}  // namespace

extern "C" {

int64_t nlb_lambda_acc_len(const nlb_struct_problem* prob) {
    if (!prob) return 0;
    return (int64_t)prob->p * prob->h + 2 * (int64_t)prob->h * prob->h + prob->n_t1c;
}

int nlb_lambda_init(const nlb_struct_problem* prob, const nlb_lambda_state* st, double tol, double mixing,
                    int32_t max_steps, nlb_stream_t stream) {
    if (!prob || !st || !st->ctrl || !st->t1 || !st->t2 || !st->prep || !st->ga || !st->ha || !st->acc)
        return lfail(NLB_ERR_ARG, "nlb_lambda_init: null argument");
    if (!st->lam1[0] || !st->lam1[1] || !st->lam2[0] || !st->lam2[1])
        return lfail(NLB_ERR_ARG, "nlb_lambda_init: null multiplier buffer");
    if (prob->diag_ladders != 1) return lfail(NLB_ERR_ARG, "nlb_lambda_init: ladders must be diagonal");
    {
        int dev = 0, optin = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        cudaFuncAttributes fa;
        cudaFuncGetAttributes(&fa, k_l_rows);
        if (optin <= 0 || l_smem(prob) + (int64_t)fa.sharedSizeBytes > optin)
            return lfail(NLB_ERR_SIZE, "nlb_lambda_init: a row does not fit in shared memory");
    }
    cudaStream_t s = (cudaStream_t)stream;
    cudaMemsetAsync(st->lam1[0], 0, sizeof(double) * prob->p * prob->h, s);
    cudaMemsetAsync(st->lam1[1], 0, sizeof(double) * prob->p * prob->h, s);
    cudaMemsetAsync(st->lam2[0], 0, sizeof(double) * prob->n_t2, s);
    cudaMemsetAsync(st->lam2[1], 0, sizeof(double) * prob->n_t2, s);
    const int64_t nprep = (int64_t)prob->h * prob->h + 2 * (int64_t)prob->p + prob->n_t1c + prob->n_xc + prob->h;
    k_l_setup<<<grid_l(nprep + prob->n_g + prob->n_t1c), kThreads, 0, s>>>(*prob, *st);
    k_l_init<<<1, 32, 0, s>>>(st->ctrl, tol, mixing, max_steps);
    return lcheck("nlb_lambda_init");
}

int nlb_lambda_step(const nlb_struct_problem* prob, const nlb_lambda_state* st, nlb_stream_t stream) {
    if (!prob || !st || !st->ctrl) return lfail(NLB_ERR_ARG, "nlb_lambda_step: null argument");
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t hh = (int64_t)prob->h * prob->h;
    k_l_prep<<<grid_l(2 * hh + (int64_t)prob->p * prob->h), kThreads, 0, s>>>(*prob, *st);
    k_l_ha<<<grid_l(prob->n_g), kThreads, 0, s>>>(*prob, *st);
    const int64_t sm = l_smem(prob);
    static int64_t attr_bytes = 0;
    if (sm > 48 * 1024 && sm > attr_bytes) {
        if (cudaFuncSetAttribute(k_l_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) != cudaSuccess)
            return lcheck("nlb_lambda_step: shared memory request");
        attr_bytes = sm;
    }
    int bps = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k_l_rows, kThreads, (size_t)sm);
    int64_t grid = (int64_t)num_sms_l() * (bps > 0 ? bps : 1);
    if (grid > prob->n_rows) grid = prob->n_rows;
    if (grid < 1) grid = 1;
    k_l_rows<<<(unsigned)grid, kThreads, (size_t)sm, s>>>(*prob, *st);
    k_l_t1<<<grid_l((int64_t)prob->p * prob->h), kThreads, 0, s>>>(*prob, *st);
    k_l_finish<<<1, 32, 0, s>>>(st->ctrl);
    return lcheck("nlb_lambda_step");
}

int nlb_lambda_coupling(const nlb_struct_problem* prob, const nlb_lambda_state* st, const double* dw,
                        const double* dv, double* out, nlb_stream_t stream) {
    if (!prob || !st || !dw || !dv || !out) return lfail(NLB_ERR_ARG, "nlb_lambda_coupling: null argument");
    cudaStream_t s = (cudaStream_t)stream;
    cudaMemsetAsync(out, 0, sizeof(double), s);
    k_l_coupling<<<grid_l(prob->n_t2), kThreads, 0, s>>>(*prob, *st, dw, dv, out);
    return lcheck("nlb_lambda_coupling");
}

}  // extern "C"
