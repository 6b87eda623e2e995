// Lattice T2 update, two rows per pass (FP32 amplitudes, seven holes per
// label).  Included by ccsd_struct.cu inside its anonymous namespace.
//
// The same terms as k_t2_lat (CCM/coupled_cluster.py:498-536,
// CCM/ccDgrams.py:215-251, 502-578 on the compact channel layout), but a
// block works on two rows a0', a1' of one channel at a time, and a thread
// holds the same (b', i', j') of both rows as one FP32x2 register pair:
//
// * the two rows are staged in shared memory interleaved (element e of row
//   r at 2e + r, copied by 4-byte cp.async, double buffered), so every
//   shared load along b, i and j is one 8-byte load that serves both rows,
//   and every multiply-add on it is one packed FFMA2;
// * the Ga values of (b', i'j') do not depend on a', so the seven L2 loads
//   of the rank-h term along a serve both rows;
// * the per-b' record (f_pp row of b' with its columns, t1 of b', the
//   ladder entries and denominators of both rows) is read once for both;
// * Gb[k'][i'j'] of both rows stays in registers for the whole row pair.
//
// Only the f_pp neighbours along a (six L2 loads per row) stay per row.
//
// Work split: the passes of a channel are its rows (0, 1), (2, 3), ... and,
// when the channel has an odd number of rows, the last row alone (its
// partner slot a copy of it whose results are dropped).  A pass is
// max(np2, 1) work units, one per b' column; the units of all passes, in
// channel order, are cut into gridDim.x contiguous ranges of equal length.
// So a block may start or end inside a pass: it then stages both rows and
// forms Gb as a whole pass does, but updates only the b' columns of its
// range, and the block holding column 0 writes the pass's F2 entries.  With
// whole passes per block the rows would not divide evenly (1254 rows on 148
// blocks at L=6: four passes on some blocks, five on others).

constexpr int kPairRec = 32;   // floats per b' record

// Work units of channel cc: passes of two rows, max(np2, 1) units each.
__device__ __forceinline__ int64_t pair_units(const nlb_struct_problem& P, int cc) {
    const nlb_channel& c = P.chan[cc];
    return (int64_t)((c.np1 + 1) / 2) * (c.np2 > 0 ? c.np2 : 1);
}

// Per-b' record (32 floats): [0,14) (f_pp value q, same value) pairs for the
// seven slots of the f_pp row of b'; [14], [15] the pp ladder entries of
// (a0', b') and (a1', b'); [16, 23) t1[b', k'], [23] zero; [24], [25] the
// particle denominators of (a0', b') and (a1', b').
struct PairSmem {
    int64_t st0, st1, gb, rec, off, total;
};

__host__ __device__ inline PairSmem pair_smem(int64_t max_row) {
    const int64_t np2 = max_row / 49;
    PairSmem s;
    s.st0 = 0;
    s.st1 = lat_round16(8 * max_row);
    s.gb = 2 * s.st1;
    s.rec = s.gb + lat_round16(8 * 343);
    s.off = s.rec + lat_round16(4 * np2 * kPairRec);
    s.total = s.off + lat_round16(4 * np2 * kLatNb);
    return s;
}

// Queue the interleaved copy of rows src0 and src1 (rowlen elements each).
template <int NT>
__device__ __forceinline__ void pair_issue(float* dst, const float* src0, const float* src1, int rowlen) {
    for (int e = threadIdx.x; e < rowlen; e += NT) {
        cp_async_el<4>(dst + 2 * e, src0 + e);
        cp_async_el<4>(dst + 2 * e + 1, src1 + e);
    }
    cp_async_commit();
}

__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 ffma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

// Row a' of channel ch: its f_pp neighbours along a (off-diagonal, at most
// kLatNa; unused slots weight 0 and the row itself), the diagonal, t1[a', H]
// and t1[a', i'].
struct PairRowA {
    int aoff[kLatNa];
    float aval[kLatNa];
    float adiag;
};

__device__ __forceinline__ void pair_row_a(const nlb_struct_problem& P, const nlb_channel& ch, int ap, int rowlen,
                                           PairRowA& r) {
    const int ra0 = P.fpp_ptr[ch.pb1 + ap], ra1 = P.fpp_ptr[ch.pb1 + ap + 1];
    float adiag = 0.f;
    int q = ra0;
#pragma unroll
    for (int s = 0; s < kLatNa; ++s) {
        r.aoff[s] = ap * rowlen;
        r.aval[s] = 0.f;
        for (; q < ra1; ++q) {
            const int col = P.fpp_col[q];
            if (col == ap) { adiag += (float)P.fpp_val[q]; continue; }
            r.aoff[s] = col * rowlen;
            r.aval[s] = (float)P.fpp_val[q];
            ++q;
            break;
        }
    }
    for (; q < ra1; ++q)
        if (P.fpp_col[q] == ap) adiag += (float)P.fpp_val[q];
    r.adiag = adiag;
}

template <int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_t2_pair(nlb_struct_problem P, nlb_struct_state S) {
    constexpr int NH = 7, NHP = 49;
    constexpr int NB = NT / NHP;
    static_assert(NB >= 1, "block must hold one hole-pair group");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const nlb_ctrl* c = S.ctrl;
    if (c->status != NLB_RUNNING || c->ccs) return;
    const int par = c->parity;
    const float* __restrict__ B = static_cast<const float*>(S.t2[par]);
    float* __restrict__ Bo = static_cast<float*>(S.t2[par ^ 1]);
    const float* __restrict__ Ga = static_cast<const float*>(S.g);
    float* __restrict__ F2 = static_cast<float*>(S.f2);
    const PrepView V = prep_view(S.prep, P);
    float* E2 = (S.diis_t2 != nullptr && c->max_diis > 0 && c->diis_count < c->max_diis)
                    ? static_cast<float*>(S.diis_t2) + (int64_t)c->diis_count * P.n_t2 : nullptr;
    const float m = (float)c->mixing, om = (float)(1.0 - c->mixing);
    const float2 md = f2(m, m), omd = f2(om, om);
    const PairSmem L = pair_smem(P.max_row);
    float2* sgb = reinterpret_cast<float2*>(smem_raw + L.gb);      // Gb[k'][i'j'] of (row 0, row 1)
    float* srec = reinterpret_cast<float*>(smem_raw + L.rec);      // [b'][kPairRec]
    int32_t* soff = reinterpret_cast<int32_t*>(smem_raw + L.off);  // [b'][8] f_pp columns * NHP

    const int tid = threadIdx.x;
    const bool active = tid < NB * NHP;
    const int grp = tid / NHP, hp = tid - grp * NHP;
    const int ip = hp / NH, jp = hp - ip * NH;
    double nrm = 0.0;
    int cur_ci = -1;
    float2 x1d[NH], x2d[NH], hhd = f2(0.f, 0.f), dhd = f2(0.f, 0.f);

    // the block's units [w0, w1): first channel ci (units from wc), pass pi
    int64_t W = 0;
    for (int cc = 0; cc < P.n_channels; ++cc) W += pair_units(P, cc);
    // (W is below 2^31: the lattice path holds a row in shared memory)
    const int w0 = (int)((int64_t)blockIdx.x * W / gridDim.x);
    const int w1 = (int)((int64_t)(blockIdx.x + 1) * W / gridDim.x);
    int ci = 0, pi = 0, blo = 0, wc = 0;
    if (w0 < w1) {
        while (wc + pair_units(P, ci) <= w0) wc += (int)pair_units(P, ci++);
        const int u = P.chan[ci].np2 > 0 ? P.chan[ci].np2 : 1;
        pi = (w0 - wc) / u;
        blo = w0 - wc - pi * u;
    }
    // rows 2pi and (2pi + 1, or 2pi again when alone) of channel cc
    auto issue = [&](int cc, int pp, int stage) {
        const nlb_channel& cn = P.chan[cc];
        const int rl = cn.np2 * NHP;
        const float* s0 = B + cn.offset + (int64_t)(2 * pp) * rl;
        pair_issue<NT>(reinterpret_cast<float*>(smem_raw + (stage ? L.st1 : L.st0)), s0,
                       2 * pp + 1 < cn.np1 ? s0 + rl : s0, rl);
    };
    if (w0 < w1) issue(ci, pi, 0);
    for (int pass = 0; w0 < w1; ++pass) {
        const int buf = pass & 1;
        const nlb_channel& ch = P.chan[ci];
        const bool two = 2 * pi + 1 < ch.np1;
        const int ap0 = 2 * pi, ap1 = two ? ap0 + 1 : ap0;
        const int np2 = ch.np2;
        const int rowlen = np2 * NHP;
        const int upp = np2 > 0 ? np2 : 1;                      // units per pass
        const int wp = wc + pi * upp;                           // first unit of this pass
        const int bhi = w1 - wp < np2 ? w1 - wp : np2;          // b' columns [blo, bhi)
        const float2* S2 = reinterpret_cast<const float2*>(smem_raw + (buf ? L.st1 : L.st0));

        // per-channel tables (the block's rows are contiguous: usually unchanged)
        if (ci != cur_ci) {
            cur_ci = ci;
            const int x1b = P.xc_base[ch.g1], x2b = P.xc_base[ch.g2];
#pragma unroll
            for (int k = 0; k < NH; ++k) {
                const float a = (float)V.xc[x1b + k * NH + ip], b = (float)V.xc[x2b + k * NH + jp];
                x1d[k] = f2(a, a);
                x2d[k] = f2(b, b);
            }
            const int32_t* hptr = P.hh_ptr + ch.hh_ptr_off;
            const float hv = (hptr[hp + 1] > hptr[hp]) ? (float)P.hh_val[ch.hh_col_off + hptr[hp]] : 0.f;
            const float dv = (float)(V.dhc[ch.hb1 + ip] + V.dhc[ch.hb2 + jp]);
            hhd = f2(hv, hv);
            dhd = f2(dv, dv);
            const int t1b_b = P.t1c_base[ch.g2];
            for (int w = tid; w < np2 * kLatNb; w += NT) {
                const int bp = w / kLatNb, k = w - bp * kLatNb;
                const int r0 = P.fpp_ptr[ch.pb2 + bp], r1 = P.fpp_ptr[ch.pb2 + bp + 1];
                soff[w] = ((k < r1 - r0) ? P.fpp_col[r0 + k] : bp) * NHP;
                if (k < NH) {
                    const float v = (k < r1 - r0) ? (float)P.fpp_val[r0 + k] : 0.f;
                    const float t = (float)V.t1c[t1b_b + bp * NH + k];
                    float* rp = srec + bp * kPairRec;
                    rp[2 * k] = v;
                    rp[2 * k + 1] = v;
                    rp[16 + 2 * k] = t;
                    rp[17 + 2 * k] = t;
                }
            }
        }
        // per-row tables of both rows
        PairRowA ra0, ra1;
        pair_row_a(P, ch, ap0, rowlen, ra0);
        pair_row_a(P, ch, ap1, rowlen, ra1);
        float2 avp[kLatNa];
#pragma unroll
        for (int q = 0; q < kLatNa; ++q) avp[q] = f2(ra0.aval[q], ra1.aval[q]);
        const float2 adg = f2(ra0.adiag, ra1.adiag);
        const int t1a_b0 = P.t1c_base[ch.g1] + ap0 * NH, t1a_b1 = P.t1c_base[ch.g1] + ap1 * NH;
        float2 ta0[3], ta1[3];
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            ta0[j] = f2((float)V.t1c[t1a_b0 + 2 * j], (float)V.t1c[t1a_b0 + 2 * j + 1]);
            ta1[j] = f2((float)V.t1c[t1a_b1 + 2 * j], (float)V.t1c[t1a_b1 + 2 * j + 1]);
        }
        const float ta0_6 = (float)V.t1c[t1a_b0 + 6], ta1_6 = (float)V.t1c[t1a_b1 + 6];
        const float2 t1ai = f2((float)V.t1c[t1a_b0 + ip], (float)V.t1c[t1a_b1 + ip]);
        {
            const double da0 = V.dpc[ch.pb1 + ap0], da1 = V.dpc[ch.pb1 + ap1];
            const int32_t* pptr = P.pp_ptr + ch.pp_ptr_off;
            const double* pval = P.pp_val + ch.pp_col_off;
            for (int bp = blo + tid; bp < bhi; bp += NT) {
                const int ab0 = ap0 * np2 + bp, ab1 = ap1 * np2 + bp;
                float* rp = srec + bp * kPairRec;
                rp[14] = (pptr[ab0 + 1] > pptr[ab0]) ? (float)pval[pptr[ab0]] : 0.f;
                rp[15] = (pptr[ab1 + 1] > pptr[ab1]) ? (float)pval[pptr[ab1]] : 0.f;
                const double dp = V.dpc[ch.pb2 + bp];
                rp[30] = (float)(da0 + dp);
                rp[31] = (float)(da1 + dp);
            }
        }
        cp_async_wait_all();
        __syncthreads();
        // next pass in flight while this one is worked on (its buffer was last
        // read by the pass before, which ended with a barrier)
        const bool more = wp + upp < w1;
        int nci = ci, npi = pi + 1, nwc = wc;
        if (more) {
            while (2 * npi >= P.chan[nci].np1) {   // past the channel's last pass
                nwc += (int)pair_units(P, nci++);
                npi = 0;
            }
            issue(nci, npi, buf ^ 1);
        }
        // Gb[k'][i'j'] = sum_c f_ck B[a'][c'][i'j'] of both rows (holes k of
        // label g2), then the T1 Fock terms F2[a'][i'] of both rows
        for (int e = tid; e < NH * NHP; e += NT) {
            const int kq = e / NHP, h2 = e - kq * NHP;
            const int row = ch.hb2 + kq;
            float2 acc = f2(0.f, 0.f);
            for (int q = P.fph_ptr[row]; q < P.fph_ptr[row + 1]; ++q) {
                const float v = (float)P.fph_val[q];
                acc = ffma2(f2(v, v), S2[P.fph_col[q] * NHP + h2], acc);
            }
            sgb[e] = acc;
        }
        __syncthreads();
        if (blo == 0 && tid < 2 * NH && (tid < NH || two)) {
            const int r = tid / NH, i = tid - r * NH;
            float acc = 0.f;
#pragma unroll
            for (int kq = 0; kq < NH; ++kq) {
                const float2 g = sgb[kq * NHP + i * NH + kq];
                acc = __fadd_rn(acc, r ? g.y : g.x);
            }
            F2[ch.f2_off + (int64_t)(r ? ap1 : ap0) * NH + i] = acc;
        }
        if (active && blo + grp < bhi) {
            float2 gb[NH];
#pragma unroll
            for (int k = 0; k < NH; ++k) gb[k] = sgb[k * NHP + hp];
            const float* __restrict__ gBc = B + ch.offset + hp;
            const float* __restrict__ gG = Ga + ch.ga_off + hp;    // Ga[b'][k'][i'j']: k' at stride NHP
            const int64_t r0 = ch.offset + (int64_t)ap0 * rowlen + hp, r1 = ch.offset + (int64_t)ap1 * rowlen + hp;
            float* __restrict__ Bout0 = Bo + r0;
            float* __restrict__ Bout1 = Bo + r1;
            float* __restrict__ Eout0 = E2 ? E2 + r0 : nullptr;
            float* __restrict__ Eout1 = E2 ? E2 + r1 : nullptr;
            float2 nrm2 = f2(0.f, 0.f);
            // the L2 loads of a b' step: f_pp neighbours along a of both rows,
            // and the Ga values (shared by both rows) as k' pairs
            auto load = [&](int bp, float2 (&nb)[kLatNa], float2 (&gp)[3], float& g6) {
                const int eb = bp * NHP;
#pragma unroll
                for (int q = 0; q < kLatNa; ++q) nb[q] = f2(__ldg(gBc + ra0.aoff[q] + eb), __ldg(gBc + ra1.aoff[q] + eb));
                const float* g = gG + eb * NH;
#pragma unroll
                for (int j = 0; j < 3; ++j) gp[j] = f2(__ldg(g + 2 * j * NHP), __ldg(g + (2 * j + 1) * NHP));
                g6 = __ldg(g + 6 * NHP);
            };
            // the element (b', i', j') of both rows given its terms along a
            auto step = [&](int bp, const float2 (&nb)[kLatNa], const float2 (&gp)[3], float g6) {
                const int eb = bp * NHP;
                const float4* rp = reinterpret_cast<const float4*>(srec + bp * kPairRec);
                float2 fq[8], tq[8];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const float4 a = rp[u], b = rp[4 + u];
                    fq[2 * u] = f2(a.x, a.y);
                    fq[2 * u + 1] = f2(a.z, a.w);
                    tq[2 * u] = f2(b.x, b.y);
                    tq[2 * u + 1] = f2(b.z, b.w);
                }
                int so[8];
                lds8(soff + bp * kLatNb, so);
                const float2 xv = S2[eb + hp];
                // f_pp along b; rank-h part along b: t1_bk Gb[k]
                float2 pb = f2(0.f, 0.f), pg = f2(0.f, 0.f);
#pragma unroll
                for (int q = 0; q < NH; ++q) pb = ffma2(fq[q], S2[so[q] + hp], pb);
#pragma unroll
                for (int k = 0; k < NH; ++k) pg = ffma2(tq[k], gb[k], pg);
                // X_hh along i and along j
                float2 xi = f2(0.f, 0.f), xj = f2(0.f, 0.f);
#pragma unroll
                for (int k = 0; k < NH; ++k) {
                    xi = ffma2(x1d[k], S2[eb + k * NH + jp], xi);
                    xj = ffma2(x2d[k], S2[eb + ip * NH + k], xj);
                }
                // along a: f_pp neighbours, and the rank-h part t1_ak Ga[k]
                // (per row, over pairs of k')
                float2 pa = __fmul2_rn(adg, xv);
#pragma unroll
                for (int q = 0; q < kLatNa; ++q) pa = ffma2(avp[q], nb[q], pa);
                float2 g0 = f2(0.f, 0.f), g1 = f2(0.f, 0.f);
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    g0 = ffma2(ta0[j], gp[j], g0);
                    g1 = ffma2(ta1[j], gp[j], g1);
                }
                const float2 ga = f2(__fmaf_rn(ta0_6, g6, __fadd_rn(g0.x, g0.y)), __fmaf_rn(ta1_6, g6, __fadd_rn(g1.x, g1.y)));
                // both ladders act on tau = t2 + t1 t1
                const float2 tbj = *reinterpret_cast<const float2*>(srec + bp * kPairRec + 16 + 2 * jp);
                const float2 lad = __fmul2_rn(__fadd2_rn(hhd, fq[7]), ffma2(t1ai, tbj, xv));
                const float2 acc = __fadd2_rn(__fadd2_rn(__fadd2_rn(pa, f2(-ga.x, -ga.y)), __fadd2_rn(pb, f2(-pg.x, -pg.y))),
                                              __fadd2_rn(__fadd2_rn(xi, xj), lad));
                const float2 dd = __fadd2_rn(tq[7], dhd);
                const float2 tn = f2(__fsub_rn(xv.x, __fdividef(acc.x, dd.x)), __fsub_rn(xv.y, __fdividef(acc.y, dd.y)));
                const float2 out = ffma2(md, xv, __fmul2_rn(omd, tn));
                __stcg(Bout0 + eb, out.x);
                if (two) __stcg(Bout1 + eb, out.y);
                const float2 d = __fadd2_rn(out, f2(-xv.x, -xv.y));
                if (Eout0) {
                    __stcg(Eout0 + eb, d.x);
                    if (two) __stcg(Eout1 + eb, d.y);
                }
                nrm2 = ffma2(d, d, nrm2);
            };
            // the L2 loads of one b' step go out a step ahead of its math
            float2 nA[kLatNa], gA[3], nB[kLatNa], gB2[3];
            float g6A, g6B;
            load(blo + grp, nA, gA, g6A);
            for (int bp = blo + grp; bp < bhi; bp += 2 * NB) {
                const int b1 = bp + NB;
                load(b1 < bhi ? b1 : bp, nB, gB2, g6B);
                step(bp, nA, gA, g6A);
                if (b1 >= bhi) break;
                const int b2 = b1 + NB;
                load(b2 < bhi ? b2 : b1, nA, gA, g6A);
                step(b1, nB, gB2, g6B);
            }
            nrm += (double)nrm2.x;
            if (two) nrm += (double)nrm2.y;
        }
        __syncthreads();
        if (!more) break;
        ci = nci;
        pi = npi;
        wc = nwc;
        blo = 0;
    }
    const double s = block_sum(nrm);
    if (threadIdx.x == 0) V.slots(kRedDt2)[blockIdx.x] = 4.0 * s;
}
