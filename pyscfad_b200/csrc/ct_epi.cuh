// Device helpers shared by the orbit epilogue kernels (float64 path in
// ct_fp64.cu, pipelined float path in ct_epi_f32.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include "ct_common.cuh"

namespace ctb {

// 16-byte asynchronous global -> shared copy (no register round-trip)
__device__ __forceinline__ void cp_async16(void *smem_dst, const void *gmem_src) {
    const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(smem_dst));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// W-bar storage of the epilogue: WB 0 = the scratch type as is (float64 path);
// 1 = float rounded to the nearest tf32 (it feeds tf32 tensor-core GEMMs, whose
// MMA would otherwise truncate); 2 = float kept whole in shared memory and
// written out as bf16 hi/lo planes (BF16x3).
template <typename ST, int WB> __device__ __forceinline__ ST wbar_store(double x) {
    if (WB == 1) {
        uint32_t r;
        asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"((float)x));
        return (ST)__uint_as_float(r);
    }
    return (ST)x;
}

// Element of a block-orbit owned by thread slot q.  T = 8, 256 threads: each
// warp covers a 2 x 4 x 4 sub-cube (u x w x t), so no coordinate spans more
// than 4 values within a warp; otherwise the canonical order.
template <int T, int NTHR>
__device__ __forceinline__ void loc_of(int q, int (&loc)[3]) {
    if (T == 8 && NTHR == 256) {
        const int wq = q & 31, wi = q >> 5;
        loc[2] = (wq & 3) | ((wi & 1) << 2);
        loc[1] = ((wq >> 2) & 3) | (((wi >> 1) & 1) << 2);
        loc[0] = ((wq >> 4) & 1) | (((wi >> 2) & 3) << 1);
    } else {
        loc[0] = q / (T * T);
        loc[1] = (q / T) % T;
        loc[2] = q % T;
    }
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }

// r3 over the six slots of an element orbit, y[s] = sum_t kR3C(t) x[kComp(s,t)]
// (weights 4 for the identity, -2 for the transpositions, 1 for the 3-cycles;
// add_and_permute, ccsd_t.c:98-119).  Row s of kComp is a permutation of the
// six slots, so with S = sum(x) this is 6 x[s] + 3 (x[kComp(s,3)] +
// x[kComp(s,4)]) - 2 S: three operations per slot after the shared sum instead
// of six multiply-adds.
template <typename AT> __device__ __forceinline__ void r3_orbit(const AT (&x)[6], AT (&y)[6]) {
    const AT tot = ((x[0] + x[1]) + (x[2] + x[3])) + (x[4] + x[5]);
    const AT m2s = (AT)-2 * tot;
#pragma unroll
    for (int s = 0; s < 6; ++s) y[s] = (AT)6 * x[s] + ((AT)3 * (x[kComp(s, 3)] + x[kComp(s, 4)]) + m2s);
}

// One element orbit {perm(i,j,k)} of a staged block-orbit (I,J,K) = (BI,BJ,BK):
// W, V, r3, the denominator, the job-energy contribution and (vjp) the
// backward quantities, all in registers (ccsd_t_vjp.c:9-117 per element;
// lno_ccsd_t.c:6-29).  Staged tiles: Gs[sigma][buffer d] blocks of BLK
// elements with u-stride TP, V tiles VA/VB[sigma][slot][T^2], t1/fvo rows
// Us/Ws[sigma][64].  Writes W-bar in place into Gs, ybar to Yg (the job's
// ybar slot) and this element's mo_energy-bar partial to tmp_s.
// AT is the arithmetic type of W, V, r3 and the bars (double on the float64
// path, float on the mixed path); the denominator, the energy terms and the
// mo_energy-bar partials are float64 in both.
//
// DIRECT: W-bar goes straight to the job's slots in global memory (Sg = slot
// 0, slot stride o^3) instead of into Gs.  TMP_OUT: the element's
// mo_energy-bar partial is returned in tmp_out instead of tmp_s.
// QRT: the job's slots are qr-tiled (the mixed path's layout): element (i,j,k)
// of a slot at i o^2 + (j/8) 8o + (k/8) 64 + (j%8) 8 + k%8; else plain (i,j,k).
// YST: ybar goes to a shared-memory staging buffer Yg laid out like the G
// tiles (index off[s]) instead of to global memory; the caller flushes it.
template <typename AT, typename ST, typename VT, int T, int TP, int BLK, int WB, bool DIRECT = false,
          bool TMP_OUT = DIRECT, bool QRT = false, bool YST = false>
__device__ __forceinline__ void orbit_element(const int (&loc)[3], int BI, int BJ, int BK, const int (&dmap)[6],
                                              ST *Gs, const VT *VA, const VT *VB, const VT *Us, const VT *Ws,
                                              const double *eocc, double *tmp_s, ST *Yg, int o, double fac,
                                              double eabc, double eb, bool vjp, KSum &eacc, double &vir_acc,
                                              bool with_fvo = true, ST *Sg = nullptr, double *tmp_out = nullptr,
                                              bool lno = false) {
    constexpr int T2 = T * T;
    const int cq = (loc[0] * T + loc[1]) * T + loc[2];   // canonical slot of this element
    if (TMP_OUT) *tmp_out = 0.0;
    else tmp_s[cq] = 0.0;
    const int ijk[3] = {BI * T + loc[0], BJ * T + loc[1], BK * T + loc[2]};
    auto gidx = [o](int i, int j, int k) -> long long {
        return QRT ? (long long)i * o * o + (j >> 3) * 8 * o + (k >> 3) * 64 + (j & 7) * 8 + (k & 7)
                   : ((long long)i * o + j) * o + k;
    };
    if (ijk[0] >= o || ijk[1] >= o || ijk[2] >= o) return;
    if ((BI == BJ && loc[0] < loc[1]) || (BJ == BK && loc[1] < loc[2])) return;
    int off[6], gr[6];
    int lp[6][2];
#pragma unroll
    for (int s = 0; s < 6; ++s) {
        off[s] = dmap[s] * BLK + loc[kR(s, 0)] * TP + loc[kR(s, 1)] * T + loc[kR(s, 2)];
        lp[s][0] = loc[kR(s, 0)];
        lp[s][1] = loc[kR(s, 1)];
        gr[s] = ijk[kR(s, 2)];
    }
    bool first[6];
#pragma unroll
    for (int s = 0; s < 6; ++s) {
        bool f = true;
#pragma unroll
        for (int t = 0; t < s; ++t) f = f && (off[t] != off[s]);
        first[s] = f;
    }
    AT W[6], Y[6], Z[6];
#pragma unroll
    for (int s = 0; s < 6; ++s) {
        AT ws = 0, vs = 0;
#pragma unroll
        for (int sg = 0; sg < 6; ++sg) {
            const int cs = kComp(s, sg);
            ws += (AT)Gs[sg * 6 * BLK + off[cs]];
            const int vi = (sg * 6 + cs) * T2 + lp[cs][0] * T + lp[cs][1];
            vs += (AT)VA[vi] * (AT)Us[sg * 64 + gr[cs]];
            if (with_fvo) vs += (AT)VB[vi] * (AT)Ws[sg * 64 + gr[cs]];
        }
        W[s] = ws;
        Y[s] = ws + (AT)0.5 * vs;
    }
    r3_orbit<AT>(Y, Z);
    // one reciprocal per element: d3 = fac / D; the orbit's distinct W.Z
    // products share d3, so they are summed before the compensated add, and
    // the mo_energy-bar partial eb d3^2 / fac = eb fac / D^2 reuses 1/D
    const double rden = 1.0 / (eocc[ijk[0]] + eocc[ijk[1]] + eocc[ijk[2]] - eabc);
    const double d3 = fac * rden;
    double wz = 0.0;
#pragma unroll
    for (int s = 0; s < 6; ++s)
        if (first[s]) wz += (double)W[s] * (double)Z[s];
    eacc.add(wz * d3);
    if (lno) {
        // LNO energy (no VJP): the W cube into slot 0 and z/D into slot 1 of
        // the staged tiles, at the orbit's own positions (read above by this
        // thread only); the projection follows in a separate kernel
#pragma unroll
        for (int s = 0; s < 6; ++s) {
            Gs[off[s]] = (ST)W[s];
            Gs[6 * BLK + off[s]] = (ST)((double)Z[s] * rden);
        }
        return;
    }
    if (vjp) {
        const AT ebd3 = (AT)(eb * d3);
        AT zb[6], wb[6];
        const double tmp = eb * d3 * rden * wz;
#pragma unroll
        for (int s = 0; s < 6; ++s) {
            zb[s] = ebd3 * W[s];
            wb[s] = ebd3 * Z[s];
        }
        AT yb[6];
        r3_orbit<AT>(zb, yb);
#pragma unroll
        for (int s = 0; s < 6; ++s) wb[s] += yb[s];
        if (TMP_OUT) *tmp_out = tmp;
        else tmp_s[cq] = tmp;
        vir_acc += tmp;
        if (DIRECT) {
            // global positions of the orbit's elements; a position shared by
            // several slots keeps the last slot's value, as the in-place path does
            const long long o3 = (long long)o * o * o;
            long long gi[6];
            bool last[6];
#pragma unroll
            for (int s2 = 0; s2 < 6; ++s2) {
                gi[s2] = gidx(ijk[kR(s2, 0)], ijk[kR(s2, 1)], ijk[kR(s2, 2)]);
                bool l = true;
#pragma unroll
                for (int t = s2 + 1; t < 6; ++t) l = l && (off[t] != off[s2]);
                last[s2] = l;
            }
#pragma unroll
            for (int sg = 0; sg < 6; ++sg)
#pragma unroll
                for (int s2 = 0; s2 < 6; ++s2)
                    if (last[s2]) Sg[sg * o3 + gi[s2]] = wbar_store<ST, WB>((double)wb[kComp(s2, kInv(sg))]);
        } else {
#pragma unroll
            for (int sg = 0; sg < 6; ++sg)
#pragma unroll
                for (int s = 0; s < 6; ++s) Gs[sg * 6 * BLK + off[s]] = wbar_store<ST, WB>((double)wb[kComp(s, kInv(sg))]);
        }
        // ybar straight to its slot (each element of the cube belongs to one orbit)
#pragma unroll
        for (int s = 0; s < 6; ++s)
            if (first[s]) {
                if (YST) Yg[off[s]] = (ST)yb[s];
                else Yg[gidx(ijk[kR(s, 0)], ijk[kR(s, 1)], ijk[kR(s, 2)])] = (ST)yb[s];
            }
    }
}

// LNO backward for one element orbit (lno_ccsd_t_vjp.c:73-140 on the sorted
// job's cubes).  Tile groups 0-4 hold q = z/D and the two parts (axes 1-2,
// axis 0) of A = sum_t wt_t M_t(w) and B = sum_t wt_t M_t^T(q) at the orbit's
// slot positions (groups 1 + 3 and 2 + 4); the energy is
// sum A q, so z_bar = eb A / D, w_bar = eb B + r3(z_bar), v_bar = r3(z_bar)
// (the canonical chain of orbit_element with those two products replaced)
// and the mo_energy-bar partial is eb A q / D.  W-bar goes in place into
// groups 0-5 (stored as wbar_store<ST, WB>), ybar to its slot.  Arithmetic
// in float64 on both paths (there is no V term to form here).
// TMP_OUT, QRT, YST as for orbit_element: the partial returned in tmp_out;
// ybar addressed in the qr-tiled layout; ybar into the staging tiles Yg.
template <typename ST, int T, int TP, int BLK, int WB = 0, bool TMP_OUT = false, bool QRT = false,
          bool YST = false>
__device__ __forceinline__ void orbit_lno_bar(const int (&loc)[3], int BI, int BJ, int BK, const int (&dmap)[6],
                                              ST *Gs, const double *eocc, double *tmp_s, ST *Yg, int o, double eabc,
                                              double eb, double &vir_acc, double *tmp_out = nullptr) {
    const int cq = (loc[0] * T + loc[1]) * T + loc[2];
    if (TMP_OUT) *tmp_out = 0.0;
    else tmp_s[cq] = 0.0;
    const int ijk[3] = {BI * T + loc[0], BJ * T + loc[1], BK * T + loc[2]};
    if (ijk[0] >= o || ijk[1] >= o || ijk[2] >= o) return;
    if ((BI == BJ && loc[0] < loc[1]) || (BJ == BK && loc[1] < loc[2])) return;
    int off[6];
#pragma unroll
    for (int s = 0; s < 6; ++s) off[s] = dmap[s] * BLK + loc[kR(s, 0)] * TP + loc[kR(s, 1)] * T + loc[kR(s, 2)];
    bool first[6];
#pragma unroll
    for (int s = 0; s < 6; ++s) {
        bool f = true;
#pragma unroll
        for (int t = 0; t < s; ++t) f = f && (off[t] != off[s]);
        first[s] = f;
    }
    const double rden = 1.0 / (eocc[ijk[0]] + eocc[ijk[1]] + eocc[ijk[2]] - eabc);
    double zb[6], wb[6], aq = 0.0;
#pragma unroll
    for (int s = 0; s < 6; ++s) {
        const double q = Gs[off[s]];
        const double A = (double)Gs[6 * BLK + off[s]] + (double)Gs[18 * BLK + off[s]];
        const double B = (double)Gs[12 * BLK + off[s]] + (double)Gs[24 * BLK + off[s]];
        zb[s] = eb * A * rden;
        wb[s] = eb * B;
        if (first[s]) aq += A * q;
    }
    const double tmp = eb * rden * aq;
    double yb[6];
#pragma unroll
    for (int s = 0; s < 6; ++s) {
        double t = 0.0;
#pragma unroll
        for (int u = 0; u < 6; ++u) t += kR3C(u) * zb[kComp(s, u)];
        yb[s] = t;
        wb[s] += t;
    }
    if (TMP_OUT) *tmp_out = tmp;
    else tmp_s[cq] = tmp;
    vir_acc += tmp;
#pragma unroll
    for (int sg = 0; sg < 6; ++sg)
#pragma unroll
        for (int s = 0; s < 6; ++s) Gs[sg * 6 * BLK + off[s]] = wbar_store<ST, WB>(wb[kComp(s, kInv(sg))]);
#pragma unroll
    for (int s = 0; s < 6; ++s)
        if (first[s]) {
            if (YST) {
                Yg[off[s]] = (ST)yb[s];
            } else {
                const int i = ijk[kR(s, 0)], j = ijk[kR(s, 1)], k = ijk[kR(s, 2)];
                const long long gi = QRT ? (long long)i * o * o + (j >> 3) * 8 * o + (k >> 3) * 64 + (j & 7) * 8 + (k & 7)
                                         : ((long long)i * o + j) * o + k;
                Yg[gi] = (ST)yb[s];
            }
        }
}

// Iterative (T) seed for one element orbit (pyscfad/cc/ccsd_t_slow.py:188-220
// on the 6-D amplitudes).  The job (a, b, c)'s cubes W and W + V, formed as in
// orbit_element, are P6(w)[., a, b, c] and P6(w + v)[., a, b, c]; P6 makes the
// 6-D arrays invariant under a simultaneous permutation of (i, j, k) and
// (a, b, c), and D (= d3) under any permutation of either, so slot s's element
// (i, j, k) = pos gives t3_c[pi(a,b,c)][pi(pos)] = (W + V)[s] / D and
// t3_x[pi(a,b,c)][pi(pos)] = r3(W)[s] / 3 (the energy is sum t3 t3_x, :210-220)
// for each of the six permutations pi.  Layout [a][b][c][i][j][k].
template <typename ST, typename VT, int T, int TP, int BLK>
__device__ __forceinline__ void orbit_t3(const int (&loc)[3], int BI, int BJ, int BK, const int (&dmap)[6],
                                         const ST *Gs, const VT *VA, const VT *VB, const VT *Us, const VT *Ws,
                                         const double *eocc, int o, int v, double eabc, int a, int b, int c,
                                         double *t3c, double *t3x) {
    constexpr int T2 = T * T;
    const int ijk[3] = {BI * T + loc[0], BJ * T + loc[1], BK * T + loc[2]};
    if (ijk[0] >= o || ijk[1] >= o || ijk[2] >= o) return;
    if ((BI == BJ && loc[0] < loc[1]) || (BJ == BK && loc[1] < loc[2])) return;
    int off[6], gr[6], lp[6][2];
#pragma unroll
    for (int s = 0; s < 6; ++s) {
        off[s] = dmap[s] * BLK + loc[kR(s, 0)] * TP + loc[kR(s, 1)] * T + loc[kR(s, 2)];
        lp[s][0] = loc[kR(s, 0)];
        lp[s][1] = loc[kR(s, 1)];
        gr[s] = ijk[kR(s, 2)];
    }
    double W[6], Y[6], R[6];
#pragma unroll
    for (int s = 0; s < 6; ++s) {
        double ws = 0, vs = 0;
#pragma unroll
        for (int sg = 0; sg < 6; ++sg) {
            const int cs = kComp(s, sg);
            ws += (double)Gs[sg * 6 * BLK + off[cs]];
            const int vi = (sg * 6 + cs) * T2 + lp[cs][0] * T + lp[cs][1];
            vs += (double)VA[vi] * (double)Us[sg * 64 + gr[cs]] + (double)VB[vi] * (double)Ws[sg * 64 + gr[cs]];
        }
        W[s] = ws;
        Y[s] = ws + 0.5 * vs;
    }
    r3_orbit<double>(W, R);
    const double rden = 1.0 / (eocc[ijk[0]] + eocc[ijk[1]] + eocc[ijk[2]] - eabc);
    const int abc[3] = {a, b, c};
    const long long o3 = (long long)o * o * o;
#pragma unroll
    for (int s = 0; s < 6; ++s) {
        const int pos[3] = {ijk[kR(s, 0)], ijk[kR(s, 1)], ijk[kR(s, 2)]};
        const double yc = Y[s] * rden, xr = R[s] * (1.0 / 3.0);
#pragma unroll
        for (int pi = 0; pi < 6; ++pi) {
            const long long ia = ((long long)abc[kR(pi, 0)] * v + abc[kR(pi, 1)]) * v + abc[kR(pi, 2)];
            const long long ii = ((long long)pos[kR(pi, 0)] * o + pos[kR(pi, 1)]) * o + pos[kR(pi, 2)];
            t3c[ia * o3 + ii] = yc;
            t3x[ia * o3 + ii] = xr;
        }
    }
}

}  // namespace ctb
