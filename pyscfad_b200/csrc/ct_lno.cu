// LNO-projected (T): the projections of a sorted job's W and q = z/D cubes by
// the occupied projector mat, on the float64 tensor pipe (DMMA m8n8k4).
//
// lnoccsdt_contract (lno_ccsd_t.c:6-138) runs the ordered jobs (x, y, z) with
// y >= z (factor 1/2 when y == z) and contracts (sum_l mat[l,i] w[l,j,k])
// z[i,j,k] / D over ijk: it projects the occupied index paired with x.  On a
// sorted job's cubes w[p,q,r] and q[p,q,r] every such ordering is the
// projection on the axis t that carries x, so the job's sum is
//   E = sum_t wt_t sum_{l,k} mat[l,k] G_t[l,k],
//   G_t[l,k] = sum over the fibers f of axis t (the other two indices) of w_f[l] q_f[k],
// with weights a>b>c: (1, 1, 1); a>b=c: (1/2, 1, 0); a=b>c: (1, 0, 1/2);
// a=b=c: (1/2, 0, 0), an axis counting only if its virtual index lies in the
// a-slab and its (y, z) in the VJP's slab block.  The VJP (lnoccsdt_energy_vjp,
// lno_ccsd_t_vjp.c:9-566) needs in addition the projected cubes
//   A = sum_t wt_t M_t(w),  B = sum_t wt_t M_t^T(q),
//   M_t(w)_f[k] = sum_l mat[l,k] w_f[l],  M_t^T(q)_f[k] = sum_l mat[k,l] q_f[l],
// and mat_bar = et_bar C with C = sum_t wt_t G_t.
//
// One CTA per job streams the cubes through shared memory twice, with no
// read-modify-write of global memory:
//  * pass 1, plane by plane (fixed p; axes 1 and 2 run inside a plane):
//      C += W_p Q_p^T (axis 1) + W_p^T Q_p (axis 2),
//      A12_p = mat^T W_p (axis 1) + W_p mat (axis 2),
//      B12_p = mat Q_p (axis 1) + Q_p mat^T (axis 2);
//  * pass 2, by chunks of 64 consecutive positions of every plane (axis 0):
//      C += W_c Q_c^T,  A0_c = mat^T W_c,  B0_c = mat Q_c,
// where W_p is plane p as an (o x o) matrix and W_c the (o x 64) chunk.
// A12, B12 go to slots 2 and 3, A0, B0 to slots 4 and 5; the backward orbit
// epilogue adds the two parts as it stages them.  E = sum mat o C (no pass
// over A).  Weights: wt_1 and wt_2 are never two different nonzero values
// (wt_1 != 0 needs a > b >= c, wt_2 = 1/2 needs a = b > c), so pass 1 runs
// with unscaled operands and scales its outputs by w12 = max(wt_1, wt_2);
// all weights are powers of two, so the rescalings are exact.
//
// Staging: each thread loads its share of the next plane or chunk into
// registers while the current one is contracted, then converts it to float64
// in a zero-padded shared-memory tile (row stride 4 doubles past the width:
// the A- and B-fragment reads of m8n8k4 are then free of bank conflicts).
// CT, QRT: the cubes' type and layout (double and plain (p,q,r) on the float64
// path; float and qr-tiled, (p,q,r) at p o^2 + (q/8) 8o + (r/8) 64 + (q%8) 8 +
// r%8, on the mixed path).  In both layouts a chunk of 64 consecutive plane
// positions is a set of (q, r) pairs, which is all pass 2 needs.
#include <cuda_runtime.h>
#include "ct_common.cuh"
#include "ct_internal.h"

namespace ctb {

// axis t carries x; (y, z) are the other two values, y >= z: (b, c), (a, c), (a, b)
__device__ __forceinline__ void lno_weights(int a, int b, int c, const EpiArgs &e, double (&wt)[3]) {
    const bool dis = a > b && b > c, abb = a > b && b == c, aab = a == b && b > c;
    const int a0 = e.lno_a0, a1 = e.lno_a1;
    const bool in0 = a >= a0 && a < a1, in1 = b >= a0 && b < a1, in2 = c >= a0 && c < a1;
    auto yz = [&](int y, int z) { return y >= e.lno_b0 && y < e.lno_b1 && z >= e.lno_c0 && z < e.lno_c1; };
    wt[0] = (in0 && yz(b, c)) ? ((dis || aab) ? 1.0 : 0.5) : 0.0;
    wt[1] = (in1 && yz(a, c) && (dis || abb)) ? 1.0 : 0.0;
    wt[2] = (in2 && yz(a, b)) ? (dis ? 1.0 : (aab ? 0.5 : 0.0)) : 0.0;
}

namespace lnoproj {

// NT 8-wide tiles along nocc (o <= 8 NT): R = 8 NT rows, 2 NT warps.  Warp w
// owns row tile w/2 and column half w%2 of every (R x R) output (CG tiles) and
// of every (R x 64) chunk output (4 tiles).
template <int NT> struct Cfg {
    static constexpr int R = 8 * NT;
    static constexpr int S = R + 4;              // row stride: mat and a staged plane
    static constexpr int SC = 64 + 4;            // row stride: a staged chunk
    static constexpr int NW = 2 * NT, NTHR = 32 * NW;
    static constexpr int CG = NT / 2;
    static constexpr int BUF = R * SC;           // doubles per staged cube (>= R * S)
    static constexpr int PP = R * R / NTHR;      // plane elements per thread (= NT)
    static constexpr int PC = R * 64 / NTHR;     // chunk elements per thread (= 8)
    static constexpr size_t smem = sizeof(double) * (size_t)(R * S + 2 * BUF);
};

// position of (q, r) in a plane of the cube
template <bool QRT> __device__ __forceinline__ long long plane_pos(int q, int r, int o) {
    return QRT ? (long long)(q >> 3) * 8 * o + (r >> 3) * 64 + (q & 7) * 8 + (r & 7) : (long long)q * o + r;
}

// Loads stage s into registers: plane s (s < np) or chunk s - np.  Element k of
// a thread is tile position i = tid + k NTHR: (q, r) = (i / R, i % R) of the
// plane, or (l, j) = (i / 64, i % 64) of the chunk (row l, plane position
// 64 ch + j).  Positions outside the cube give 0.
template <int NT, typename CT, bool QRT>
__device__ __forceinline__ void load_stage(int s, int np, int o, const CT *W, const CT *Q, CT (&rw)[8],
                                           CT (&rq)[8], bool active) {
    using C = Cfg<NT>;
    const int tid = threadIdx.x;
    const long long oo = (long long)o * o;
#pragma unroll
    for (int k = 0; k < 8; ++k) { rw[k] = CT(0); rq[k] = CT(0); }
    if (!active) return;
    if (s < np) {
        const long long pb = (long long)s * oo;
#pragma unroll
        for (int k = 0; k < C::PP; ++k) {
            const int i = tid + k * C::NTHR, q = i / C::R, r = i - q * C::R;
            if (q < o && r < o) {
                const long long pos = pb + plane_pos<QRT>(q, r, o);
                rw[k] = __ldg(W + pos);
                rq[k] = __ldg(Q + pos);
            }
        }
    } else {
        const long long cb = 64LL * (s - np);
#pragma unroll
        for (int k = 0; k < C::PC; ++k) {
            const int i = tid + k * C::NTHR, l = i >> 6, j = i & 63;
            if (l < o && cb + j < oo) {
                const long long pos = l * oo + cb + j;
                rw[k] = __ldg(W + pos);
                rq[k] = __ldg(Q + pos);
            }
        }
    }
}

// the registers of stage s into the float64 tiles Ws, Qs (every tile position
// written, zeros included)
template <int NT, typename CT>
__device__ __forceinline__ void store_stage(int s, int np, double *Ws, double *Qs, const CT (&rw)[8],
                                            const CT (&rq)[8]) {
    using C = Cfg<NT>;
    const int tid = threadIdx.x;
    if (s < np) {
#pragma unroll
        for (int k = 0; k < C::PP; ++k) {
            const int i = tid + k * C::NTHR, q = i / C::R, r = i - q * C::R;
            Ws[q * C::S + r] = (double)rw[k];
            Qs[q * C::S + r] = (double)rq[k];
        }
    } else {
#pragma unroll
        for (int k = 0; k < C::PC; ++k) {
            const int i = tid + k * C::NTHR, l = i >> 6, j = i & 63;
            Ws[l * C::SC + j] = (double)rw[k];
            Qs[l * C::SC + j] = (double)rq[k];
        }
    }
}

// One job per CTA.  VJP: the energy, the A12/B12 (slots 2, 3) and A0/B0
// (slots 4, 5) cubes and the job's mat_bar partial eb C; otherwise the energy.
template <int NT, typename CT, bool QRT, bool VJP>
__global__ void __launch_bounds__(Cfg<NT>::NTHR, NT <= 4 ? 2 : 1) proj_kernel(const WaveView w, const EpiArgs e,
                                                                             CT *scratch) {
    using C = Cfg<NT>;
    constexpr int R = C::R, S = C::S, SC = C::SC, CG = C::CG;
    extern __shared__ __align__(16) double lsm[];
    double *Ms = lsm, *Ws = lsm + R * S, *Qs = Ws + C::BUF;
    __shared__ double wred[C::NW];
    const int o = e.o, tid = threadIdx.x, jl = blockIdx.x;
    const int lane = tid & 31, warp = tid >> 5, g = lane >> 2, c = lane & 3;
    const long long oo = (long long)o * o, o3 = oo * o;
    int a, b, cz;
    unpack_job(w.jobs[jl], a, b, cz);
    double wt[3];
    lno_weights(a, b, cz, e, wt);
    const bool d1 = wt[1] != 0.0, d2 = wt[2] != 0.0, p1 = d1 || d2, p2 = wt[0] != 0.0;
    const double w12 = fmax(wt[1], wt[2]);
    CT *Sj = scratch + (long long)jl * kSlots * o3;
    const CT *Wg = Sj, *Qg = Sj + o3;
    CT *A12 = Sj + 2 * o3, *B12 = Sj + 3 * o3, *A0 = Sj + 4 * o3, *B0 = Sj + 5 * o3;

    for (int i = tid; i < R * S; i += C::NTHR) {
        const int l = i / S, k = i - l * S;
        Ms[i] = (l < o && k < o) ? e.lno_mat[l * o + k] : 0.0;
    }
    const int mt = warp >> 1, half = warp & 1, row = mt * 8 + g;
    double aC[CG][2], aA[4][2], aB[4][2];
#pragma unroll
    for (int j = 0; j < CG; ++j) aC[j][0] = aC[j][1] = 0.0;
    auto rescale = [&](double f) {
#pragma unroll
        for (int j = 0; j < CG; ++j) { aC[j][0] *= f; aC[j][1] *= f; }
    };
    // stages: the o planes (pass 1), then the chunks (pass 2); the VJP runs
    // both always (its outputs are written even where a weight is zero)
    const int np = (VJP || p1) ? o : 0;
    const int nc = (VJP || p2) ? (int)((oo + 63) / 64) : 0;
    const int ns = np + nc;
    CT rw[8], rq[8];
    if (ns > 0) load_stage<NT, CT, QRT>(0, np, o, Wg, Qg, rw, rq, np > 0 ? p1 : p2);
    for (int s = 0; s < ns; ++s) {
        const bool plane = s < np, act = plane ? p1 : p2;
        __syncthreads();   // the previous stage's tiles are no longer read
        if (act) store_stage<NT, CT>(s, np, Ws, Qs, rw, rq);
        __syncthreads();
        if (s + 1 < ns) load_stage<NT, CT, QRT>(s + 1, np, o, Wg, Qg, rw, rq, (s + 1 < np) ? p1 : p2);
        if (plane) {
            // ---- pass 1, plane p = s: axes 1 and 2
#pragma unroll
            for (int j = 0; j < 4; ++j) aA[j][0] = aA[j][1] = aB[j][0] = aB[j][1] = 0.0;
            if (act) {
#pragma unroll 2
                for (int kk = 0; kk < R; kk += 4) {
                    const int kr = kk + c;
                    if (d1) {
                        const double aw = Ws[row * S + kr];            // W_p[row][kr]
#pragma unroll
                        for (int j = 0; j < CG; ++j)                   // C += W_p Q_p^T
                            dmma(aC[j], aw, Qs[((half * CG + j) * 8 + g) * S + kr]);
                        if (VJP) {
                            const double am = Ms[kr * S + row], amr = Ms[row * S + kr];
#pragma unroll
                            for (int j = 0; j < CG; ++j) {
                                const int col = (half * CG + j) * 8 + g;
                                dmma(aA[j], am, Ws[kr * S + col]);     // A += mat^T W_p
                                dmma(aB[j], amr, Qs[kr * S + col]);    // B += mat Q_p
                            }
                        }
                    }
                    if (d2) {
                        const double awt = Ws[kr * S + row];           // W_p[kr][row]
#pragma unroll
                        for (int j = 0; j < CG; ++j)                   // C += W_p^T Q_p
                            dmma(aC[j], awt, Qs[kr * S + (half * CG + j) * 8 + g]);
                        if (VJP) {
                            const double aw = Ws[row * S + kr], aq = Qs[row * S + kr];
#pragma unroll
                            for (int j = 0; j < CG; ++j) {
                                const int col = (half * CG + j) * 8 + g;
                                dmma(aA[j], aw, Ms[kr * S + col]);     // A += W_p mat
                                dmma(aB[j], aq, Ms[col * S + kr]);     // B += Q_p mat^T
                            }
                        }
                    }
                }
            }
            if (VJP) {
                const long long pb = (long long)s * oo;
#pragma unroll
                for (int j = 0; j < CG; ++j)
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const int r = (half * CG + j) * 8 + 2 * c + h;
                        if (row < o && r < o) {
                            const long long pos = pb + plane_pos<QRT>(row, r, o);
                            A12[pos] = CT(w12 * aA[j][h]);
                            B12[pos] = CT(w12 * aB[j][h]);
                        }
                    }
            }
        } else {
            // ---- pass 2, chunk ch = s - np: axis 0
            if (s == np && np > 0) rescale(p2 ? w12 / wt[0] : w12);
#pragma unroll
            for (int j = 0; j < 4; ++j) aA[j][0] = aA[j][1] = aB[j][0] = aB[j][1] = 0.0;
            if (act) {
#pragma unroll 4
                for (int jj = 0; jj < 64; jj += 4) {                   // C += W_c Q_c^T
                    const double aw = Ws[row * SC + jj + c];
#pragma unroll
                    for (int j = 0; j < CG; ++j) dmma(aC[j], aw, Qs[((half * CG + j) * 8 + g) * SC + jj + c]);
                }
                if (VJP) {
#pragma unroll 2
                    for (int kk = 0; kk < R; kk += 4) {
                        const int kr = kk + c;
                        const double am = Ms[kr * S + row], amr = Ms[row * S + kr];
#pragma unroll
                        for (int j = 0; j < 4; ++j) {
                            const int col = (half * 4 + j) * 8 + g;
                            dmma(aA[j], am, Ws[kr * SC + col]);        // A0 = mat^T W_c
                            dmma(aB[j], amr, Qs[kr * SC + col]);       // B0 = mat Q_c
                        }
                    }
                }
            }
            if (VJP) {
                const long long cb = 64LL * (s - np);
#pragma unroll
                for (int j = 0; j < 4; ++j)
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const long long P = cb + (half * 4 + j) * 8 + 2 * c + h;
                        if (row < o && P < oo) {
                            const long long pos = row * oo + P;
                            A0[pos] = CT(wt[0] * aA[j][h]);
                            B0[pos] = CT(wt[0] * aB[j][h]);
                        }
                    }
            }
        }
    }
    if (nc > 0) {
        if (p2) rescale(wt[0]);
    } else {
        rescale(w12);
    }
    // E = sum mat o C over this warp's C tiles; mat_bar partial eb C
    double es = 0.0;
    double *part = VJP ? e.lno_mat_bar_part + (long long)jl * oo : nullptr;
#pragma unroll
    for (int j = 0; j < CG; ++j)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int k = (half * CG + j) * 8 + 2 * c + h;
            if (row < o && k < o) {
                es = fma(Ms[row * S + k], aC[j][h], es);
                if (VJP) part[row * o + k] = e.et_bar * aC[j][h];
            }
        }
#pragma unroll
    for (int m = 16; m >= 1; m >>= 1) es += __shfl_xor_sync(0xffffffffu, es, m);
    if (lane == 0) wred[warp] = es;
    __syncthreads();
    if (tid == 0) {
        double tot = 0.0;
        for (int i = 0; i < C::NW; ++i) tot += wred[i];
        const long long amaj = (long long)a * (a + 1) * (a + 2) / 6 + (long long)b * (b + 1) / 2 + cz;
        e.job_e[amaj] = tot;
    }
}

template <int NT, typename CT, bool QRT, bool VJP>
static cudaError_t launch_nt(const WaveView &w, const EpiArgs &e, CT *scratch, cudaStream_t st) {
    using C = Cfg<NT>;
    cudaError_t ce = smem_optin(reinterpret_cast<const void *>(proj_kernel<NT, CT, QRT, VJP>), (int)C::smem);
    if (ce != cudaSuccess) return ce;
    proj_kernel<NT, CT, QRT, VJP><<<w.n_jobs, C::NTHR, C::smem, st>>>(w, e, scratch);
    return cudaGetLastError();
}

// nocc <= 32: the 4-tile build (256 threads, 44 KB); else the 8-tile one (512 threads, 104 KB)
template <typename CT, bool QRT, bool VJP>
static cudaError_t launch(const WaveView &w, const EpiArgs &e, CT *scratch, cudaStream_t st) {
    if (w.n_jobs <= 0) return cudaSuccess;
    if (!e.lno_mat || e.o < 1 || e.o > 64 || (VJP && !e.lno_mat_bar_part) || (QRT && e.o % 8 != 0))
        return cudaErrorInvalidValue;
    return e.o <= 32 ? launch_nt<4, CT, QRT, VJP>(w, e, scratch, st) : launch_nt<8, CT, QRT, VJP>(w, e, scratch, st);
}

__global__ void mat_bar_kernel(const double *part, int n_jobs, int oo, double *mat_bar) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= oo) return;
    double s = 0.0;
    for (int j = 0; j < n_jobs; ++j) s += part[(long long)j * oo + i];
    mat_bar[i] += s;
}

}  // namespace lnoproj

cudaError_t f64_lno_contract(const WaveView &w, const EpiArgs &e, const double *scratch, cudaStream_t st) {
    return lnoproj::launch<double, false, false>(w, e, const_cast<double *>(scratch), st);
}

cudaError_t f32_lno_contract(const WaveView &w, const EpiArgs &e, const float *scratch, cudaStream_t st) {
    return lnoproj::launch<float, true, false>(w, e, const_cast<float *>(scratch), st);
}

cudaError_t f64_lno_vjp_project(const WaveView &w, const EpiArgs &e, double *scratch, cudaStream_t st) {
    return lnoproj::launch<double, false, true>(w, e, scratch, st);
}

cudaError_t f32_lno_vjp_project(const WaveView &w, const EpiArgs &e, float *scratch, cudaStream_t st) {
    return lnoproj::launch<float, true, true>(w, e, scratch, st);
}

// mat_bar += the wave's per-job partials, summed in job order
cudaError_t f64_lno_mat_bar(const WaveView &w, const EpiArgs &e, double *mat_bar, cudaStream_t st) {
    if (w.n_jobs <= 0) return cudaSuccess;
    const int oo = e.o * e.o;
    lnoproj::mat_bar_kernel<<<(oo + 255) / 256, 256, 0, st>>>(e.lno_mat_bar_part, w.n_jobs, oo, mat_bar);
    return cudaGetLastError();
}

}  // namespace ctb
