// Mixed-precision path: every contraction of the (T) energy + VJP runs on the
// 5th-generation tensor cores (tcgen05, TMEM accumulators, TMA-fed shared
// memory), with float32 accumulation; the orbit epilogue, the denominators,
// the per-job energies and the final reduction stay float64 (ct_fp64.cu
// kernels instantiated on float scratch).
//
// GEMM kinds of one wave (same arithmetic as the float64 path):
//   F1  G_t[p,qr]  = sum_f vvop[x,y,p,o+f] t2T[z,f,qr]      D[qr,(t,p)]   terms grouped by z
//   F2  G_t[pq,r] -= sum_l vooo[x,pq,l] t2T[z,y,l,r]         D[pq,(t,r)]   terms grouped by x
//   VB  vvop_bar[x,y,p,o+f] += sum_qr t2T[z,f,qr] Wbar_t[p,qr]  D[f,(t,p)] grouped by z
//   TB  t2T_bar[z,f,qr] += sum_t sum_p vvop[x,y,p,o+f] Wbar_t[p,qr]  D[f,qr], K over (t,p)
//   OB1 vooo_bar[x,pq,l] -= sum_t sum_r Wbar_t[pq,r] t2T[z,y,l,r]    D[pq,l], K over (t,r)
//   OB2 t2T_bar[z,y,l,r] -= sum_pq vooo[x,pq,l] Wbar_t[pq,r]          D[l,(t,r)]
// (reference: get_wv ccsd_t.c:121-152; get_vvov_bar / get_vooo_bar /
//  get_t2T_bar ccsd_t_vjp.c:139-231)
//
// Kernel: one persistent CTA per SM; warp 0 issues TMA loads into a ring of
// shared-memory stages, warp 1 (one thread) issues tcgen05.mma into one of two
// TMEM accumulators, warps 2-5 drain the other accumulator (tcgen05.ld) and
// write results, so epilogues overlap the next tile's main loop.  Every
// mbarrier wait is bounded; a timeout sets an error flag that the host turns
// into CT_ERR_TIMEOUT.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cstdio>
#include <cstdlib>
#include <vector>
#include "ct_common.cuh"
#include "ct_internal.h"
#include "ct_mixed.h"
#include "tc_ptx.cuh"

namespace ctb {

enum TcKind { TK_F1 = 0, TK_F2, TK_VB, TK_TB, TK_OB1, TK_OB2, TK_COUNT };

constexpr int kMaxStages = 4;
constexpr int kTmemCols = 512;   // two 256-column accumulators
constexpr int kThreads = 192;    // 6 warps

struct TcParams {
    CUtensorMap mapA;
    CUtensorMap mapB;
    int o, v, n, vp, o32;
    int nwork, m_tiles, n_tiles;
    int stages, stage_bytes, a_bytes;
    const int *jobs;
    const int *groups;   // (key, e_begin, e_end) triples
    const int *entries;  // term ids jl*6+sigma
    float *G;            // float scratch (7 slots per job)
    double *out;         // gradient output base for VB/TB/OB1/OB2
    int *err;
};

struct Term {
    int x, y, z, slot;
};

__device__ __forceinline__ Term term_of(const TcParams &P, int eid) {
    const int jl = eid / 6, sg = eid - 6 * (eid / 6);
    int a, b, c;
    unpack_job(P.jobs[jl], a, b, c);
    Term t;
    term_xyz(sg, a, b, c, t.x, t.y, t.z);
    t.slot = jl * kSlots + sg;
    return t;
}

struct Work {
    int g, mt, nt;
    int key, e0, nterms;
    int nk;     // k-iterations
    int N;      // MMA N
};

template <int KIND>
__device__ __forceinline__ void decode(const TcParams &P, int w, Work &W) {
    if (KIND == TK_TB) {
        const int per = P.m_tiles * P.n_tiles;
        W.g = w / per;
        const int r = w - W.g * per;
        W.mt = r / P.n_tiles;
        W.nt = r - W.mt * P.n_tiles;
    } else if (KIND == TK_OB2) {
        W.g = w; W.mt = 0; W.nt = 0;
    } else {
        W.g = w / P.m_tiles;
        W.mt = w - W.g * P.m_tiles;
        W.nt = 0;
    }
    W.key = P.groups[3 * W.g];
    W.e0 = P.groups[3 * W.g + 1];
    W.nterms = P.groups[3 * W.g + 2] - W.e0;
    const int o = P.o, o2 = o * o;
    switch (KIND) {
    case TK_F1: W.nk = (P.v + 31) / 32; W.N = ((W.nterms * o + 15) / 16) * 16; break;
    case TK_VB: W.nk = (o2 + 31) / 32;  W.N = ((W.nterms * o + 15) / 16) * 16; break;
    case TK_TB: {
        W.nk = W.nterms;
        const int rem = o2 - W.nt * 256;
        W.N = rem >= 256 ? 256 : ((rem + 31) / 32) * 32;
        break;
    }
    case TK_F2: W.nk = (o + 31) / 32; W.N = W.nterms * P.o32; break;
    case TK_OB1: W.nk = W.nterms * ((o + 31) / 32); W.N = ((o + 15) / 16) * 16; break;
    default: W.nk = (o2 + 31) / 32; W.N = W.nterms * P.o32; break;
    }
}

// Issues the TMA loads of k-iteration kit into stage buffers sA/sB; returns bytes.
template <int KIND>
__device__ __forceinline__ uint32_t issue_loads(const TcParams &P, const Work &W, int kit, uint32_t sA, uint32_t sB,
                                                uint32_t bar) {
    const int o = P.o;
    const CUtensorMap *mA = &P.mapA, *mB = &P.mapB;
    uint32_t bytes = 0;
    switch (KIND) {
    case TK_F1: {
        bytes = 16384u + (uint32_t)W.nterms * o * 128u;
        tc::mbar_expect_tx(bar, bytes);
        const int z = W.key;
        for (int c = 0; c < 4; ++c) tc::tma_load_3d(sA + c * 4096, mA, bar, W.mt * 128 + 32 * c, 32 * kit, z);
        for (int t = 0; t < W.nterms; ++t) {
            const Term T = term_of(P, P.entries[W.e0 + t]);
            tc::tma_load_3d(sB + t * o * 128, mB, bar, 32 * kit, 0, T.x * P.v + T.y);
        }
        break;
    }
    case TK_VB: {
        bytes = 16384u + (uint32_t)W.nterms * o * 128u;
        tc::mbar_expect_tx(bar, bytes);
        tc::tma_load_3d(sA, mA, bar, 32 * kit, W.mt * 128, W.key);
        for (int t = 0; t < W.nterms; ++t) {
            const Term T = term_of(P, P.entries[W.e0 + t]);
            tc::tma_load_3d(sB + t * o * 128, mB, bar, 32 * kit, 0, T.slot);
        }
        break;
    }
    case TK_TB: {
        const int nch = W.N / 32;
        bytes = (uint32_t)(4 + nch) * o * 128u;
        tc::mbar_expect_tx(bar, bytes);
        const Term T = term_of(P, P.entries[W.e0 + kit]);
        for (int c = 0; c < 4; ++c) tc::tma_load_3d(sA + c * o * 128, mA, bar, W.mt * 128 + 32 * c, 0, T.x * P.v + T.y);
        for (int c = 0; c < nch; ++c) tc::tma_load_3d(sB + c * o * 128, mB, bar, W.nt * 256 + 32 * c, 0, T.slot);
        break;
    }
    case TK_F2: {
        const int nch = P.o32 / 32;
        bytes = 16384u + (uint32_t)W.nterms * nch * 4096u;
        tc::mbar_expect_tx(bar, bytes);
        tc::tma_load_3d(sA, mA, bar, 32 * kit, W.mt * 128, W.key);
        for (int t = 0; t < W.nterms; ++t) {
            const Term T = term_of(P, P.entries[W.e0 + t]);
            for (int c = 0; c < nch; ++c)
                tc::tma_load_3d(sB + (t * nch + c) * 4096, mB, bar, 32 * c, 32 * kit, T.z * P.v + T.y);
        }
        break;
    }
    case TK_OB1: {
        const int kper = (o + 31) / 32;
        const int t = kit / kper, kr = kit - t * kper;
        bytes = 16384u + (uint32_t)o * 128u;
        tc::mbar_expect_tx(bar, bytes);
        const Term T = term_of(P, P.entries[W.e0 + t]);
        tc::tma_load_3d(sA, mA, bar, 32 * kr, W.mt * 128, T.slot);
        tc::tma_load_3d(sB, mB, bar, 32 * kr, 0, T.z * P.v + T.y);
        break;
    }
    default: {  // TK_OB2
        const int nch = P.o32 / 32;
        bytes = (uint32_t)nch * 4096u + (uint32_t)W.nterms * nch * 4096u;
        tc::mbar_expect_tx(bar, bytes);
        for (int c = 0; c < nch; ++c) tc::tma_load_3d(sA + c * 4096, mA, bar, 32 * c, 32 * kit, W.key);
        for (int t = 0; t < W.nterms; ++t) {
            const Term T = term_of(P, P.entries[W.e0 + t]);
            for (int c = 0; c < nch; ++c)
                tc::tma_load_3d(sB + (t * nch + c) * 4096, mB, bar, 32 * c, 32 * kit, T.slot);
        }
        break;
    }
    }
    return bytes;
}

// MMAs of one stage (tf32: K = 8 per instruction)
template <int KIND>
__device__ __forceinline__ void issue_mmas(const TcParams &P, const Work &W, uint32_t sA, uint32_t sB, uint32_t tacc,
                                           bool first) {
    const int o = P.o;
    int ksteps;
    bool amn, bmn;
    uint32_t a_lbo, b_lbo;
    switch (KIND) {
    case TK_F1: ksteps = 4; amn = true; bmn = false; a_lbo = 4096; b_lbo = 16; break;
    case TK_VB: ksteps = 4; amn = false; bmn = false; a_lbo = 16; b_lbo = 16; break;
    case TK_TB: ksteps = o / 8; amn = true; bmn = true; a_lbo = o * 128; b_lbo = o * 128; break;
    case TK_F2: ksteps = 4; amn = false; bmn = true; a_lbo = 16; b_lbo = 4096; break;
    case TK_OB1: ksteps = 4; amn = false; bmn = false; a_lbo = 16; b_lbo = 16; break;
    default: ksteps = 4; amn = true; bmn = true; a_lbo = 4096; b_lbo = 4096; break;
    }
    const uint32_t id = tc::idesc(2, 128, W.N, amn, bmn);
    for (int kk = 0; kk < ksteps; ++kk) {
        const uint32_t ao = amn ? kk * 1024u : kk * 32u;
        const uint32_t bo = bmn ? kk * 1024u : kk * 32u;
        // tf32 MN-major operands use the 32-B-atom swizzle (4-row atoms)
        const uint64_t da = amn ? tc::sdesc(sA + ao, a_lbo, 512, tc::kSw128Base32) : tc::sdesc(sA + ao, a_lbo, 1024);
        const uint64_t db = bmn ? tc::sdesc(sB + bo, b_lbo, 512, tc::kSw128Base32) : tc::sdesc(sB + bo, b_lbo, 1024);
        tc::mma_tf32(tacc, da, db, id, (first && kk == 0) ? 0u : 1u);
    }
}

// Epilogue of one work item: this warp holds rows 32*q .. 32*q+31 of D.
// Term descriptors of the work item are held one per lane and broadcast with
// shuffles; outputs whose rows are contiguous in memory (F2, OB1, OB2) or whose
// rows are long contiguous runs (TB) are transposed through the warp's shared
// buffer ebuf[32][65] so every read-modify-write is coalesced.
constexpr int kEbufLd = 65;
// per-warp transpose buffer (floats): t2-bar tiles go 16 columns at a time
__host__ __device__ constexpr int ebuf_floats(int kind) { return kind == TK_TB ? 32 * 17 : 32 * kEbufLd; }

template <int KIND>
__device__ __forceinline__ void epilogue(const TcParams &P, const Work &W, uint32_t tacc, int q, int lane,
                                         float *ebuf) {
    const int o = P.o, v = P.v, n = P.n;
    const long long o2 = (long long)o * o, o3 = o2 * o;
    const int row = 32 * q + lane;
    const uint32_t tbase = tacc + ((uint32_t)(32 * q) << 16);
    // this lane's term descriptor (lane t <-> term t of the work item)
    Term mine{0, 0, 0, 0};
    if (KIND != TK_TB && KIND != TK_OB1 && lane < W.nterms) mine = term_of(P, P.entries[W.e0 + lane]);
    auto bcast = [&](int t) {
        Term r;
        r.x = __shfl_sync(0xffffffffu, mine.x, t);
        r.y = __shfl_sync(0xffffffffu, mine.y, t);
        r.z = __shfl_sync(0xffffffffu, mine.z, t);
        r.slot = __shfl_sync(0xffffffffu, mine.slot, t);
        return r;
    };
    float vals[16];
    if (KIND == TK_F1 || KIND == TK_VB) {
        for (int c0 = 0; c0 < W.N; c0 += 16) {
            tc::tmem_ld16(tbase + c0, vals);
            const int t_lo = c0 / o;
            const int t_hi = (c0 + 15) / o;
            const Term T0 = bcast(t_lo < 32 ? t_lo : 31), T1 = bcast(t_hi < 32 ? t_hi : 31);
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const int col = c0 + j, t = col / o, p = col - t * o;
                if (t >= W.nterms) continue;
                const Term T = (t == t_lo) ? T0 : T1;
                if (KIND == TK_F1) {
                    const int qr = W.mt * 128 + row;
                    if (qr < o2) P.G[(long long)T.slot * o3 + (long long)p * o2 + qr] = vals[j];
                } else {
                    const int f = W.mt * 128 + row;
                    if (f < v) atomicAdd(P.out + (((long long)T.x * v + T.y) * o + p) * n + o + f, (double)vals[j]);
                }
            }
        }
    } else if (KIND == TK_TB) {
        // 16 columns per pass; half-warps take alternate rows -> 128-byte runs
        const int f0 = W.mt * 128 + 32 * q;
        for (int c0 = 0; c0 < W.N; c0 += 16) {
            tc::tmem_ld16(tbase + c0, vals);
#pragma unroll
            for (int j = 0; j < 16; ++j) ebuf[lane * 17 + j] = vals[j];
            __syncwarp();
            const int qr = W.nt * 256 + c0 + (lane & 15);
            double *base = P.out + (long long)W.key * v * o2 + qr;
            double cur[16];
#pragma unroll
            for (int rr = 0; rr < 16; ++rr) {  // all loads first: independent, in flight together
                const int f = f0 + 2 * rr + (lane >> 4);
                cur[rr] = (f < v && qr < o2) ? base[(long long)f * o2] : 0.0;
            }
#pragma unroll
            for (int rr = 0; rr < 16; ++rr) {
                const int r = 2 * rr + (lane >> 4);
                const int f = f0 + r;
                if (f < v && qr < o2) base[(long long)f * o2] = cur[rr] + (double)ebuf[r * 17 + (lane & 15)];
            }
            __syncwarp();
        }
    } else {
        // F2 / OB1 / OB2: per term, a (rows x o) block that is contiguous in memory
        const int nt = (KIND == TK_OB1) ? 1 : W.nterms;
        const int cstride = (KIND == TK_OB1) ? 0 : P.o32;
        for (int t = 0; t < nt; ++t) {
            for (int c0 = 0; c0 < o; c0 += 16) {
                tc::tmem_ld16(tbase + t * cstride + c0, vals);
#pragma unroll
                for (int j = 0; j < 16; ++j) ebuf[lane * kEbufLd + c0 + j] = vals[j];
            }
            __syncwarp();
            if (KIND == TK_F2) {
                const Term T = bcast(t);
                const int pq0 = W.mt * 128 + 32 * q;
                float *dst = P.G + (long long)T.slot * o3 + (long long)pq0 * o;
                const int lim = (int)min((long long)32, o2 - pq0) * o;
                for (int i0 = 0; i0 < lim; i0 += 16 * 32) {
                    float cur[16];
#pragma unroll
                    for (int k = 0; k < 16; ++k) {
                        const int i = i0 + k * 32 + lane;
                        cur[k] = i < lim ? dst[i] : 0.f;
                    }
#pragma unroll
                    for (int k = 0; k < 16; ++k) {
                        const int i = i0 + k * 32 + lane;
                        if (i < lim) dst[i] = cur[k] - ebuf[(i / o) * kEbufLd + i % o];
                    }
                }
            } else if (KIND == TK_OB1) {
                const int pq0 = W.mt * 128 + 32 * q;
                double *dst = P.out + (long long)W.key * o3 + (long long)pq0 * o;
                const int lim = (int)min((long long)32, o2 - pq0) * o;
                for (int i0 = 0; i0 < lim; i0 += 16 * 32) {
                    double cur[16];
#pragma unroll
                    for (int k = 0; k < 16; ++k) {
                        const int i = i0 + k * 32 + lane;
                        cur[k] = i < lim ? dst[i] : 0.0;
                    }
#pragma unroll
                    for (int k = 0; k < 16; ++k) {
                        const int i = i0 + k * 32 + lane;
                        if (i < lim) dst[i] = cur[k] - (double)ebuf[(i / o) * kEbufLd + i % o];
                    }
                }
            } else {  // OB2: rows l < o of t2T_bar[z,y,l,:]
                const Term T = bcast(t);
                const int l0 = 32 * q;
                if (l0 < o) {
                    double *dst = P.out + ((long long)T.z * v + T.y) * o2 + (long long)l0 * o;
                    const int lim = min(32, o - l0) * o;
                    for (int i = lane; i < lim; i += 32) atomicAdd(dst + i, -(double)ebuf[(i / o) * kEbufLd + i % o]);
                }
            }
            __syncwarp();
        }
    }
}

template <int KIND>
__global__ void __launch_bounds__(kThreads, 1) tc_gemm_kernel(const __grid_constant__ TcParams P) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int S = P.stages;
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + (size_t)S * P.stage_bytes);
    // bars: full[0..3], empty[4..7], acc_full[8..9], acc_empty[10..11], drain[12]
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 16);
    float *ebuf_all = reinterpret_cast<float *>(smem + (size_t)S * P.stage_bytes + 256);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t sbase = tc::smem_u32(smem);
    auto bar = [&](int i) { return tc::smem_u32(bars + i); };

    if (threadIdx.x == 0) {
        for (int s = 0; s < kMaxStages; ++s) {
            tc::mbar_init(bar(s), 1);
            tc::mbar_init(bar(4 + s), 1);
        }
        tc::mbar_init(bar(8), 1);
        tc::mbar_init(bar(9), 1);
        tc::mbar_init(bar(10), 4);
        tc::mbar_init(bar(11), 4);
        tc::mbar_init(bar(12), 1);
        tc::fence_mbar_init();
    }
    if (warp == 1) {
        tc::tmem_alloc(tc::smem_u32(tmem_slot), kTmemCols);
        tc::tmem_relinquish();
    }
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tmem = *tmem_slot;
    int *err = P.err;

    if (warp == 0) {
        if (lane == 0) {
            int it = 0;
            bool ok = true;
            for (int w = blockIdx.x; w < P.nwork && ok; w += gridDim.x) {
                Work W;
                decode<KIND>(P, w, W);
                for (int kit = 0; kit < W.nk; ++kit, ++it) {
                    const int s = it % S;
                    if (it >= S && !tc::mbar_wait(bar(4 + s), ((it / S) - 1) & 1, err)) { ok = false; break; }
                    const uint32_t sA = sbase + s * P.stage_bytes;
                    issue_loads<KIND>(P, W, kit, sA, sA + P.a_bytes, bar(s));
                }
            }
            // drain: every issued copy has landed before this CTA can exit
            const int issued = it;
            for (int k = issued - 1; k >= 0 && k >= issued - S; --k)
                tc::mbar_wait(bar(k % S), (k / S) & 1, err);
        }
    } else if (warp == 1) {
        if (lane == 0) {
            int it = 0, wi = 0;
            bool ok = true;
            for (int w = blockIdx.x; w < P.nwork && ok; w += gridDim.x, ++wi) {
                Work W;
                decode<KIND>(P, w, W);
                const int buf = wi & 1, use = wi >> 1;
                if (use > 0 && !tc::mbar_wait(bar(10 + buf), (use - 1) & 1, err)) break;
                tc::fence_after();
                const uint32_t tacc = tmem + (uint32_t)(buf * 256);
                for (int kit = 0; kit < W.nk; ++kit, ++it) {
                    const int s = it % S;
                    if (!tc::mbar_wait(bar(s), (it / S) & 1, err)) { ok = false; break; }
                    tc::fence_after();
                    const uint32_t sA = sbase + s * P.stage_bytes;
                    issue_mmas<KIND>(P, W, sA, sA + P.a_bytes, tacc, kit == 0);
                    tc::mma_commit(bar(4 + s));
                }
                if (!ok) break;
                tc::mma_commit(bar(8 + buf));
            }
            // all issued MMAs complete before TMEM is released
            tc::mma_commit(bar(12));
            tc::mbar_wait(bar(12), 0, err);
        }
    } else {
        const int q = warp & 3;
        int wi = 0;
        for (int w = blockIdx.x; w < P.nwork; w += gridDim.x, ++wi) {
            Work W;
            decode<KIND>(P, w, W);
            const int buf = wi & 1, use = wi >> 1;
            if (!tc::mbar_wait(bar(8 + buf), use & 1, err)) break;
            tc::fence_after();
            epilogue<KIND>(P, W, tmem + (uint32_t)(buf * 256), q, lane, ebuf_all + q * ebuf_floats(KIND));
            tc::fence_before();
            __syncwarp();
            if (lane == 0) tc::mbar_arrive(bar(10 + buf));
        }
    }
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    if (warp == 1) tc::tmem_dealloc(tmem, kTmemCols);
}

// ---------------------------------------------------------------------------
// operand preparation: float64 -> float32 copies in the layouts the tensor maps use
// ---------------------------------------------------------------------------
// round to the nearest tf32 value (the tensor core truncates the low 13
// mantissa bits; pre-rounding makes that truncation exact and the product
// errors unbiased)
__device__ __forceinline__ float to_tf32(double x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"((float)x));
    return __uint_as_float(r);
}

__global__ void cvt_f32_kernel(const double *__restrict__ src, float *__restrict__ dst, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[i] = to_tf32(src[i]);
}

// vvf[xy][p][f] = vvop[xy][p][o+f], f padded to vp (zeros)
__global__ void cvt_vv_kernel(const double *__restrict__ vvop, float *__restrict__ vvf, int o, int v, int vp,
                              long long rows) {
    const int n = o + v;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < rows * vp;
         i += (long long)gridDim.x * blockDim.x) {
        const long long r = i / vp;
        const int f = (int)(i - r * vp);
        vvf[i] = f < v ? to_tf32(vvop[r * n + o + f]) : 0.f;
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    return fn;
}

// 3-D float32 tensor map, 128-byte swizzle; dims innermost first, strides in elements
static bool make_map(CUtensorMap *m, const void *base, long long d0, long long d1, long long d2, long long s1,
                     long long s2, int b0, int b1, bool mn_tf32 = false) {
    EncodeTiledFn enc = encode_fn();
    if (!enc) return false;
    cuuint64_t dims[3] = {(cuuint64_t)d0, (cuuint64_t)d1, (cuuint64_t)d2};
    cuuint64_t strides[2] = {(cuuint64_t)(s1 * 4), (cuuint64_t)(s2 * 4)};
    cuuint32_t box[3] = {(cuuint32_t)b0, (cuuint32_t)b1, 1};
    cuuint32_t es[3] = {1, 1, 1};
    CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<void *>(base), dims, strides, box, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE,
                     mn_tf32 ? CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B : CU_TENSOR_MAP_SWIZZLE_128B,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS && std::getenv("CTB_DEBUG"))
        std::fprintf(stderr, "ctb: cuTensorMapEncodeTiled failed (%d) dims %lld %lld %lld box %d %d\n", (int)r, d0, d1,
                     d2, b0, b1);
    return r == CUDA_SUCCESS;
}

double mixed_extra_bytes_per_job(int o, int mode) {
    (void)o; (void)mode;
    return 0.0;
}

static int g_sms = 0;
static int *g_err = nullptr;

int mixed_prepare(const ct_problem *p, int mode, MixedOperands *mo, cudaStream_t st) {
    if (mode != CT_MODE_TF32) return CT_ERR_MODE;
    const int o = p->nocc, v = p->nvir;
    if (o % 8 != 0 || o > 64) return CT_ERR_SHAPE;
    if (!encode_fn()) return CT_ERR_CUDA;
    if (!g_sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, dev);
    }
    if (!g_err) {
        if (cudaMalloc(&g_err, sizeof(int)) != cudaSuccess) return CT_ERR_NOMEM;
    }
    if (cudaMemsetAsync(g_err, 0, sizeof(int), st) != cudaSuccess) return CT_ERR_CUDA;
    const int vp = (v + 3) / 4 * 4;
    const size_t n_t2 = (size_t)v * v * o * o, n_vv = (size_t)v * v * o * vp, n_vo = (size_t)v * o * o * o;
    const size_t bytes = (n_t2 + n_vv + n_vo) * sizeof(float);
    void *buf = nullptr;
    if (cudaMallocAsync(&buf, bytes, st) != cudaSuccess) return CT_ERR_NOMEM;
    mo->t2 = buf;
    mo->vvop = (float *)buf + n_t2;
    mo->vooo = (float *)buf + n_t2 + n_vv;
    mo->bytes = bytes;
    mo->mode = mode;
    mo->vp = vp;
    const int blocks = g_sms * 8;
    cvt_f32_kernel<<<blocks, 256, 0, st>>>(p->t2T, (float *)mo->t2, (long long)n_t2);
    cvt_vv_kernel<<<blocks, 256, 0, st>>>(p->vvop, (float *)mo->vvop, o, v, vp, (long long)v * v * o);
    cvt_f32_kernel<<<blocks, 256, 0, st>>>(p->vooo, (float *)mo->vooo, (long long)n_vo);
    return cudaGetLastError() == cudaSuccess ? CT_OK : CT_ERR_CUDA;
}

void mixed_release(MixedOperands *mo, cudaStream_t st) {
    if (mo->t2) cudaFreeAsync(mo->t2, st);
    mo->t2 = mo->vvop = mo->vooo = nullptr;
}

template <int KIND>
static int launch_tc(TcParams &P, cudaStream_t st) {
    if (P.nwork <= 0) return CT_OK;
    const int smem = P.stages * P.stage_bytes + 1024 + 256 + 4 * ebuf_floats(KIND) * 4;
    static int configured = 0;
    if (configured < smem) {
        if (cudaFuncSetAttribute(tc_gemm_kernel<KIND>, cudaFuncAttributeMaxDynamicSharedMemorySize, 232448) !=
            cudaSuccess)
            return CT_ERR_CUDA;
        configured = 232448;
    }
    const int grid = P.nwork < g_sms ? P.nwork : g_sms;
    // at least ~116 KB so that a second CTA never shares the SM's tensor memory
    const int smem_req = smem < 120 * 1024 ? 120 * 1024 : smem;
    tc_gemm_kernel<KIND><<<grid, kThreads, smem_req, st>>>(P);
    return cudaGetLastError() == cudaSuccess ? CT_OK : CT_ERR_CUDA;
}

static int stages_for(int stage_bytes, int kind) {
    int s = (232448 - 1024 - 256 - 4 * ebuf_floats(kind) * 4) / stage_bytes;
    return s > kMaxStages ? kMaxStages : (s < 2 ? 2 : s);
}

int mixed_wave(const WaveView &w, const EpiArgs &e, const ct_problem *p, const ct_grads *g, const MixedOperands &mo,
               int mode, bool vjp, void *scratch, cudaStream_t st, int (*prof)(int, int, void *), void *pctx) {
    (void)mode;
    const int o = w.o, v = w.v, n = w.n, vp = mo.vp;
    const long long o2 = (long long)o * o;
    float *G = (float *)scratch;
    const long long slots = (long long)w.n_jobs * kSlots;
    const float *t2 = (const float *)mo.t2, *vv = (const float *)mo.vvop, *vo = (const float *)mo.vooo;
    TcParams base{};
    base.o = o; base.v = v; base.n = n; base.vp = vp; base.o32 = (o + 31) / 32 * 32;
    base.jobs = w.jobs;
    base.G = G;
    base.err = g_err;
    int rc;
    // ---- F1: D[qr,(t,p)], A = t2 (qr,f,z) MN-major, B = vvf (f,p,xy) K-major
    {
        TcParams P = base;
        if (!make_map(&P.mapA, t2, o2, v, v, o2, (long long)v * o2, 32, 32, true)) return CT_ERR_CUDA;
        if (!make_map(&P.mapB, vv, vp, o, (long long)v * v, vp, (long long)o * vp, 32, o)) return CT_ERR_CUDA;
        P.m_tiles = (int)((o2 + 127) / 128);
        P.groups = w.zchunks; P.entries = w.tb_entries;
        P.nwork = w.n_zchunks * P.m_tiles;
        P.a_bytes = 16384; P.stage_bytes = 16384 + 256 * 128; P.stages = stages_for(P.stage_bytes, TK_F1);
        if (prof) prof(PK_MF, 0, pctx);
        if ((rc = launch_tc<TK_F1>(P, st)) != CT_OK) return rc;
        if (prof) prof(PK_MF, 1, pctx);
    }
    // ---- F2: D[pq,(t,r)], A = voof (l,pq,x) K-major, B = t2 (r,l,zy) MN-major
    {
        TcParams P = base;
        if (!make_map(&P.mapA, vo, o, o2, v, o, o2 * o, 32, 128)) return CT_ERR_CUDA;
        if (!make_map(&P.mapB, t2, o, o, (long long)v * v, o, o2, 32, 32, true)) return CT_ERR_CUDA;
        P.m_tiles = (int)((o2 + 127) / 128);
        P.groups = w.xchunks; P.entries = w.x_entries;
        P.nwork = w.n_xchunks * P.m_tiles;
        P.a_bytes = 16384; P.stage_bytes = 16384 + 256 * 128; P.stages = stages_for(P.stage_bytes, TK_F2);
        if (prof) prof(PK_MOO, 0, pctx);
        if ((rc = launch_tc<TK_F2>(P, st)) != CT_OK) return rc;
        if (prof) prof(PK_MOO, 1, pctx);
    }
    { if (prof) prof(PK_EPI, 0, pctx);
      cudaError_t ce = f32_epilogue(w, e, G, st);
      if (prof) prof(PK_EPI, 1, pctx);
      if (ce != cudaSuccess) return CT_ERR_CUDA; }
    if (vjp) {
        { if (prof) prof(PK_VT, 0, pctx);
          cudaError_t ce = f32_vterm(w, e, G, st);
          if (prof) prof(PK_VT, 1, pctx);
          if (ce != cudaSuccess) return CT_ERR_CUDA; }
        // ---- VB: D[f,(t,p)], A = t2 (qr,f,z) K-major box(32,128), B = Wbar (qr,p,slot) K-major
        {
            TcParams P = base;
            if (!make_map(&P.mapA, t2, o2, v, v, o2, (long long)v * o2, 32, 128)) return CT_ERR_CUDA;
            if (!make_map(&P.mapB, G, o2, o, slots, o2, o2 * o, 32, o)) return CT_ERR_CUDA;
            P.m_tiles = (v + 127) / 128;
            P.groups = w.zchunks; P.entries = w.tb_entries;
            P.nwork = w.n_zchunks * P.m_tiles;
            P.out = g->vvop;
            P.a_bytes = 16384; P.stage_bytes = 16384 + 256 * 128; P.stages = stages_for(P.stage_bytes, TK_VB);
            if (prof) prof(PK_MVB, 0, pctx);
            if ((rc = launch_tc<TK_VB>(P, st)) != CT_OK) return rc;
            if (prof) prof(PK_MVB, 1, pctx);
        }
        // ---- TB: D[f,qr], A = vvf (f,p,xy) MN-major, B = Wbar (qr,p,slot) MN-major
        {
            TcParams P = base;
            if (!make_map(&P.mapA, vv, vp, o, (long long)v * v, vp, (long long)o * vp, 32, o, true)) return CT_ERR_CUDA;
            if (!make_map(&P.mapB, G, o2, o, slots, o2, o2 * o, 32, o, true)) return CT_ERR_CUDA;
            P.m_tiles = (v + 127) / 128;
            P.n_tiles = (int)((o2 + 255) / 256);
            P.groups = w.tb_groups; P.entries = w.tb_entries;
            P.nwork = w.n_tb_groups * P.m_tiles * P.n_tiles;
            P.out = g->t2T;
            P.a_bytes = 4 * o * 128; P.stage_bytes = 12 * o * 128; P.stages = stages_for(P.stage_bytes, TK_TB);
            if (prof) prof(PK_MTB, 0, pctx);
            if ((rc = launch_tc<TK_TB>(P, st)) != CT_OK) return rc;
            if (prof) prof(PK_MTB, 1, pctx);
        }
        // ---- OB1: D[pq,l], A = Wbar (r,pq,slot) K-major, B = t2 (r,l,zy) K-major box(32,o)
        {
            TcParams P = base;
            if (!make_map(&P.mapA, G, o, o2, slots, o, o2 * o, 32, 128)) return CT_ERR_CUDA;
            if (!make_map(&P.mapB, t2, o, o, (long long)v * v, o, o2, 32, o)) return CT_ERR_CUDA;
            P.m_tiles = (int)((o2 + 127) / 128);
            P.groups = w.xgroups; P.entries = w.x_entries;
            P.nwork = w.n_xgroups * P.m_tiles;
            P.out = g->vooo;
            P.a_bytes = 16384; P.stage_bytes = 16384 + 64 * 128; P.stages = stages_for(P.stage_bytes, TK_OB1);
            if (prof) prof(PK_MOB1, 0, pctx);
            if ((rc = launch_tc<TK_OB1>(P, st)) != CT_OK) return rc;
            if (prof) prof(PK_MOB1, 1, pctx);
        }
        // ---- OB2: D[l,(t,r)], A = voof (l,pq,x) MN-major box(32,32), B = Wbar (r,pq,slot) MN-major
        {
            TcParams P = base;
            if (!make_map(&P.mapA, vo, o, o2, v, o, o2 * o, 32, 32, true)) return CT_ERR_CUDA;
            if (!make_map(&P.mapB, G, o, o2, slots, o, o2 * o, 32, 32, true)) return CT_ERR_CUDA;
            P.groups = w.xchunks; P.entries = w.x_entries;
            P.nwork = w.n_xchunks;
            P.out = g->t2T;
            P.a_bytes = 16384; P.stage_bytes = 16384 + 256 * 128; P.stages = stages_for(P.stage_bytes, TK_OB2);
            if (prof) prof(PK_MOB2, 0, pctx);
            if ((rc = launch_tc<TK_OB2>(P, st)) != CT_OK) return rc;
            if (prof) prof(PK_MOB2, 1, pctx);
        }
    }
    return CT_OK;
}

int mixed_debug_wave(const WaveView &w, const ct_problem *p, const MixedOperands &mo, int mode, int steps,
                     void *scratch, cudaStream_t st) {
    (void)p; (void)mode;
    const int o = w.o, v = w.v, vp = mo.vp;
    const long long o2 = (long long)o * o;
    const float *t2 = (const float *)mo.t2, *vv = (const float *)mo.vvop, *vo = (const float *)mo.vooo;
    TcParams base{};
    base.o = o; base.v = v; base.n = w.n; base.vp = vp; base.o32 = (o + 31) / 32 * 32;
    base.jobs = w.jobs; base.G = (float *)scratch; base.err = g_err;
    int rc = CT_OK;
    if (steps & 1) {
        TcParams P = base;
        if (!make_map(&P.mapA, t2, o2, v, v, o2, (long long)v * o2, 32, 32, true)) return CT_ERR_CUDA;
        if (!make_map(&P.mapB, vv, vp, o, (long long)v * v, vp, (long long)o * vp, 32, o)) return CT_ERR_CUDA;
        P.m_tiles = (int)((o2 + 127) / 128);
        P.groups = w.zchunks; P.entries = w.tb_entries;
        P.nwork = w.n_zchunks * P.m_tiles;
        P.a_bytes = 16384; P.stage_bytes = 16384 + 256 * 128; P.stages = stages_for(P.stage_bytes, TK_F1);
        if ((rc = launch_tc<TK_F1>(P, st)) != CT_OK) return rc;
    }
    if (steps & 2) {
        TcParams P = base;
        if (!make_map(&P.mapA, vo, o, o2, v, o, o2 * o, 32, 128)) return CT_ERR_CUDA;
        if (!make_map(&P.mapB, t2, o, o, (long long)v * v, o, o2, 32, 32, true)) return CT_ERR_CUDA;
        P.m_tiles = (int)((o2 + 127) / 128);
        P.groups = w.xchunks; P.entries = w.x_entries;
        P.nwork = w.n_xchunks * P.m_tiles;
        P.a_bytes = 16384; P.stage_bytes = 16384 + 256 * 128; P.stages = stages_for(P.stage_bytes, TK_F2);
        if ((rc = launch_tc<TK_F2>(P, st)) != CT_OK) return rc;
    }
    return rc;
}

int mixed_check_error(cudaStream_t st) {
    if (!g_err) return CT_OK;
    int h = 0;
    if (cudaMemcpyAsync(&h, g_err, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess) return CT_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return CT_ERR_CUDA;
    return h ? CT_ERR_TIMEOUT : CT_OK;
}

}  // namespace ctb
