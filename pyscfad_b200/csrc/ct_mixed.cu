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
// Slot layout (mixed path): each o^3 slot of the wave scratch (G, then W-bar,
// and ybar) is qr-tiled: element (p,q,r) lives at p o^2 + (q/8) 8o + (r/8) 64 +
// (q%8) 8 + r%8, so every 8x8x8 block of the orbit epilogue is eight runs of
// 256 contiguous bytes and its stores write whole cache lines.  The qr plane
// of a slot is a permutation of the o^2 pairs; F1 and VB use copies of t2T
// whose (q,r) planes are tiled the same way (F1: [z][tiled qr][f], so that its
// A operand is K-major and comes in 16 KB boxes of 128 rows; VB:
// [z][f][tiled qr], K-major over qr) and TB un-tiles its output columns.  OB1 and OB2 need Wbar_t with r split from (p,q); they read
// it from another slot of the same job: the six W-bar slots of a job are index
// permutations of one cube (Wbar_s[n] = wbar[n o R(INV s)]), and slot
// kRotTerm[t] holds Wbar_t[p,q,r] at (r, tiled (p,q)).  There OB1's A is a
// plain MN-major box (M = tiled pq, K rows = r) and OB2's B a K-major box
// (N rows = r, K = a 128-byte run of tiled pq, the order of OB2's vooo rows).
//
// Precision (template PREC): 0 = TF32 (float32 operands pre-rounded to tf32,
// kind::tf32, K = 8 per MMA); 1 = BF16x3 (each operand split x = hi + lo into
// two bf16 planes, D += hi*hi + hi*lo + lo*hi on kind::f16, K = 16 per MMA),
// float32 accumulation in TMEM either way.  A stage row is always 128 bytes:
// 32 tf32 or 64 bf16 elements of K (or of M/N for MN-major operands).
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

// Paired kinds (TF32 F1 and VB): a work item covers two 128-row M-tiles that
// share the B operand of every stage, accumulated in the two 256-column halves
// of TMEM (single-buffered).  Each stage then brings 2 x 128 rows of A and one
// B tile: 1.5x fewer operand bytes per MMA than one M-tile per item, which is
// what bounds these kinds (L2 -> shared-memory traffic).  P.m_tiles counts
// tile pairs for them.
__host__ __device__ constexpr bool paired(int kind, int prec) { return prec == 0 && (kind == TK_F1 || kind == TK_VB); }

constexpr int kMaxStages = 8;
// mbarrier slots: full[kMaxStages] | empty[kMaxStages] | acc_full[2] | acc_empty[2] | drain
constexpr int kBarEmpty = kMaxStages, kBarAccFull = 2 * kMaxStages, kBarAccEmpty = kBarAccFull + 2,
              kBarDrain = kBarAccEmpty + 2, kBarCount = kBarDrain + 1;
constexpr int kTmemCols = 512;   // two 256-column accumulators

struct TcParams {
    CUtensorMap mapA;
    CUtensorMap mapB;
    CUtensorMap mapA2;   // lo planes (BF16x3)
    CUtensorMap mapB2;
    int o, v, n, vp, ock;   // ock: o rounded up to a 128-byte row of elements
    int nb;                 // o / 8: tiles along q and r of a qr-tiled slot
    unsigned o_magic;      // ceil(2^32 / o): i / o = umulhi(i, o_magic) for small i
    int pairs;              // work items cover two M-tiles (paired kinds)
    int nwork, m_tiles, n_tiles;
    int stages, stage_bytes, a_bytes, b_bytes;   // a_bytes / b_bytes per operand plane
    const int *jobs;
    const int *groups;   // (key, e_begin, e_end) triples
    const int *entries;  // term ids jl*6+sigma
    float *G;            // float scratch (7 slots per job)
    double *out;         // gradient output base for VB/TB/OB1/OB2
    int *err;
};

struct Term {
    int x, y, z, slot, wslot;   // slot: float scratch slot; wslot: W-bar plane index (BF16x3)
};

// kRotTerm[s]: the term whose W-bar slot holds Wbar_s[p,q,r] at position
// (r,p,q).  With Wbar_s[n] = wbar[n o R(INV s)] (n o R)_m = n_R(m), slot s'
// has it when R(INV s') = c^-1 o R(INV s) for the rotation c = (2,0,1).
__host__ __device__ constexpr int kRotTerm(int s) {
    return (0x130524 >> (4 * s)) & 15;   // {4, 2, 5, 0, 3, 1}, 4 bits each (no local array)
}

__device__ __forceinline__ Term term_of(const TcParams &P, int eid) {
    const int jl = eid / 6, sg = eid - 6 * (eid / 6);
    int a, b, c;
    unpack_job(P.jobs[jl], a, b, c);
    Term t;
    term_xyz(sg, a, b, c, t.x, t.y, t.z);
    t.slot = jl * kSlots + sg;
    t.wslot = jl * 6 + sg;
    return t;
}

// W-bar operand index of a term: the float slot (TF32) or the bf16 plane pair (BF16x3)
template <int PREC> __device__ __forceinline__ int wsl(const Term &T) { return PREC ? T.wslot : T.slot; }

// W-bar operand index of the slot that holds term eid's W-bar as (r, tiled pq)
template <int PREC> __device__ __forceinline__ int wsl_rot(int eid) {
    const int jl = eid / 6, s = kRotTerm(eid - 6 * (eid / 6));
    return PREC ? jl * 6 + s : jl * kSlots + s;
}

struct Work {
    int g, mt, nt;
    int key, e0, nterms;
    int nk;     // k-iterations
    int N;      // MMA N
};

template <int KIND, int PREC>
__device__ __forceinline__ void decode(const TcParams &P, int w, Work &W) {
    constexpr int CK = PREC ? 64 : 32;   // elements per 128-byte row
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
    case TK_F1: W.nk = (P.v + CK - 1) / CK; W.N = ((W.nterms * o + 15) / 16) * 16; break;
    case TK_VB: W.nk = (o2 + CK - 1) / CK;  W.N = ((W.nterms * o + 15) / 16) * 16; break;
    case TK_TB: {
        W.nk = W.nterms;
        const int rem = o2 - W.nt * 256;
        W.N = rem >= 256 ? 256 : ((rem + CK - 1) / CK) * CK;
        break;
    }
    case TK_F2: W.nk = (o + CK - 1) / CK; W.N = W.nterms * P.ock; break;
    case TK_OB1: W.nk = W.nterms; W.N = ((o + 15) / 16) * 16; break;   // one stage per term: all r
    default: W.nk = (o / (CK / 8)) * P.nb; W.N = ((W.nterms * o + 15) / 16) * 16; break;   // (p-group, Q) K chunks
    }
}

// Issues the TMA loads of k-iteration kit into the stage at sA (planes
// [A][A lo][B][B lo], each a_bytes / b_bytes); returns the bytes expected.
// CG2 (CTA pair, F1 only): this CTA (rank) loads its 128 rows of the item's
// 256-row M-tile and its half of B, half-term boxes rank*nterms ..
// (rank+1)*nterms - 1 of o/2 rows each; the bytes of both CTAs complete on
// the leader's full barrier (cbar, shared::cluster address), whose
// transaction count the leader sets.
template <int KIND, int PREC, bool CG2 = false>
__device__ __forceinline__ uint32_t issue_loads(const TcParams &P, const Work &W, int kit, uint32_t sA, uint32_t bar,
                                                uint32_t rank = 0, uint32_t cbar = 0) {
    constexpr int CK = PREC ? 64 : 32;           // elements per 128-byte row
    constexpr uint32_t NP = PREC ? 2u : 1u;      // operand planes
    const int o = P.o;
    const uint32_t sB = sA + NP * (uint32_t)P.a_bytes;
    auto ldA = [&](uint32_t off, int c0, int c1, int c2) {
        if (CG2) {
            tc::tma_load_3d_cg2(sA + off, &P.mapA, cbar, c0, c1, c2);
            if (PREC) tc::tma_load_3d_cg2(sA + P.a_bytes + off, &P.mapA2, cbar, c0, c1, c2);
        } else {
            tc::tma_load_3d(sA + off, &P.mapA, bar, c0, c1, c2);
            if (PREC) tc::tma_load_3d(sA + P.a_bytes + off, &P.mapA2, bar, c0, c1, c2);
        }
    };
    auto ldB = [&](uint32_t off, int c0, int c1, int c2) {
        if (CG2) {
            tc::tma_load_3d_cg2(sB + off, &P.mapB, cbar, c0, c1, c2);
            if (PREC) tc::tma_load_3d_cg2(sB + P.b_bytes + off, &P.mapB2, cbar, c0, c1, c2);
        } else {
            tc::tma_load_3d(sB + off, &P.mapB, bar, c0, c1, c2);
            if (PREC) tc::tma_load_3d(sB + P.b_bytes + off, &P.mapB2, bar, c0, c1, c2);
        }
    };
    const uint32_t chunk = (uint32_t)CK * 128u;  // bytes of a CK x CK MN-major chunk
    uint32_t bytes = 0;                          // per plane
    if constexpr (CG2) {
        static_assert(KIND == TK_F1, "CTA-pair loads are laid out for F1");
        const int hr = o / 2;                    // rows of a half-term box
        bytes = 16384u + (uint32_t)W.nterms * hr * 128u;
        if (rank == 0) tc::mbar_expect_tx(bar, 2u * NP * bytes);
        const int z = W.key;
        ldA(0, CK * kit, (2 * W.mt + (int)rank) * 128, z);
        for (int i = 0; i < W.nterms; ++i) {
            const int hb = (int)rank * W.nterms + i;
            const Term T = term_of(P, P.entries[W.e0 + (hb >> 1)]);
            ldB(i * hr * 128, CK * kit, (hb & 1) * hr, T.x * P.v + T.y);
        }
        return NP * bytes;
    }
    switch (KIND) {
    case TK_F1: {
        constexpr int NT = paired(TK_F1, PREC) ? 2 : 1;   // M-tiles per item
        bytes = NT * 16384u + (uint32_t)W.nterms * o * 128u;
        tc::mbar_expect_tx(bar, NP * bytes);
        const int z = W.key;
        for (int u = 0; u < NT; ++u) ldA(u * 16384u, CK * kit, (NT * W.mt + u) * 128, z);
        for (int t = 0; t < W.nterms; ++t) {
            const Term T = term_of(P, P.entries[W.e0 + t]);
            ldB(t * o * 128, CK * kit, 0, T.x * P.v + T.y);
        }
        break;
    }
    case TK_VB: {
        constexpr int NT = paired(TK_VB, PREC) ? 2 : 1;
        bytes = NT * 16384u + (uint32_t)W.nterms * o * 128u;
        tc::mbar_expect_tx(bar, NP * bytes);
        for (int u = 0; u < NT; ++u) ldA(u * 16384u, CK * kit, (NT * W.mt + u) * 128, W.key);
        for (int t = 0; t < W.nterms; ++t) {
            const Term T = term_of(P, P.entries[W.e0 + t]);
            ldB(t * o * 128, CK * kit, 0, wsl<PREC>(T));
        }
        break;
    }
    case TK_TB: {
        const int kp = PREC ? (o + 15) / 16 * 16 : o;   // K rows (p) of one term, zero-filled past o
        const int nch = W.N / CK;
        bytes = (uint32_t)(128 / CK + nch) * kp * 128u;
        tc::mbar_expect_tx(bar, NP * bytes);
        const Term T = term_of(P, P.entries[W.e0 + kit]);
        for (int c = 0; c < 128 / CK; ++c) ldA(c * kp * 128, W.mt * 128 + CK * c, 0, T.x * P.v + T.y);
        for (int c = 0; c < nch; ++c) ldB(c * kp * 128, W.nt * 256 + CK * c, 0, wsl<PREC>(T));
        break;
    }
    case TK_F2: {
        const int nch = P.ock / CK;
        bytes = 16384u + (uint32_t)W.nterms * nch * chunk;
        tc::mbar_expect_tx(bar, NP * bytes);
        ldA(0, CK * kit, W.mt * 128, W.key);
        for (int t = 0; t < W.nterms; ++t) {
            const Term T = term_of(P, P.entries[W.e0 + t]);
            for (int c = 0; c < nch; ++c) ldB((t * nch + c) * chunk, CK * c, CK * kit, T.z * P.v + T.y);
        }
        break;
    }
    case TK_OB1: {
        // stage kit = term kit, all of K = r: A = its W-bar from the rotated
        // slot (M = 128 tiled pq positions, K rows r < kr8 = o rounded up to a
        // k-step (8 tf32, 16 bf16), MN-major, one box of kr8 rows per CK
        // positions, rows past o zero-filled); B = t2T rows l, K-major, one
        // box per CK of r
        const int kr8 = PREC ? (o + 15) / 16 * 16 : (o + 7) / 8 * 8, nkc = (kr8 + CK - 1) / CK;
        bytes = (uint32_t)(128 / CK) * kr8 * 128u + (uint32_t)nkc * o * 128u;
        tc::mbar_expect_tx(bar, NP * bytes);
        const int eid = P.entries[W.e0 + kit];
        const Term T = term_of(P, eid);
        const int rs = wsl_rot<PREC>(eid);
        for (int c = 0; c < 128 / CK; ++c) ldA(c * kr8 * 128u, W.mt * 128 + CK * c, 0, rs);
        for (int kc = 0; kc < nkc; ++kc) ldB(kc * o * 128u, CK * kc, 0, T.z * P.v + T.y);
        break;
    }
    default: {  // TK_OB2
        // A = vooo rows (p, q8) of K chunk kit = (p-group pk, Q), CK l per
        // chunk (MN-major); B = per term the o rows r of its rotated W-bar
        // slot at the same CK (p, q8) positions, one 128-byte run of the
        // tiled pq plane (K-major)
        const int nch = P.ock / CK;
        const int PK = CK / 8, pk = kit / P.nb, Q = kit - pk * P.nb;
        const int p0 = PK * pk;
        const int koff = (p0 >> 3) * 8 * o + Q * 64 + (p0 & 7) * 8;
        bytes = (uint32_t)nch * chunk + (uint32_t)W.nterms * o * 128u;
        tc::mbar_expect_tx(bar, NP * bytes);
        for (int c = 0; c < nch; ++c) {
            tc::tma_load_4d(sA + c * chunk, &P.mapA, bar, CK * c, 0, Q, W.key * o + p0);
            if (PREC) tc::tma_load_4d(sA + P.a_bytes + c * chunk, &P.mapA2, bar, CK * c, 0, Q, W.key * o + p0);
        }
        for (int t = 0; t < W.nterms; ++t) ldB(t * o * 128, koff, 0, wsl_rot<PREC>(P.entries[W.e0 + t]));
        break;
    }
    }
    return NP * bytes;
}

// MMAs of one stage.  TF32: K = 8 per instruction, MN-major operands in the
// 128-B swizzle with 32-B atoms (4-row atoms, SBO 512).  BF16x3: K = 16 per
// instruction, MN-major operands in the plain 128-B swizzle (8-row atoms, SBO
// 1024); three MMAs per k-step (hi*hi, hi*lo, lo*hi).  K-major operands: 128-B
// swizzle, SBO 1024, +32 bytes per k-step in both.
template <int KIND, int PREC, bool CG2 = false>
__device__ __forceinline__ void issue_mmas(const TcParams &P, const Work &W, int kit, uint32_t sA, uint32_t tacc,
                                           bool first) {
    constexpr int CK = PREC ? 64 : 32;
    constexpr int KS = PREC ? 16 : 8;                    // K per MMA
    constexpr uint32_t MN_SBO = PREC ? 1024u : 512u;
    constexpr uint32_t MN_LAYOUT = PREC ? tc::kSw128 : tc::kSw128Base32;
    constexpr uint32_t MN_STEP = KS * 128u;              // bytes per k-step along K rows
    constexpr uint32_t NP = PREC ? 2u : 1u;
    const int o = P.o;
    const uint32_t sB = sA + NP * (uint32_t)P.a_bytes;
    const uint32_t chunk = (uint32_t)CK * 128u;
    int ksteps = CK / KS;
    // K = l (F2) runs past o in the last chunk: its zero-filled k-steps are
    // not issued
    if (KIND == TK_F2) {
        const int valid = o - CK * kit < CK ? o - CK * kit : CK;
        ksteps = (valid + KS - 1) / KS;
    }
    // OB1: one stage holds all of K = r (kr8 rows of A; B in CK-wide K chunks of o rows)
    const int kr8 = PREC ? (o + 15) / 16 * 16 : (o + 7) / 8 * 8;
    if (KIND == TK_OB1) ksteps = (kr8 + KS - 1) / KS;
    bool amn, bmn;
    uint32_t a_lbo, b_lbo;
    switch (KIND) {
    case TK_F1: amn = false; bmn = false; a_lbo = 16; b_lbo = 16; break;
    case TK_VB: amn = false; bmn = false; a_lbo = 16; b_lbo = 16; break;
    case TK_TB: {
        const int kp = PREC ? (o + 15) / 16 * 16 : o;
        ksteps = kp / KS; amn = true; bmn = true; a_lbo = kp * 128; b_lbo = kp * 128;
        break;
    }
    case TK_F2: amn = false; bmn = true; a_lbo = 16; b_lbo = chunk; break;
    case TK_OB1: amn = true; bmn = false; a_lbo = kr8 * 128; b_lbo = 16; break;
    default: amn = true; bmn = false; a_lbo = chunk; b_lbo = 16; break;   // OB2
    }
    // CTA pair: M = 256 (128 rows in each CTA), B rows split between the CTAs
    const uint32_t id = tc::idesc(PREC ? 1 : 2, CG2 ? 256 : 128, W.N, amn, bmn);
    // K-major k-step kk: 32 bytes along a 128-byte row; OB1's B has one such
    // row block (o rows) per CK of K
    auto desc = [&](uint32_t base, bool mn, uint32_t lbo, int kk) {
        if (mn) return tc::sdesc(base + kk * MN_STEP, lbo, MN_SBO, MN_LAYOUT);
        if (KIND == TK_OB1) {
            constexpr int KPC = CK / KS;   // k-steps per 128-byte row
            return tc::sdesc(base + (kk / KPC) * (uint32_t)o * 128u + (kk % KPC) * 32u, lbo, 1024);
        }
        return tc::sdesc(base + kk * 32u, lbo, 1024);
    };
    for (int kk = 0; kk < ksteps; ++kk) {
        const uint64_t da = desc(sA, amn, a_lbo, kk), db = desc(sB, bmn, b_lbo, kk);
        const uint32_t acc = (first && kk == 0) ? 0u : 1u;
        if (CG2) {
            if (PREC) {
                const uint64_t da2 = desc(sA + P.a_bytes, amn, a_lbo, kk), db2 = desc(sB + P.b_bytes, bmn, b_lbo, kk);
                tc::mma_f16_cg2(tacc, da, db, id, acc);
                tc::mma_f16_cg2(tacc, da, db2, id, 1u);
                tc::mma_f16_cg2(tacc, da2, db, id, 1u);
            } else {
                tc::mma_tf32_cg2(tacc, da, db, id, acc);
            }
        } else if (paired(KIND, PREC)) {
            // second M-tile: A rows at +16 KB, accumulator in TMEM columns 256..
            tc::mma_tf32(tacc, da, db, id, acc);
            tc::mma_tf32(tacc + 256u, desc(sA + 16384u, amn, a_lbo, kk), db, id, acc);
        } else if (PREC) {
            const uint64_t da2 = desc(sA + P.a_bytes, amn, a_lbo, kk), db2 = desc(sB + P.b_bytes, bmn, b_lbo, kk);
            tc::mma_f16(tacc, da, db, id, acc);
            tc::mma_f16(tacc, da, db2, id, 1u);
            tc::mma_f16(tacc, da2, db, id, 1u);
        } else {
            tc::mma_tf32(tacc, da, db, id, acc);
        }
    }
}

// Epilogue of one work item.  Eight epilogue warps: warp w reads TMEM lanes
// 32*(w%4) .. +31 (rows 32*q.. of D), and the two warps of a lane quadrant
// take alternate 16-column chunks (h = 0, 1).  Term descriptors of the work
// item are held one per lane and broadcast with shuffles.  VB reductions go
// straight from registers (coalesced along the rows); F1, TB, F2, OB1 and
// OB2 chunks are transposed through the warp's 32 x 17 shared buffer, so
// that F1 writes G with 16-byte stores (four rows of a column per lane:
// 380 -> 285 ms per benchmark step against 4-byte stores of one row) and
// each reduction instruction of the others covers contiguous runs.
constexpr int kEpiWarps = 8;
constexpr int kThreads = 64 + 32 * kEpiWarps;   // producer warp, MMA warp, epilogue warps
__host__ __device__ constexpr int ebuf_floats(int kind) { return (kind == TK_VB) ? 0 : 32 * 17; }
// epilogue warps that take part: TB keeps one warp per lane quadrant, so its
// transpose buffers leave room for a third shared-memory stage
__host__ __device__ constexpr int epi_active(int kind) { return kind == TK_TB ? 4 : kEpiWarps; }

template <int KIND>
__device__ __forceinline__ void epilogue(const TcParams &P, const Work &W, uint32_t tacc, int q, int h, int lane,
                                         float *ebuf) {
    const int o = P.o, v = P.v, n = P.n;
    const long long o2 = (long long)o * o, o3 = o2 * o;
    const int row = 32 * q + lane;
    const uint32_t tbase = tacc + ((uint32_t)(32 * q) << 16);
    // this lane's term descriptor (lane t <-> term t of the work item)
    Term mine{0, 0, 0, 0, 0};
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
        // this lane's row: qr (F1) or f (VB); column j of a chunk -> (term, p).
        // Paired items: warp half h drains M-tile 2 mt + h (TMEM columns 256 h..);
        // otherwise the halves take alternate 16-column chunks.
        const bool pr = P.pairs != 0;
        const int m = (pr ? 2 * W.mt + h : W.mt) * 128 + row;
        const bool row_ok = (KIND == TK_F1) ? m < o2 : m < v;
        const uint32_t tb = tbase + (pr ? 256u * h : 0u);
        for (int c0 = pr ? 0 : 16 * h; c0 < W.N; c0 += pr ? 16 : 32) {
            tc::tmem_ld16(tb + c0, vals);
            const int t_lo = c0 / o;
            const int p_lo = c0 - t_lo * o;
            const int t_hi = (c0 + 15) / o;   // o >= 8: a 16-column chunk spans at most two terms
            const Term T0 = bcast(t_lo < 32 ? t_lo : 31), T1 = bcast(t_hi < 32 ? t_hi : 31);
            if (!row_ok && KIND != TK_F1) continue;
            if (KIND == TK_F1) {
                // G[slot][p][qr], 16-byte stores: the warp's 32 rows x 16 columns
                // pass through its 32 x 17 transpose buffer, then lane i writes 4
                // consecutive rows (qr) of one column (term, p); each row group
                // lies inside the slot (o^2 % 4 == 0), so one check covers it
#pragma unroll
                for (int j = 0; j < 16; ++j) ebuf[lane * 17 + j] = vals[j];
                __syncwarp();
                const int mrow0 = m - lane;   // first row of this warp's 32
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int f = lane + 32 * u, j = f >> 3, rg = f & 7;   // column, row group
                    const float4 x = make_float4(ebuf[(4 * rg) * 17 + j], ebuf[(4 * rg + 1) * 17 + j],
                                                 ebuf[(4 * rg + 2) * 17 + j], ebuf[(4 * rg + 3) * 17 + j]);
                    const bool wrap = p_lo + j >= o;
                    const int mr = mrow0 + 4 * rg;
                    if ((wrap ? t_lo + 1 : t_lo) < W.nterms && mr < o2) {
                        const long long sl = wrap ? T1.slot : T0.slot;
                        *reinterpret_cast<float4 *>(P.G + sl * o3 + (long long)(wrap ? p_lo + j - o : p_lo + j) * o2 +
                                                    mr) = x;
                    }
                }
                __syncwarp();
            } else {
                // vvop_bar[x,y,p,o+f]: one base per term, p strides of nmo
                double *b0 = P.out + ((long long)T0.x * v + T0.y) * o * n + o + m;
                double *b1 = P.out + ((long long)T1.x * v + T1.y) * o * n + o + m;
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const bool wrap = p_lo + j >= o;
                    if ((wrap ? t_lo + 1 : t_lo) >= W.nterms) continue;
                    atomicAdd((wrap ? b1 : b0) + (long long)(wrap ? p_lo + j - o : p_lo + j) * n, (double)vals[j]);
                }
            }
        }
    } else if (KIND == TK_TB) {
        // 16 columns per pass; half-warps take alternate rows -> 128-byte runs
        const int f0 = W.mt * 128 + 32 * q;
        for (int c0 = 0; c0 < W.N; c0 += 16) {   // one warp per quadrant (h == 0)
            tc::tmem_ld16(tbase + c0, vals);
#pragma unroll
            for (int j = 0; j < 16; ++j) ebuf[lane * 17 + j] = vals[j];
            __syncwarp();
            // column = qr-tiled pair index; t2T-bar is in the plain (q, r) order
            const int qt = W.nt * 256 + c0 + (lane & 15);
            const int Qb = (int)__umulhi((unsigned)qt, P.o_magic) >> 3;   // qt / (8 o)
            const int rem = qt - Qb * 8 * o;
            const int qr = (8 * Qb + ((rem >> 3) & 7)) * o + 8 * (rem >> 6) + (rem & 7);
            double *base = P.out + (long long)W.key * v * o2 + qr;
            // fire-and-forget reductions (the tile has one owner per launch, so
            // each element receives exactly one add: the result is deterministic)
#pragma unroll
            for (int rr = 0; rr < 16; ++rr) {
                const int r = 2 * rr + (lane >> 4);
                const int f = f0 + r;
                if (f < v && qt < o2) atomicAdd(base + (long long)f * o2, (double)ebuf[r * 17 + (lane & 15)]);
            }
            __syncwarp();
        }
    } else if (KIND == TK_OB2) {
        // D[l,(t,r)], o columns per term: a 16-column chunk spans at most two
        // terms (o >= 8); lane i of pass k reduces row 2k + i/16 (l), column
        // i%16 of the chunk into t2T_bar[z,y,l,r] (16 consecutive r per half-warp)
        const int l0 = 32 * q, rows = min(32, o - l0);
        for (int c0 = 16 * h; c0 < W.N; c0 += 32) {
            const int t_lo = c0 / o;
            if (t_lo >= W.nterms || rows <= 0) continue;   // warp-uniform
            const int t_hi = (c0 + 15) / o;
            const Term T0 = bcast(t_lo), T1 = bcast(t_hi < 32 ? t_hi : 31);
            tc::tmem_ld16(tbase + c0, vals);
#pragma unroll
            for (int j = 0; j < 16; ++j) ebuf[lane * 17 + j] = vals[j];
            __syncwarp();
            const int cc = lane & 15;
            const int r0 = c0 + cc - t_lo * o;
            const bool wrap = r0 >= o;
            const bool col_ok = (wrap ? t_lo + 1 : t_lo) < W.nterms;
            const int tz = wrap ? T1.z : T0.z, ty = wrap ? T1.y : T0.y;
            double *dstd = P.out + ((long long)tz * v + ty) * o2 + (long long)l0 * o + (wrap ? r0 - o : r0);
#pragma unroll
            for (int k = 0; k < 16; ++k) {
                const int rr = 2 * k + (lane >> 4);
                if (rr < rows && col_ok) atomicAdd(dstd + rr * o, -(double)ebuf[rr * 17 + cc]);
            }
            __syncwarp();
        }
    } else {
        // F2 / OB1: a chunk is 16 columns of one term's (rows x o) block,
        // contiguous rows of o in memory; lane i of pass k reduces element
        // (row 2k + lane/16, column lane%16) of the chunk
        const int ncols = (KIND == TK_OB1) ? o : W.N;
        for (int c0 = 16 * h; c0 < ncols; c0 += 32) {
            const int t = (KIND == TK_OB1) ? 0 : c0 / P.ock;
            const int cw = (KIND == TK_OB1) ? c0 : c0 - t * P.ock;   // column within the term
            if (t >= ((KIND == TK_OB1) ? 1 : W.nterms) || cw >= o) continue;   // warp-uniform
            const Term T = (KIND == TK_OB1) ? Term{0, 0, 0, 0, 0} : bcast(t);
            tc::tmem_ld16(tbase + c0, vals);
#pragma unroll
            for (int j = 0; j < 16; ++j) ebuf[lane * 17 + j] = vals[j];
            __syncwarp();
            int rows;
            float *dstf = nullptr;
            double *dstd = nullptr;
            const int pq0 = W.mt * 128 + 32 * q;
            rows = (int)min((long long)32, o2 - pq0);
            if (KIND == TK_F2) {
                dstf = P.G + (long long)T.slot * o3;
            } else {
                // OB1 rows: tiled pq positions of the rotated slot
                dstd = P.out + (long long)W.key * o3 + cw;
            }
            if (KIND == TK_F2) {
                // float4 reductions: lane -> (row 8k + lane/4, columns 4*(lane%4) .. +3);
                // o % 8 == 0 and cw % 16 == 0 keep every target 16-byte aligned
                const int c4 = 4 * (lane & 3);
                const bool col_ok = cw + c4 < o;
                const int r = cw + c4;   // four consecutive r inside one 8-tile
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const int rr = 8 * k + (lane >> 2);
                    if (rr < rows && col_ok) {
                        const int pq = pq0 + rr;
                        const int p = (int)__umulhi((unsigned)pq, P.o_magic), qq = pq - p * o;
                        const float *e4 = ebuf + rr * 17 + c4;
                        // qr-tiled slot; one add per element per launch: deterministic
                        tc::red_add_v4(dstf + (long long)p * o2 + (qq >> 3) * 8 * o + (r >> 3) * 64 + (qq & 7) * 8 + (r & 7),
                                       -e4[0], -e4[1], -e4[2], -e4[3]);
                    }
                }
            } else {
                // row = tiled position k -> (p, q): p = 8 (k / 8o) + (k % 64) / 8,
                // q = 8 ((k % 8o) / 64) + k % 8; vooo_bar[x,p,q,:] rows of o
                const int cc = lane & 15;
                const bool col_ok = cw + cc < o;
#pragma unroll
                for (int k = 0; k < 16; ++k) {
                    const int rr = 2 * k + (lane >> 4);
                    const int pt = pq0 + rr;
                    const int Pb = (int)__umulhi((unsigned)pt, P.o_magic) >> 3;   // pt / (8 o)
                    const int rem = pt - Pb * 8 * o;
                    const int pq = (8 * Pb + ((rem >> 3) & 7)) * o + 8 * (rem >> 6) + (rem & 7);
                    if (rr < rows && col_ok) atomicAdd(dstd + (long long)pq * o + cc, -(double)ebuf[rr * 17 + cc]);
                }
            }
            __syncwarp();
        }
    }
}

// CG2: the kernel runs as clusters of two CTAs (a CTA pair on two SMs) that
// share every work item: one thread of the leader (rank 0) issues
// cta_group::2 MMAs with M = 256 (128 rows of A and D in each CTA) and B split
// by rows between the CTAs, so each SM loads half of B; each CTA drains its
// own 128 accumulator rows.  The leader's full barriers count the loads of
// both CTAs, its commits arrive on the stage-empty and accumulator-full
// barriers of both CTAs, and both CTAs' epilogue warps arrive on the leader's
// accumulator-empty barriers.  Accumulators are double-buffered.
template <int KIND, int PREC, bool CG2 = false>
__global__ void __launch_bounds__(kThreads, 1) tc_gemm_kernel(const __grid_constant__ TcParams P) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int S = P.stages;
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + (size_t)S * P.stage_bytes);
    // bars: full[kMaxStages], empty[kMaxStages], acc_full[2], acc_empty[2], drain
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + kBarCount);
    static_assert(8 * kBarCount + 4 <= 256, "barriers and the TMEM slot fit the 256-byte area");
    float *ebuf_all = reinterpret_cast<float *>(smem + (size_t)S * P.stage_bytes + 256);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t sbase = tc::smem_u32(smem);
    auto bar = [&](int i) { return tc::smem_u32(bars + i); };
    constexpr bool PAIRED = paired(KIND, PREC) && !CG2;   // two M-tiles per item in one CTA
    const uint32_t rank = CG2 ? tc::cluster_ctarank() : 0u;
    const int cid = CG2 ? (int)(blockIdx.x >> 1) : (int)blockIdx.x;
    const int ncl = CG2 ? (int)(gridDim.x >> 1) : (int)gridDim.x;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kMaxStages; ++s) {
            tc::mbar_init(bar(s), 1);
            tc::mbar_init(bar(kBarEmpty + s), 1);
        }
        tc::mbar_init(bar(kBarAccFull), 1);
        tc::mbar_init(bar(kBarAccFull + 1), 1);
        tc::mbar_init(bar(kBarAccEmpty), CG2 ? 2 * kEpiWarps : kEpiWarps);
        tc::mbar_init(bar(kBarAccEmpty + 1), CG2 ? 2 * kEpiWarps : kEpiWarps);
        tc::mbar_init(bar(kBarDrain), 1);
        tc::fence_mbar_init();
    }
    if (CG2) {
        // the peer's barriers are initialised before any load or arrive reaches them
        __syncthreads();
        tc::cluster_sync();
    }
    if (warp == 1) {
        if (CG2) {
            tc::tmem_alloc_cg2(tc::smem_u32(tmem_slot), kTmemCols);
            tc::tmem_relinquish_cg2();
        } else {
            tc::tmem_alloc(tc::smem_u32(tmem_slot), kTmemCols);
            tc::tmem_relinquish();
        }
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
            for (int w = cid; w < P.nwork && ok; w += ncl) {
                Work W;
                decode<KIND, PREC>(P, w, W);
                for (int kit = 0; kit < W.nk; ++kit, ++it) {
                    const int s = it % S;
                    if (it >= S && !tc::mbar_wait(bar(kBarEmpty + s), ((it / S) - 1) & 1, err)) { ok = false; break; }
                    const uint32_t sA = sbase + s * P.stage_bytes;
                    issue_loads<KIND, PREC, CG2>(P, W, kit, sA, bar(s), rank, CG2 ? tc::mapa(bar(s), 0) : 0u);
                }
            }
            // drain: every issued copy has landed before this CTA can exit (on
            // a CTA pair the leader's full barriers count the copies of both)
            if (rank == 0) {
                const int issued = it;
                for (int k = issued - 1; k >= 0 && k >= issued - S; --k)
                    tc::mbar_wait(bar(k % S), (k / S) & 1, err);
            }
        }
    } else if (warp == 1) {
        if (lane == 0 && rank == 0) {
            int it = 0, wi = 0;
            bool ok = true;
            for (int w = cid; w < P.nwork && ok; w += ncl, ++wi) {
                Work W;
                decode<KIND, PREC>(P, w, W);
                // paired kinds use both TMEM halves for one item: single-buffered
                const int buf = PAIRED ? 0 : (wi & 1), use = PAIRED ? wi : (wi >> 1);
                if (use > 0 && !tc::mbar_wait(bar(kBarAccEmpty + buf), (use - 1) & 1, err)) break;
                tc::fence_after();
                const uint32_t tacc = tmem + (uint32_t)(buf * 256);
                for (int kit = 0; kit < W.nk; ++kit, ++it) {
                    const int s = it % S;
                    if (!tc::mbar_wait(bar(s), (it / S) & 1, err)) { ok = false; break; }
                    tc::fence_after();
                    const uint32_t sA = sbase + s * P.stage_bytes;
                    issue_mmas<KIND, PREC, CG2>(P, W, kit, sA, tacc, kit == 0);
                    if (CG2) tc::mma_commit_pair(bar(kBarEmpty + s));
                    else tc::mma_commit(bar(kBarEmpty + s));
                }
                if (!ok) break;
                if (CG2) tc::mma_commit_pair(bar(kBarAccFull + buf));
                else tc::mma_commit(bar(kBarAccFull + buf));
            }
            // all issued MMAs complete before TMEM is released
            if (CG2) tc::mma_commit_cg2(bar(kBarDrain));
            else tc::mma_commit(bar(kBarDrain));
            tc::mbar_wait(bar(kBarDrain), 0, err);
        }
    } else {
        const int q = warp & 3, h = (warp - 2) >> 2;   // TMEM lane quadrant, column half
        int wi = 0;
        for (int w = cid; w < P.nwork; w += ncl, ++wi) {
            Work W;
            decode<KIND, PREC>(P, w, W);
            if (CG2) W.mt = 2 * W.mt + (int)rank;   // this CTA's 128-row half of the item
            const int buf = PAIRED ? 0 : (wi & 1), use = PAIRED ? wi : (wi >> 1);
            if (!tc::mbar_wait(bar(kBarAccFull + buf), use & 1, err)) break;
            tc::fence_after();
            if (warp - 2 < epi_active(KIND))
                epilogue<KIND>(P, W, tmem + (uint32_t)(buf * 256), q, h, lane,
                               ebuf_all + (warp - 2) * ebuf_floats(KIND));
            tc::fence_before();
            __syncwarp();
            if (lane == 0) {
                if (CG2) tc::mbar_arrive_cluster(tc::mapa(bar(kBarAccEmpty + buf), 0));
                else tc::mbar_arrive(bar(kBarAccEmpty + buf));
            }
        }
    }
    tc::fence_before();
    __syncthreads();
    // a CTA pair leaves together: no arrive, load or MMA of one CTA may still
    // target the other's shared or tensor memory
    if (CG2) tc::cluster_sync();
    tc::fence_after();
    if (warp == 1) {
        if (CG2) tc::tmem_dealloc_cg2(tmem, kTmemCols);
        else tc::tmem_dealloc(tmem, kTmemCols);
    }
}

// ---------------------------------------------------------------------------
// operand preparation: float64 -> float32 (tf32-rounded) copies, or bf16 hi/lo
// planes, in the layouts the tensor maps use
// ---------------------------------------------------------------------------
// round to the nearest tf32 value (the tensor core truncates the low 13
// mantissa bits; pre-rounding makes that truncation exact and the product
// errors unbiased)
__device__ __forceinline__ float to_tf32(double x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"((float)x));
    return __uint_as_float(r);
}

// x = hi + lo with hi = bf16(x), lo = bf16(x - hi) (both round-to-nearest-even)
__device__ __forceinline__ void split_bf16(double x, __nv_bfloat16 &hi, __nv_bfloat16 &lo) {
    hi = __float2bfloat16_rn((float)x);
    lo = __float2bfloat16_rn((float)(x - (double)__bfloat162float(hi)));
}

template <int PREC>
__global__ void cvt_kernel(const double *__restrict__ src, void *__restrict__ dst, long long n, long long i0,
                           long long i1) {
    for (long long i = i0 + blockIdx.x * (long long)blockDim.x + threadIdx.x; i < i1;
         i += (long long)gridDim.x * blockDim.x) {
        if (PREC) {
            __nv_bfloat16 *d = static_cast<__nv_bfloat16 *>(dst);
            split_bf16(src[i], d[i], d[n + i]);
        } else {
            static_cast<float *>(dst)[i] = to_tf32(src[i]);
        }
    }
}

// vvf[xy][p][f] = vvop[xy][p][o+f], f padded to vp (zeros), for the pairs
// x in [x0, x1), y in [y0, y1) (lo plane v v o vp elements after the hi plane)
template <int PREC>
__global__ void cvt_vv_kernel(const double *__restrict__ vvop, void *__restrict__ vvf, int o, int v, int vp,
                              int x0, int x1, int y0, int y1) {
    const int n = o + v, ny = y1 - y0;
    const long long tot = (long long)v * v * o * vp;
    const long long cnt = (long long)(x1 - x0) * ny * o * vp;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < cnt;
         k += (long long)gridDim.x * blockDim.x) {
        const long long rr = k / vp;                 // row of the rectangle: (x, y, p)
        const int f = (int)(k - rr * vp);
        const long long xy = rr / o;
        const int p = (int)(rr - xy * o), xi = (int)(xy / ny), yi = (int)(xy - (long long)xi * ny);
        const long long r = ((long long)(x0 + xi) * v + y0 + yi) * o + p;
        const long long i = r * vp + f;
        const double x = f < v ? vvop[r * n + o + f] : 0.0;
        if (PREC) {
            __nv_bfloat16 *d = static_cast<__nv_bfloat16 *>(vvf);
            split_bf16(x, d[i], d[tot + i]);
        } else {
            static_cast<float *>(vvf)[i] = to_tf32(x);
        }
    }
}

// t2T with every (q,r) plane qr-tiled: element (zf, q, r) at zf o^2 + (q/8) 8o +
// (r/8) 64 + (q%8) 8 + r%8 (the layout of the scratch slots); tf32 floats or
// bf16 hi/lo planes (lo plane n elements after the hi plane)
template <int PREC>
__global__ void cvt_t2q_kernel(const double *__restrict__ src, void *__restrict__ dst, int o, long long n,
                               long long i0, long long i1) {
    const long long o2 = (long long)o * o;
    for (long long i = i0 + blockIdx.x * (long long)blockDim.x + threadIdx.x; i < i1;
         i += (long long)gridDim.x * blockDim.x) {
        const long long zf = i / o2;
        const int rem = (int)(i - zf * o2), q = rem / o, r = rem - q * o;
        const long long j = zf * o2 + (q >> 3) * 8 * o + (r >> 3) * 64 + (q & 7) * 8 + (r & 7);
        if (PREC) {
            __nv_bfloat16 *d = static_cast<__nv_bfloat16 *>(dst);
            split_bf16(src[i], d[j], d[n + j]);
        } else {
            static_cast<float *>(dst)[j] = to_tf32(src[i]);
        }
    }
}

// t2T[z][f][q][r] -> t2k[z][tiled (q,r)][f] (rows of vp elements), F1's K-major
// A operand: a 32 x 32 tile per (z, f block, qr block), read along (q,r) and
// written along f through shared memory; tf32 floats or bf16 hi/lo planes
// (lo plane n elements after the hi plane)
template <int PREC>
__global__ void __launch_bounds__(256) cvt_t2k_kernel(const double *__restrict__ src, void *__restrict__ dst, int o,
                                                     int v, int vp, long long n, int z0, int z1) {
    __shared__ double tile[32][33];
    const int o2 = o * o;
    const int nqb = (o2 + 31) / 32, nfb = (v + 31) / 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;   // 32 x 8
    for (long long b = (long long)z0 * nfb * nqb + blockIdx.x; b < (long long)z1 * nfb * nqb; b += gridDim.x) {
        const int qb = (int)(b % nqb);
        const long long zf = b / nqb;
        const int fb = (int)(zf % nfb), z = (int)(zf / nfb);
        __syncthreads();
        for (int i = ty; i < 32; i += 8) {
            const int f = fb * 32 + i, pq = qb * 32 + tx;
            tile[i][tx] = (f < v && pq < o2) ? src[((long long)z * v + f) * o2 + pq] : 0.0;
        }
        __syncthreads();
        for (int i = ty; i < 32; i += 8) {
            const int pq = qb * 32 + i, f = fb * 32 + tx;
            if (pq >= o2 || f >= v) continue;
            const int q = pq / o, r = pq - q * o;
            const long long row = (long long)z * o2 + (q >> 3) * 8 * o + (r >> 3) * 64 + (q & 7) * 8 + (r & 7);
            const long long j = row * vp + f;
            if (PREC) {
                __nv_bfloat16 *d = static_cast<__nv_bfloat16 *>(dst);
                split_bf16(tile[tx][i], d[j], d[n + j]);
            } else {
                static_cast<float *>(dst)[j] = to_tf32(tile[tx][i]);
            }
        }
    }
}

// float copies for the epilogue's V tiles: vvoo[xy][p][q] = vvop[xy][p][q < o]
// for the pairs x in [x0, x1), y in [y0, y1); t2f = t2T on elements [i0, i1)
__global__ void cvt_vvoo_kernel(const double *__restrict__ vvop, float *__restrict__ vvoo, int o, int v, int x0,
                                int x1, int y0, int y1) {
    const int n = o + v, ny = y1 - y0;
    const long long cnt = (long long)(x1 - x0) * ny * o * o;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < cnt;
         k += (long long)gridDim.x * blockDim.x) {
        const long long rr = k / o;
        const int q = (int)(k - rr * o);
        const long long xy = rr / o;
        const int p = (int)(rr - xy * o), xi = (int)(xy / ny), yi = (int)(xy - (long long)xi * ny);
        const long long r = ((long long)(x0 + xi) * v + y0 + yi) * o + p;
        vvoo[r * o + q] = (float)vvop[r * n + q];
    }
}

__global__ void cvt_f32_kernel(const double *__restrict__ src, float *__restrict__ dst, long long i0, long long i1) {
    for (long long i = i0 + blockIdx.x * (long long)blockDim.x + threadIdx.x; i < i1;
         i += (long long)gridDim.x * blockDim.x)
        dst[i] = (float)src[i];
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

// 3-D tensor map with a 128-byte swizzle; dims innermost first, strides in
// elements.  prec 0: float32 (MN-major tiles use the 32-B-atom swizzle);
// prec 1: bf16.  Reads outside the dims are zero-filled.
static bool make_map(CUtensorMap *m, const void *base, long long d0, long long d1, long long d2, long long s1,
                     long long s2, int b0, int b1, bool mn, int prec) {
    EncodeTiledFn enc = encode_fn();
    if (!enc) return false;
    const int es = prec ? 2 : 4;
    cuuint64_t dims[3] = {(cuuint64_t)d0, (cuuint64_t)d1, (cuuint64_t)d2};
    cuuint64_t strides[2] = {(cuuint64_t)(s1 * es), (cuuint64_t)(s2 * es)};
    cuuint32_t box[3] = {(cuuint32_t)b0, (cuuint32_t)b1, 1};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = enc(m, prec ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3,
                     const_cast<void *>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     (mn && !prec) ? CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B : CU_TENSOR_MAP_SWIZZLE_128B,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS && std::getenv("CTB_DEBUG"))
        std::fprintf(stderr, "ctb: cuTensorMapEncodeTiled failed (%d) dims %lld %lld %lld box %d %d\n", (int)r, d0, d1,
                     d2, b0, b1);
    return r == CUDA_SUCCESS;
}

// an operand: hi plane (float32 for TF32) and, for BF16x3, the lo plane
struct Opnd {
    const void *hi, *lo;
};

// maps of both planes of an operand
static bool make_maps(CUtensorMap *m, CUtensorMap *m2, Opnd x, long long d0, long long d1, long long d2, long long s1,
                      long long s2, int b0, int b1, bool mn, int prec) {
    if (!make_map(m, x.hi, d0, d1, d2, s1, s2, b0, b1, mn, prec)) return false;
    return !prec || make_map(m2, x.lo, d0, d1, d2, s1, s2, b0, b1, mn, prec);
}

// N-D tensor map (rank 3..5): dims innermost first, element strides of dims
// 1..rank-1, box per dim; the swizzle follows the operand's major-ness as in
// make_map.  Reads outside the dims are zero-filled.
static bool make_map_nd(CUtensorMap *m, const void *base, int rank, const long long *dims, const long long *strides,
                        const int *box, bool mn, int prec) {
    EncodeTiledFn enc = encode_fn();
    if (!enc || rank < 1 || rank > 5) return false;
    const int es = prec ? 2 : 4;
    cuuint64_t d[5], st[4];
    cuuint32_t b[5], estr[5];
    for (int i = 0; i < rank; ++i) {
        d[i] = (cuuint64_t)dims[i];
        b[i] = (cuuint32_t)box[i];
        estr[i] = 1;
        if (i > 0) st[i - 1] = (cuuint64_t)(strides[i - 1] * es);
    }
    CUresult r = enc(m, prec ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, (cuuint32_t)rank,
                     const_cast<void *>(base), d, st, b, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     (mn && !prec) ? CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B : CU_TENSOR_MAP_SWIZZLE_128B,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS && std::getenv("CTB_DEBUG"))
        std::fprintf(stderr, "ctb: cuTensorMapEncodeTiled (rank %d) failed (%d)\n", rank, (int)r);
    return r == CUDA_SUCCESS;
}

static bool make_maps_nd(CUtensorMap *m, CUtensorMap *m2, Opnd x, int rank, const long long *dims,
                         const long long *strides, const int *box, bool mn, int prec) {
    if (!make_map_nd(m, x.hi, rank, dims, strides, box, mn, prec)) return false;
    return !prec || make_map_nd(m2, x.lo, rank, dims, strides, box, mn, prec);
}

double mixed_extra_bytes_per_job(int o, int mode) {
    // BF16x3: the six W-bar slots as bf16 hi/lo planes beside the float slots
    return mode == CT_MODE_BF16X3 ? 6.0 * o * o * o * 2 * sizeof(__nv_bfloat16) : 0.0;
}

// Per-device state of the mixed path (device memory belongs to the device it
// was allocated on): SM count, the device-side timeout flag and the operand
// buffer kept across calls.  Callers hold that device's workspace lock.
struct MixedDev {
    int sms = 0;
    int *err = nullptr;
    void *mbuf = nullptr;
    size_t mbytes = 0;
};
static MixedDev g_md[64];
static MixedDev &md() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) dev = 0;
    return g_md[dev];
}

size_t mixed_operand_bytes(int o, int v, int mode) {
    const int prec = mode == CT_MODE_BF16X3 ? 1 : 0;
    const int vp = prec ? (v + 7) / 8 * 8 : (v + 3) / 4 * 4;
    const size_t n_t2 = (size_t)v * v * o * o, n_vv = (size_t)v * v * o * vp, n_vo = (size_t)v * o * o * o;
    const size_t n_tk = (size_t)v * o * o * vp;
    const size_t es = prec ? 2 * sizeof(__nv_bfloat16) : sizeof(float);
    return (2 * n_t2 + n_vv + n_vo + n_tk) * es + 2 * (size_t)v * v * o * o * sizeof(float);
}

int mixed_setup(const ct_problem *p, int mode, MixedOperands *mo, cudaStream_t st) {
    if (mode != CT_MODE_TF32 && mode != CT_MODE_BF16X3) return CT_ERR_MODE;
    const int prec = mode == CT_MODE_BF16X3 ? 1 : 0;
    const int o = p->nocc, v = p->nvir;
    if (o % 8 != 0 || o > 64) return CT_ERR_SHAPE;
    if (!encode_fn()) return CT_ERR_CUDA;
    MixedDev &M = md();
    if (!M.sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&M.sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) M.sms = 148;
    }
    if (!M.err) {
        if (cudaMalloc(&M.err, sizeof(int)) != cudaSuccess) { M.err = nullptr; return CT_ERR_NOMEM; }
    }
    if (cudaMemsetAsync(M.err, 0, sizeof(int), st) != cudaSuccess) return CT_ERR_CUDA;
    // rows of the vvop copy padded to 16 bytes
    const int vp = prec ? (v + 7) / 8 * 8 : (v + 3) / 4 * 4;
    const size_t n_t2 = (size_t)v * v * o * o, n_vv = (size_t)v * v * o * vp, n_vo = (size_t)v * o * o * o;
    const size_t es = prec ? 2 * sizeof(__nv_bfloat16) : sizeof(float);   // both planes
    const size_t n_oo = (size_t)v * v * o * o;                            // epilogue V-tile copies
    const size_t n_tk = (size_t)v * o * o * vp;                           // K-major t2 copy (F1)
    const size_t bytes = (2 * n_t2 + n_vv + n_vo + n_tk) * es + 2 * n_oo * sizeof(float);
    // the operand buffer is kept across calls (grown when needed): allocating
    // tens of GB per call costs more than the call's conversions
    if (bytes > M.mbytes) {
        if (M.mbuf) {
            cudaStreamSynchronize(st);
            cudaFree(M.mbuf);
        }
        M.mbuf = nullptr;
        M.mbytes = 0;
        if (cudaMalloc(&M.mbuf, bytes) != cudaSuccess) {
            M.mbuf = nullptr;
            return CT_ERR_NOMEM;
        }
        M.mbytes = bytes;
    }
    uint8_t *b8 = static_cast<uint8_t *>(M.mbuf);
    mo->t2 = b8;
    mo->vvop = b8 + n_t2 * es;
    mo->vooo = b8 + (n_t2 + n_vv) * es;
    const size_t pl = prec ? sizeof(__nv_bfloat16) : 0;   // lo plane follows the hi plane
    mo->t2q = b8 + (n_t2 + n_vv + n_vo) * es;
    mo->t2_lo = static_cast<uint8_t *>(mo->t2) + n_t2 * pl;
    mo->vvop_lo = static_cast<uint8_t *>(mo->vvop) + n_vv * pl;
    mo->vooo_lo = static_cast<uint8_t *>(mo->vooo) + n_vo * pl;
    mo->t2q_lo = static_cast<uint8_t *>(mo->t2q) + n_t2 * pl;
    mo->t2k = b8 + (2 * n_t2 + n_vv + n_vo) * es;
    mo->t2k_lo = static_cast<uint8_t *>(mo->t2k) + n_tk * pl;
    mo->vvoo_f = reinterpret_cast<float *>(b8 + (2 * n_t2 + n_vv + n_vo + n_tk) * es);
    mo->t2_f = mo->vvoo_f + n_oo;
    mo->bytes = bytes;
    mo->mode = mode;
    mo->vp = vp;
    return CT_OK;
}

template <int PREC>
static void convert_region(const ct_problem *p, const MixedOperands &mo, const MixedRegion &r, int blocks,
                           cudaStream_t st) {
    const int o = p->nocc, v = p->nvir, vp = mo.vp;
    const long long o2 = (long long)o * o, n_t2 = (long long)v * v * o2, n_vo = (long long)v * o2 * o;
    const long long n_tk = (long long)v * o2 * vp, zrow = (long long)v * o2;
    if (r.z1 > r.z0) {
        const long long i0 = r.z0 * zrow, i1 = r.z1 * zrow;
        cvt_kernel<PREC><<<blocks, 256, 0, st>>>(p->t2T, mo.t2, n_t2, i0, i1);
        cvt_t2q_kernel<PREC><<<blocks, 256, 0, st>>>(p->t2T, mo.t2q, o, n_t2, i0, i1);
        cvt_t2k_kernel<PREC><<<blocks, 256, 0, st>>>(p->t2T, mo.t2k, o, v, vp, n_tk, r.z0, r.z1);
        cvt_f32_kernel<<<blocks, 256, 0, st>>>(p->t2T, mo.t2_f, i0, i1);
    }
    if (r.x1 > r.x0)
        cvt_kernel<PREC><<<blocks, 256, 0, st>>>(p->vooo, mo.vooo, n_vo, r.x0 * o2 * o, r.x1 * o2 * o);
    for (int k = 0; k < r.nrect; ++k) {
        const int *q = r.rect[k];
        if (q[1] <= q[0] || q[3] <= q[2]) continue;
        cvt_vv_kernel<PREC><<<blocks, 256, 0, st>>>(p->vvop, mo.vvop, o, v, vp, q[0], q[1], q[2], q[3]);
        cvt_vvoo_kernel<<<blocks, 256, 0, st>>>(p->vvop, mo.vvoo_f, o, v, q[0], q[1], q[2], q[3]);
    }
}

int mixed_convert(const ct_problem *p, const MixedOperands &mo, const MixedRegion &r, cudaStream_t st) {
    const int v = p->nvir;
    if (r.z0 < 0 || r.z1 > v || r.x0 < 0 || r.x1 > v || r.nrect < 0 || r.nrect > 4) return CT_ERR_SHAPE;
    for (int k = 0; k < r.nrect; ++k)
        if (r.rect[k][0] < 0 || r.rect[k][1] > v || r.rect[k][2] < 0 || r.rect[k][3] > v) return CT_ERR_SHAPE;
    const int blocks = md().sms * 8;
    if (mo.mode == CT_MODE_BF16X3) convert_region<1>(p, mo, r, blocks, st);
    else convert_region<0>(p, mo, r, blocks, st);
    return cudaGetLastError() == cudaSuccess ? CT_OK : CT_ERR_CUDA;
}

int mixed_prepare(const ct_problem *p, int mode, MixedOperands *mo, cudaStream_t st) {
    int rc = mixed_setup(p, mode, mo, st);
    if (rc != CT_OK) return rc;
    MixedRegion all;
    all.z0 = 0; all.z1 = p->nvir;
    all.x0 = 0; all.x1 = p->nvir;
    all.nrect = 1;
    all.rect[0][0] = 0; all.rect[0][1] = p->nvir; all.rect[0][2] = 0; all.rect[0][3] = p->nvir;
    return mixed_convert(p, *mo, all, st);
}

void mixed_release(MixedOperands *mo, cudaStream_t st) {
    (void)st;   // the buffer stays cached for the next call (mixed_free_cache releases it)
    mo->t2 = mo->vvop = mo->vooo = nullptr;
    mo->t2q = mo->t2k = nullptr;
    mo->t2_lo = mo->vvop_lo = mo->vooo_lo = mo->t2q_lo = mo->t2k_lo = nullptr;
    mo->vvoo_f = mo->t2_f = nullptr;
}

constexpr int kSmemMax = 232448;

template <int KIND, int PREC>
static int launch_tc(TcParams &P, cudaStream_t st) {
    if (P.nwork <= 0) return CT_OK;
    const int smem = P.stages * P.stage_bytes + 1024 + 256 + epi_active(KIND) * ebuf_floats(KIND) * 4;
    if (smem > kSmemMax) return CT_ERR_SHAPE;
    if (smem_optin(reinterpret_cast<const void *>(tc_gemm_kernel<KIND, PREC>), kSmemMax) != cudaSuccess)
        return CT_ERR_CUDA;
    const int sms = md().sms;
    const int grid = P.nwork < sms ? P.nwork : sms;
    // at least ~116 KB so that a second CTA never shares the SM's tensor memory
    const int smem_req = smem < 120 * 1024 ? 120 * 1024 : smem;
    tc_gemm_kernel<KIND, PREC><<<grid, kThreads, smem_req, st>>>(P);
    return cudaGetLastError() == cudaSuccess ? CT_OK : CT_ERR_CUDA;
}

// CTA pairs for F1: off by default (CTB_CTA_PAIRS=1 selects them).  Measured
// on the nocc=48/nvir=500 benchmark block, F1 took 466 ms per step on CTA
// pairs against 374 ms with paired M-tiles in one CTA (same box): the pairs
// overlap F1's G stores with the next item's MMAs, but each SM then carries
// half the work per stage with its own loads and the cross-SM barriers, and
// that costs more than the store phase it hides.
static bool cta_pairs_enabled() {
    static const bool on = [] {
        const char *e = std::getenv("CTB_CTA_PAIRS");
        return e && e[0] == '1';
    }();
    return on;
}

// CTA-pair launch: clusters of two CTAs, one pair per two SMs
template <int KIND, int PREC>
static int launch_tc_pair(TcParams &P, cudaStream_t st) {
    if (P.nwork <= 0) return CT_OK;
    const int smem = P.stages * P.stage_bytes + 1024 + 256 + epi_active(KIND) * ebuf_floats(KIND) * 4;
    if (smem > kSmemMax) return CT_ERR_SHAPE;
    const void *fn = reinterpret_cast<const void *>(tc_gemm_kernel<KIND, PREC, true>);
    if (smem_optin(fn, kSmemMax) != cudaSuccess) return CT_ERR_CUDA;
    const int pairs = md().sms / 2;
    const int grid = 2 * (P.nwork < pairs ? P.nwork : pairs);
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = smem < 120 * 1024 ? 120 * 1024 : smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, tc_gemm_kernel<KIND, PREC, true>, P) == cudaSuccess ? CT_OK : CT_ERR_CUDA;
}

// stage layout and depth: per-plane operand bytes a/b, both planes for BF16x3
static void set_stages(TcParams &P, int a_bytes, int b_bytes, int prec, int kind) {
    P.a_bytes = a_bytes;
    P.b_bytes = b_bytes;
    P.stage_bytes = (prec ? 2 : 1) * (a_bytes + b_bytes);
    int s = (kSmemMax - 1024 - 256 - epi_active(kind) * ebuf_floats(kind) * 4) / P.stage_bytes;
    P.stages = s > kMaxStages ? kMaxStages : s;
}

template <int PREC>
static int mixed_wave_p(const WaveView &w, const EpiArgs &e, const ct_grads *g, const MixedOperands &mo, bool vjp,
                        void *scratch, cudaStream_t st, int (*prof)(int, int, void *), void *pctx) {
    constexpr int CK = PREC ? 64 : 32;
    const int o = w.o, v = w.v, n = w.n, vp = mo.vp;
    const long long o2 = (long long)o * o, o3 = o2 * o;
    float *G = (float *)scratch;
    const long long slots = (long long)w.n_jobs * kSlots;
    const Opnd t2{mo.t2, mo.t2_lo}, t2q{mo.t2q, mo.t2q_lo}, t2k{mo.t2k, mo.t2k_lo}, vv{mo.vvop, mo.vvop_lo},
        vo{mo.vooo, mo.vooo_lo};
    // W-bar operand: the float slots (TF32) or the bf16 planes after the wave's
    // slots (every hi plane, then every lo plane)
    __nv_bfloat16 *wb = reinterpret_cast<__nv_bfloat16 *>(G + slots * o3);
    const long long wn = PREC ? (long long)w.n_jobs * 6 : slots;   // W-bar operand count
    const long long ws = o3;                                        // W-bar operand stride
    const Opnd Wb = PREC ? Opnd{wb, wb + wn * o3} : Opnd{G, nullptr};
    const int nb = o / 8;
    const int kp = PREC ? (o + 15) / 16 * 16 : o;                   // TB K rows per term
    TcParams base{};
    base.o = o; base.v = v; base.n = n; base.vp = vp; base.ock = (o + CK - 1) / CK * CK;
    base.nb = nb;
    base.o_magic = (unsigned)(((1ull << 32) + o - 1) / o);
    base.jobs = w.jobs;
    base.G = G;
    base.err = md().err;
    int rc;
    // ---- F1: D[qr,(t,p)], A = K-major t2 copy (f,qr,z) box(CK,128), B = vvf (f,p,xy) K-major.
    //      Paired M-tiles in one CTA (TF32); optionally (nocc % 16 == 0) CTA pairs:
    //      256 qr rows per item, each CTA loading its 128 rows and half of the
    //      terms' B rows as o/2-row boxes, double-buffered accumulators
    {
        TcParams P = base;
        const bool pair_ctas = o % 16 == 0 && cta_pairs_enabled();
        if (!make_maps(&P.mapA, &P.mapA2, t2k, v, o2, v, vp, o2 * vp, CK, 128, false, PREC)) return CT_ERR_CUDA;
        if (!make_maps(&P.mapB, &P.mapB2, vv, vp, o, (long long)v * v, vp, (long long)o * vp, CK, pair_ctas ? o / 2 : o,
                       false, PREC))
            return CT_ERR_CUDA;
        P.groups = w.zchunks; P.entries = w.tb_entries;
        if (pair_ctas) {
            P.pairs = 0;
            P.m_tiles = (int)((o2 + 255) / 256);
            P.nwork = w.n_zchunks * P.m_tiles;
            set_stages(P, 16384, 128 * 128, PREC, TK_F1);
        } else {
            P.pairs = paired(TK_F1, PREC) ? 1 : 0;
            P.m_tiles = (int)((o2 + 127) / 128);
            if (P.pairs) P.m_tiles = (P.m_tiles + 1) / 2;
            P.nwork = w.n_zchunks * P.m_tiles;
            set_stages(P, (P.pairs ? 2 : 1) * 16384, 256 * 128, PREC, TK_F1);
        }
        if (prof) prof(PK_MF, 0, pctx);
        rc = pair_ctas ? launch_tc_pair<TK_F1, PREC>(P, st) : launch_tc<TK_F1, PREC>(P, st);
        if (rc != CT_OK) return rc;
        if (prof) prof(PK_MF, 1, pctx);
    }
    // ---- F2: D[pq,(t,r)], A = voof (l,pq,x) K-major, B = t2 (r,l,zy) MN-major
    {
        TcParams P = base;
        if (!make_maps(&P.mapA, &P.mapA2, vo, o, o2, v, o, o2 * o, CK, 128, false, PREC)) return CT_ERR_CUDA;
        if (!make_maps(&P.mapB, &P.mapB2, t2, o, o, (long long)v * v, o, o2, CK, CK, true, PREC)) return CT_ERR_CUDA;
        P.m_tiles = (int)((o2 + 127) / 128);
        P.groups = w.xchunks; P.entries = w.x_entries;
        P.nwork = w.n_xchunks * P.m_tiles;
        set_stages(P, 16384, 256 * 128, PREC, TK_F2);
        if (prof) prof(PK_MOO, 0, pctx);
        if ((rc = launch_tc<TK_F2, PREC>(P, st)) != CT_OK) return rc;
        if (prof) prof(PK_MOO, 1, pctx);
    }
    {
        EpiArgs e2 = e;
        e2.wbar_bf16 = PREC ? wb : nullptr;
        e2.vvoo_f = mo.vvoo_f;
        e2.t2_f = mo.t2_f;
        if (vjp && e.lno_phase == 2) {
            // LNO VJP: the forward pass (W, z/D into slots 0-1), then the
            // projected cubes A, B (slots 2-5) with the job energies and the
            // mat_bar partials; the epilogue below is the backward pass
            EpiArgs ef = e2;
            ef.with_vjp = 0;
            ef.lno_phase = 1;
            if (prof) prof(PK_EPI, 0, pctx);
            cudaError_t ce = f32_epilogue(w, ef, G, st);
            if (prof) prof(PK_EPI, 1, pctx);
            if (ce != cudaSuccess) return CT_ERR_CUDA;
            if (prof) prof(PK_RED, 0, pctx);
            ce = f32_lno_vjp_project(w, e, G, st);
            if (prof) prof(PK_RED, 1, pctx);
            if (ce != cudaSuccess) return CT_ERR_CUDA;
        }
        if (prof) prof(PK_EPI, 0, pctx);
        cudaError_t ce = f32_epilogue(w, e2, G, st);
        if (prof) prof(PK_EPI, 1, pctx);
        if (ce != cudaSuccess) return CT_ERR_CUDA;
    }
    if (!vjp && e.lno_phase == 1) {
        // LNO energy: project the W and z/D cubes the epilogue left in slots 0-1
        if (prof) prof(PK_VT, 0, pctx);
        cudaError_t ce = f32_lno_contract(w, e, G, st);
        if (prof) prof(PK_VT, 1, pctx);
        if (ce != cudaSuccess) return CT_ERR_CUDA;
    }
    if (vjp) {
        { if (prof) prof(PK_VT, 0, pctx);
          cudaError_t ce = f32_vterm(w, e, G, st);
          if (prof) prof(PK_VT, 1, pctx);
          if (ce != cudaSuccess) return CT_ERR_CUDA; }
        // ---- VB: D[f,(t,p)], A = qr-tiled t2 (qr,f,z) K-major box(CK,128), B = Wbar (qr,p,slot) K-major
        {
            TcParams P = base;
            if (!make_maps(&P.mapA, &P.mapA2, t2q, o2, v, v, o2, (long long)v * o2, CK, 128, false, PREC))
                return CT_ERR_CUDA;
            if (!make_maps(&P.mapB, &P.mapB2, Wb, o2, o, wn, o2, ws, CK, o, false, PREC)) return CT_ERR_CUDA;
            P.pairs = paired(TK_VB, PREC) ? 1 : 0;
            P.m_tiles = (v + 127) / 128;
            if (P.pairs) P.m_tiles = (P.m_tiles + 1) / 2;
            P.groups = w.zchunks; P.entries = w.tb_entries;
            P.nwork = w.n_zchunks * P.m_tiles;
            P.out = g->vvop;
            set_stages(P, (P.pairs ? 2 : 1) * 16384, 256 * 128, PREC, TK_VB);
            if (prof) prof(PK_MVB, 0, pctx);
            if ((rc = launch_tc<TK_VB, PREC>(P, st)) != CT_OK) return rc;
            if (prof) prof(PK_MVB, 1, pctx);
        }
        // ---- TB: D[f,qr], A = vvf (f,p,xy) MN-major, B = Wbar (qr,p,slot) MN-major
        {
            TcParams P = base;
            if (!make_maps(&P.mapA, &P.mapA2, vv, vp, o, (long long)v * v, vp, (long long)o * vp, CK, kp, true, PREC))
                return CT_ERR_CUDA;
            if (!make_maps(&P.mapB, &P.mapB2, Wb, o2, o, wn, o2, ws, CK, kp, true, PREC)) return CT_ERR_CUDA;
            P.m_tiles = (v + 127) / 128;
            P.n_tiles = (int)((o2 + 255) / 256);
            P.groups = w.tb_groups; P.entries = w.tb_entries;
            P.nwork = w.n_tb_groups * P.m_tiles * P.n_tiles;
            P.out = g->t2T;
            set_stages(P, (128 / CK) * kp * 128, (256 / CK) * kp * 128, PREC, TK_TB);
            if (prof) prof(PK_MTB, 0, pctx);
            if ((rc = launch_tc<TK_TB, PREC>(P, st)) != CT_OK) return rc;
            if (prof) prof(PK_MTB, 1, pctx);
        }
        // ---- OB1: D[tiled pq,l], A = rotated Wbar (tiled pq, r, slot) MN-major box(CK, o8),
        //      B = t2 (r,l,zy) K-major box(CK,o); one stage per term (all of r)
        {
            TcParams P = base;
            const int kr8 = PREC ? (o + 15) / 16 * 16 : (o + 7) / 8 * 8;   // K rows: whole k-steps
            if (!make_maps(&P.mapA, &P.mapA2, Wb, o2, o, wn, o2, ws, CK, kr8, true, PREC)) return CT_ERR_CUDA;
            if (!make_maps(&P.mapB, &P.mapB2, t2, o, o, (long long)v * v, o, o2, CK, o, false, PREC)) return CT_ERR_CUDA;
            P.m_tiles = (int)((o2 + 127) / 128);
            P.groups = w.xgroups; P.entries = w.x_entries;
            P.nwork = w.n_xgroups * P.m_tiles;
            P.out = g->vooo;
            set_stages(P, 128 * kr8 * (PREC ? 2 : 4), ((kr8 + CK - 1) / CK) * o * 128, PREC, TK_OB1);
            if (prof) prof(PK_MOB1, 0, pctx);
            if ((rc = launch_tc<TK_OB1, PREC>(P, st)) != CT_OK) return rc;
            if (prof) prof(PK_MOB1, 1, pctx);
        }
        // ---- OB2: D[l,(t,r)], A = voof rows (p,q8) (l,q8,Q,xp) MN-major, B = rotated Wbar
        //      (tiled pq, r, slot) K-major box(CK,o) per term; K chunks (CK/8 p, one Q);
        //      o accumulator columns per term
        {
            TcParams P = base;
            const long long dA[4] = {o, 8, nb, (long long)v * o}, sA[3] = {o, 8LL * o, o2};
            const int bA[4] = {CK, 8, 1, CK / 8};
            if (!make_maps_nd(&P.mapA, &P.mapA2, vo, 4, dA, sA, bA, true, PREC)) return CT_ERR_CUDA;
            if (!make_maps(&P.mapB, &P.mapB2, Wb, o2, o, wn, o2, ws, CK, o, false, PREC)) return CT_ERR_CUDA;
            P.groups = w.ochunks; P.entries = w.x_entries;
            P.nwork = w.n_ochunks;
            P.out = g->t2T;
            set_stages(P, 16384, 256 * 128, PREC, TK_OB2);
            if (prof) prof(PK_MOB2, 0, pctx);
            if ((rc = launch_tc<TK_OB2, PREC>(P, st)) != CT_OK) return rc;
            if (prof) prof(PK_MOB2, 1, pctx);
        }
    }
    return CT_OK;
}

int mixed_wave(const WaveView &w, const EpiArgs &e, const ct_problem *p, const ct_grads *g, const MixedOperands &mo,
               int mode, bool vjp, void *scratch, cudaStream_t st, int (*prof)(int, int, void *), void *pctx) {
    (void)p;
    if (mode == CT_MODE_BF16X3) return mixed_wave_p<1>(w, e, g, mo, vjp, scratch, st, prof, pctx);
    return mixed_wave_p<0>(w, e, g, mo, vjp, scratch, st, prof, pctx);
}

void mixed_free_cache() {
    MixedDev &M = md();
    if (M.mbuf) cudaFree(M.mbuf);
    M.mbuf = nullptr;
    M.mbytes = 0;
}

int mixed_check_error(cudaStream_t st) {
    MixedDev &M = md();
    if (!M.err) return CT_OK;
    int h = 0;
    if (cudaMemcpyAsync(&h, M.err, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess) return CT_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return CT_ERR_CUDA;
    return h ? CT_ERR_TIMEOUT : CT_OK;
}

}  // namespace ctb
