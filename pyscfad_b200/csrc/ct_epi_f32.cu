// Orbit epilogue of the mixed-precision path, software-pipelined.
//
// Same arithmetic as the float64 path's epi_kernel (ct_epi.cuh:
// orbit_element), on float scratch: one CTA of 512 threads per job, T = 8
// blocks, one element orbit per thread per block-orbit.  The staged operands
// of a block-orbit (the 36 G tiles of its permuted blocks and the 36 + 36
// V-term tiles) are double-buffered in shared memory and fetched with
// cp.async one block-orbit ahead, so the loads of block-orbit i+1 overlap the
// arithmetic of block-orbit i; on the TF32 path W-bar replaces the G tiles in
// shared memory and leaves with 16-byte stores one block-orbit later.  The V-term tiles come
// from float copies of vvop[:,:,:,:o] and t2T made once per call, so they can
// be copied asynchronously as well.
//
// Requires nocc % 8 == 0 (every block full), nocc <= 64.
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include "ct_common.cuh"
#include "ct_internal.h"
#include "ct_epi.cuh"

namespace ctb {
namespace epipipe {

constexpr int T = 8, T2 = 64, T3 = 512, TP = T2 + 4, BLK = T * TP, NTHR = 512;

struct Smem {
    static constexpr size_t g_bytes = sizeof(float) * 36 * BLK;      // one buffer of G tiles
    static constexpr size_t v_bytes = sizeof(float) * 36 * T2;       // one buffer of VA (or VB)
    static constexpr size_t buf_bytes = g_bytes + 2 * v_bytes;
    static constexpr size_t u_off = 2 * buf_bytes;                   // float[6][64]
    static constexpr size_t w_off = u_off + sizeof(float) * 6 * 64;  // float[6][64]
    static constexpr size_t occ_off = w_off + sizeof(float) * 6 * 64;        // double[64]
    static constexpr size_t eocc_off = occ_off + sizeof(double) * 64;        // double[64]
    static constexpr size_t tmp_off = eocc_off + sizeof(double) * 64;        // double[T3]
    static constexpr size_t y_off = tmp_off + sizeof(double) * T3;           // float[2][6 * BLK]: ybar staging
    static constexpr size_t y_bytes = sizeof(float) * 6 * BLK;
    static constexpr size_t bytes = y_off + 2 * y_bytes;
};
static_assert(Smem::bytes <= 227 * 1024, "shared memory");

// Neumaier pair (s, c) and a plain partial v summed down a warp by a fixed
// shuffle tree (offsets top, top/2, ..., 1); lane 0 holds the result
__device__ __forceinline__ void warp_ksum(double &s, double &c, double &v, int top) {
    for (int m = top; m >= 1; m >>= 1) {
        const double s2 = __shfl_down_sync(0xffffffffu, s, m), c2 = __shfl_down_sync(0xffffffffu, c, m);
        v += __shfl_down_sync(0xffffffffu, v, m);
        KSum k;
        k.s = s;
        k.c = c + c2;
        k.add(s2);
        s = k.s;
        c = k.c;
    }
}

// sorted block triple I >= J >= K, K fastest
struct BlockIter {
    int I = 0, J = 0, K = 0;
    __device__ void next() {
        if (K < J) ++K;
        else if (J < I) { ++J; K = 0; }
        else { ++I; J = 0; K = 0; }
    }
};

// permuted blocks of a block-orbit: bs[s] = block of slot s, dmap[s] = its
// staging buffer, fresh[s] = first slot with that block (compile-time indices)
struct OrbitBlocks {
    int bs[6][3], dmap[6];
    bool fresh[6];
    __device__ __forceinline__ void set(const BlockIter &it) {
        const int blk[3] = {it.I, it.J, it.K};
        int nd = 0;
#pragma unroll
        for (int s = 0; s < 6; ++s) {
#pragma unroll
            for (int m = 0; m < 3; ++m) bs[s][m] = blk[kR(s, m)];
            int found = -1;
#pragma unroll
            for (int t = 0; t < s; ++t)
                if (found < 0 && bs[t][0] == bs[s][0] && bs[t][1] == bs[s][1] && bs[t][2] == bs[s][2]) found = dmap[t];
            fresh[s] = found < 0;
            dmap[s] = found < 0 ? nd++ : found;
        }
    }
};

// cp.async of block-orbit `it`'s G tiles and V tiles into buffer (G, VA, VB).
// lbar (LNO backward pass): the z/D cube and the two parts of the A and B
// cubes (slots 1-5) into tile groups 0-4, and no V tiles.
__device__ __forceinline__ void issue_stage(const BlockIter &it, const OrbitBlocks &ob, const float *S, long long o3,
                                            int o, float *G, float *VA, float *VB, const float *vvf, const float *t2f,
                                            const long long *vv_off, const long long *tt_off, int tid, bool with_fvo,
                                            bool lbar = false) {
    const int ng = lbar ? 5 : 6, s0 = lbar ? 1 : 0;
#pragma unroll
    for (int s = 0; s < 6; ++s) {
        if (!ob.fresh[s]) continue;
        const int d = ob.dmap[s];
        const int p0 = ob.bs[s][0] * T, q0 = ob.bs[s][1] * T, r0 = ob.bs[s][2] * T;
        // ng slots x 128 16-byte pieces of an 8^3 block
        for (int j = tid; j < ng * 128; j += NTHR) {
            const int sg = j >> 7, e3 = (j & 127) * 4;
            const int u = e3 >> 6;
            // qr-tiled slot: row u of the block is 64 contiguous floats
            cp_async16(G + (sg * 6 + d) * BLK + u * TP + (e3 & 63),
                       S + (sg + s0) * o3 + (long long)(p0 + u) * o * o + q0 * o + 8 * r0 + (e3 & 63));
        }
    }
    if (lbar) return;
    // V tiles: for each term sg and slot cc, the T x T tile (rows P, columns Q)
    // on the blocks of slot cc's first two axes; 2 x 16 pieces per tile
    constexpr unsigned int KR01 = (0u | 1u << 2) | (0u | 2u << 2) << 4 | (1u | 0u << 2) << 8 | (1u | 2u << 2) << 12 |
                                  (2u | 0u << 2) << 16 | (2u | 1u << 2) << 20;
    for (int j = tid; j < (with_fvo ? 2 : 1) * 36 * 16; j += NTHR) {
        const int which = j / (36 * 16), jj = j - which * (36 * 16);
        const int tile = jj >> 4, piece = jj & 15;
        const int sg = tile / 6, cc = tile - 6 * sg;
        const int k0 = (KR01 >> (4 * cc)) & 3, k1 = (KR01 >> (4 * cc + 2)) & 3;
        const int P = (k0 == 0 ? it.I : (k0 == 1 ? it.J : it.K)) * T + (piece >> 1);
        const int Q = (k1 == 0 ? it.I : (k1 == 1 ? it.J : it.K)) * T + (piece & 1) * 4;
        const long long src = (which ? tt_off[sg] : vv_off[sg]) + (long long)P * o + Q;
        cp_async16((which ? VB : VA) + tile * T2 + (piece >> 1) * T + (piece & 1) * 4, (which ? t2f : vvf) + src);
    }
}

// W-bar (tf32-rounded floats) of a finished block-orbit, written in place of
// its G tiles in buffer G, out to the job's slots 0-5 in 16-byte pieces along
// r.  A thread flushes exactly the pieces it fetches into the same buffer with
// issue_stage (piece j of every tile belongs to thread j mod NTHR), and its
// global stores consume its shared loads, so the buffer can be refilled right
// after without another barrier.
// With nsg = 2 (LNO energy) only slots 0-1 leave: the W and z/D cubes the
// element orbits wrote there in place of the G tiles.
__device__ __forceinline__ void flush_wbar(const OrbitBlocks &ob, const float *G, float *S, long long o3, int o,
                                           int tid, int nsg = 6) {
#pragma unroll
    for (int s = 0; s < 6; ++s) {
        if (!ob.fresh[s]) continue;
        const int d = ob.dmap[s];
        const int p0 = ob.bs[s][0] * T, q0 = ob.bs[s][1] * T, r0 = ob.bs[s][2] * T;
        for (int j = tid; j < nsg * 128; j += NTHR) {
            const int sg = j >> 7, e3 = (j & 127) * 4;
            const int u = e3 >> 6, ww = (e3 >> 3) & 7, t = e3 & 7;
            (void)ww; (void)t;
            const float4 x = *reinterpret_cast<const float4 *>(G + (sg * 6 + d) * BLK + u * TP + (e3 & 63));
            *reinterpret_cast<float4 *>(S + sg * o3 + (long long)(p0 + u) * o * o + q0 * o + 8 * r0 + (e3 & 63)) = x;
        }
    }
}

// BF16x3: the same staged W-bar (whole floats) out as the bf16 hi/lo planes
// the GEMMs read (x = hi + lo, elementwise in the slots' qr-tiled order), in
// 8-element pieces: 16-byte stores to each plane.  A piece here is two of the
// refill's 4-element pieces, owned by other threads, so the caller puts a
// barrier between this write-back and the refill.
__device__ __forceinline__ void flush_wbar_bf16(const OrbitBlocks &ob, const float *G, __nv_bfloat16 *hi,
                                                __nv_bfloat16 *lo, long long o3, int o, int tid) {
#pragma unroll
    for (int s = 0; s < 6; ++s) {
        if (!ob.fresh[s]) continue;
        const int d = ob.dmap[s];
        const int p0 = ob.bs[s][0] * T, q0 = ob.bs[s][1] * T, r0 = ob.bs[s][2] * T;
        for (int j = tid; j < 6 * 64; j += NTHR) {
            const int sg = j >> 6, e8 = (j & 63) * 8, u = e8 >> 6, col = e8 & 63;
            const float *src = G + (sg * 6 + d) * BLK + u * TP + col;
            const float4 x0 = *reinterpret_cast<const float4 *>(src);
            const float4 x1 = *reinterpret_cast<const float4 *>(src + 4);
            const float xs[8] = {x0.x, x0.y, x0.z, x0.w, x1.x, x1.y, x1.z, x1.w};
            __align__(16) __nv_bfloat16 h[8], l[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                h[k] = __float2bfloat16_rn(xs[k]);
                l[k] = __float2bfloat16_rn(xs[k] - __bfloat162float(h[k]));
            }
            const long long pos = sg * o3 + (long long)(p0 + u) * o * o + q0 * o + 8 * r0 + col;
            *reinterpret_cast<uint4 *>(hi + pos) = *reinterpret_cast<const uint4 *>(h);
            *reinterpret_cast<uint4 *>(lo + pos) = *reinterpret_cast<const uint4 *>(l);
        }
    }
}

// ybar of a finished block-orbit, staged in shared memory in the layout of the
// G tiles (block d of the orbit at d * BLK), out to the job's slot 6 with
// 16-byte stores: each block is eight runs of 64 contiguous floats there.
__device__ __forceinline__ void flush_ybar(const OrbitBlocks &ob, const float *Y, float *S6, int o, int tid) {
#pragma unroll
    for (int s = 0; s < 6; ++s) {
        if (!ob.fresh[s]) continue;
        const int d = ob.dmap[s];
        const int p0 = ob.bs[s][0] * T, q0 = ob.bs[s][1] * T, r0 = ob.bs[s][2] * T;
        for (int j = tid; j < 128; j += NTHR) {
            const int e3 = j * 4, u = e3 >> 6;
            const float4 x = *reinterpret_cast<const float4 *>(Y + d * BLK + u * TP + (e3 & 63));
            *reinterpret_cast<float4 *>(S6 + (long long)(p0 + u) * o * o + q0 * o + 8 * r0 + (e3 & 63)) = x;
        }
    }
}

// W-bar is written into the block-orbit's shared G tiles and leaves one
// block-orbit later: WB 1 (TF32) rounded to tf32, to the float slots with
// 16-byte stores (flush_wbar); WB 2 (BF16x3) as whole floats, converted on
// the way out to the bf16 hi/lo planes the GEMMs read, 16-byte stores to each
// plane (flush_wbar_bf16).  BF16x3 used to store W-bar from registers and
// split the slots into planes in a second kernel (633 ms of a 1973 ms
// benchmark step for the two).
template <int WB>
__global__ void __launch_bounds__(NTHR, 1) epi_pipe_kernel(const WaveView w, const EpiArgs e, float *scratch) {
    extern __shared__ __align__(16) uint8_t esm[];
    float *Us = reinterpret_cast<float *>(esm + Smem::u_off);
    float *Ws = reinterpret_cast<float *>(esm + Smem::w_off);
    double *occ_acc = reinterpret_cast<double *>(esm + Smem::occ_off);
    double *eocc = reinterpret_cast<double *>(esm + Smem::eocc_off);
    double *tmp_s = reinterpret_cast<double *>(esm + Smem::tmp_off);
    auto bufG = [&](int i) { return reinterpret_cast<float *>(esm + i * Smem::buf_bytes); };
    auto bufA = [&](int i) { return reinterpret_cast<float *>(esm + i * Smem::buf_bytes + Smem::g_bytes); };
    auto bufB = [&](int i) {
        return reinterpret_cast<float *>(esm + i * Smem::buf_bytes + Smem::g_bytes + Smem::v_bytes);
    };
    auto bufY = [&](int i) { return reinterpret_cast<float *>(esm + Smem::y_off + i * Smem::y_bytes); };
    __shared__ long long vv_off[6], tt_off[6];

    const int o = e.o, v = e.v;
    const long long o3 = (long long)o * o * o;
    const int jl = blockIdx.x, tid = threadIdx.x;
    int a, b, c;
    unpack_job(w.jobs[jl], a, b, c);
    const double fac = job_fac(a, b, c);
    const double eabc = e.mo_energy[o + a] + e.mo_energy[o + b] + e.mo_energy[o + c];
    float *S = scratch + (long long)jl * kSlots * o3;
    const bool vjp = e.with_vjp != 0;
    // LNO energy: the element orbits leave the W cube in slot 0 and z/D in
    // slot 1 (staged in the G tiles, flushed like W-bar) for the projection
    const bool lno = e.lno_phase == 1 && !vjp;
    // LNO backward pass: z/D, A and B staged from slots 1-5; W-bar and ybar
    // leave as on the canonical VJP path
    const bool lbar = e.lno_phase == 2 && vjp;
    if (tid < 6) {
        int x, y, z;
        term_xyz(tid, a, b, c, x, y, z);
        vv_off[tid] = ((long long)(x * v + y) * o) * o;
        tt_off[tid] = ((long long)(y * v + x) * o) * o;
    }
    for (int i = tid; i < o; i += NTHR) { occ_acc[i] = 0.0; eocc[i] = e.mo_energy[i]; }
    int fvo_nz = 0;
    for (int i = tid; i < 6 * o; i += NTHR) {
        const int sg = i / o, r = i - sg * o;
        int x, y, z;
        term_xyz(sg, a, b, c, x, y, z);
        Us[sg * 64 + r] = (float)e.t1T[z * o + r];
        const double f = e.fvo[z * o + r];
        Ws[sg * 64 + r] = (float)f;
        fvo_nz |= (f != 0.0);
    }
    // the fvo part of V (and its t2T tiles) is skipped when this job's fvo rows are zero
    const bool with_fvo = __syncthreads_or(fvo_nz) != 0;

    KSum eacc;
    double vir_acc = 0.0;
    const double eb = e.et_bar;
    const int nb = o / T;
    const int nbo = nb * (nb + 1) * (nb + 2) / 6;
    constexpr bool STAGED = WB == 1 || WB == 2;   // W-bar staged in the G tiles
    // BF16x3: this job's hi / lo planes (plane jl*6 + sigma of npl = 6 n_jobs)
    __nv_bfloat16 *whi = nullptr, *wlo = nullptr;
    if (WB == 2) {
        __nv_bfloat16 *planes = static_cast<__nv_bfloat16 *>(e.wbar_bf16);
        whi = planes + (long long)jl * 6 * o3;
        wlo = planes + ((long long)6 * w.n_jobs + (long long)jl * 6) * o3;
    }
    BlockIter cur, nxt;
    OrbitBlocks ob_cur, ob_nxt, ob_prev;
    ob_cur.set(cur);
    issue_stage(cur, ob_cur, S, o3, o, bufG(0), bufA(0), bufB(0), e.vvoo_f, e.t2_f, vv_off, tt_off, tid, with_fvo,
                lbar);
    cp_async_commit();
    int loc[3];
    loc_of<T, 256>(tid, loc);   // 16 warps: warp w covers a 2x4x4 sub-cube
    for (int bo = 0; bo < nbo; ++bo) {
        const int bi = bo & 1;
        cp_async_wait_all();
        __syncthreads();  // stage bo landed for every thread; buffer bi^1 is free
        if (WB == 1 && vjp && bo > 0) flush_wbar(ob_prev, bufG(bi ^ 1), S, o3, o, tid);
        if (lno && bo > 0) flush_wbar(ob_prev, bufG(bi ^ 1), S, o3, o, tid, 2);
        if (WB == 2 && vjp && bo > 0) flush_wbar_bf16(ob_prev, bufG(bi ^ 1), whi, wlo, o3, o, tid);
        if (vjp && bo > 0) flush_ybar(ob_prev, bufY(bi ^ 1), S + 6 * o3, o, tid);
        if (WB == 2 && vjp && bo > 0) __syncthreads();   // bf16 pieces span two refill pieces
        if (bo + 1 < nbo) {
            nxt = cur;
            nxt.next();
            ob_nxt.set(nxt);
            issue_stage(nxt, ob_nxt, S, o3, o, bufG(bi ^ 1), bufA(bi ^ 1), bufB(bi ^ 1), e.vvoo_f, e.t2_f, vv_off,
                        tt_off, tid, with_fvo, lbar);
            cp_async_commit();
        }
        float *G = bufG(bi);
        // W-bar into the staged G tiles (TF32) or straight to the float slots
        // (BF16x3); mo_energy-bar partials reduced in the warp
        double tmp = 0.0;
        if (lbar)
            orbit_lno_bar<float, T, TP, BLK, (WB == 1 ? 1 : 0), true, true, true>(
                loc, cur.I, cur.J, cur.K, ob_cur.dmap, G, eocc, tmp_s, bufY(bi), o, eabc, eb, vir_acc, &tmp);
        else
            orbit_element<float, float, float, T, TP, BLK, (WB == 1 ? 1 : 0), !STAGED, true, true, true>(
                loc, cur.I, cur.J, cur.K, ob_cur.dmap, G, bufA(bi), bufB(bi), Us, Ws, eocc, tmp_s, bufY(bi), o, fac,
                eabc, eb, vjp, eacc, vir_acc, with_fvo, S, &tmp, lno);
        if (vjp) {
            // lane bits: 0-1 -> loc[2], 2-3 -> loc[1], 4 -> loc[0] (low bits; loc_of)
            const int lane = tid & 31;
            double s0 = tmp, s1 = tmp, s2 = tmp;
#pragma unroll
            for (int m = 1; m <= 8; m <<= 1) s0 += __shfl_xor_sync(0xffffffffu, s0, m);
            s1 += __shfl_xor_sync(0xffffffffu, s1, 1);
            s1 += __shfl_xor_sync(0xffffffffu, s1, 2);
            s1 += __shfl_xor_sync(0xffffffffu, s1, 16);
            s2 += __shfl_xor_sync(0xffffffffu, s2, 4);
            s2 += __shfl_xor_sync(0xffffffffu, s2, 8);
            s2 += __shfl_xor_sync(0xffffffffu, s2, 16);
            if ((lane & 15) == 0) atomicAdd(&occ_acc[cur.I * T + loc[0]], -s0);
            if ((lane & 19) == 0) atomicAdd(&occ_acc[cur.J * T + loc[1]], -s1);
            if ((lane & 28) == 0) atomicAdd(&occ_acc[cur.K * T + loc[2]], -s2);
        }
        ob_prev = ob_cur;
        cur = nxt;
        ob_cur = ob_nxt;
    }
    // job energy (Neumaier pairs) and the virtual mo_energy-bar partial: a
    // fixed shuffle tree in each warp, then over the 16 warp results, so the
    // sum is deterministic and no thread sums the block serially
    __shared__ double wred[3][NTHR / 32];
    const int lane = tid & 31, warp = tid >> 5;
    double es = eacc.s, ec = eacc.c, vt = vir_acc;
    warp_ksum(es, ec, vt, 16);
    if (lane == 0) { wred[0][warp] = es; wred[1][warp] = ec; wred[2][warp] = vt; }
    __syncthreads();  // also orders every warp's occ_acc atomics and W-bar tiles before the flushes below
    if (WB == 1 && vjp) flush_wbar(ob_prev, bufG((nbo - 1) & 1), S, o3, o, tid);
    if (lno) flush_wbar(ob_prev, bufG((nbo - 1) & 1), S, o3, o, tid, 2);
    if (WB == 2 && vjp) flush_wbar_bf16(ob_prev, bufG((nbo - 1) & 1), whi, wlo, o3, o, tid);
    if (vjp) flush_ybar(ob_prev, bufY((nbo - 1) & 1), S + 6 * o3, o, tid);
    if (warp == 0) {
        const bool in = lane < NTHR / 32;
        es = in ? wred[0][lane] : 0.0;
        ec = in ? wred[1][lane] : 0.0;
        vt = in ? wred[2][lane] : 0.0;
        warp_ksum(es, ec, vt, NTHR / 64);
        if (lane == 0) {
            const long long amaj = (long long)a * (a + 1) * (a + 2) / 6 + (long long)b * (b + 1) / 2 + c;
            if (!lbar) e.job_e[amaj] = 2.0 * (es + ec);   // LNO: the projection kernel's energy stands
            if (vjp) {
                atomicAdd(&e.mo_energy_bar[o + a], vt);
                atomicAdd(&e.mo_energy_bar[o + b], vt);
                atomicAdd(&e.mo_energy_bar[o + c], vt);
            }
        }
    }
    if (vjp)
        for (int i = tid; i < o; i += NTHR) atomicAdd(&e.mo_energy_bar[i], occ_acc[i]);
}

template <int WB>
static cudaError_t launch(const WaveView &w, const EpiArgs &e, float *scratch, cudaStream_t st) {
    {
        cudaError_t ce = smem_optin(reinterpret_cast<const void *>(epi_pipe_kernel<WB>), (int)Smem::bytes);
        if (ce != cudaSuccess) return ce;
    }
    epi_pipe_kernel<WB><<<w.n_jobs, NTHR, Smem::bytes, st>>>(w, e, scratch);
    return cudaGetLastError();
}

}  // namespace epipipe

// float path: W-bar rounded to tf32 in place (TF32) or to bf16 hi/lo planes (BF16x3)
cudaError_t f32_epilogue(const WaveView &w, const EpiArgs &e, float *scratch, cudaStream_t st) {
    if (w.n_jobs <= 0) return cudaSuccess;
    if (e.o % epipipe::T != 0 || e.o > 64 || !e.vvoo_f || !e.t2_f) return cudaErrorInvalidValue;
    if (e.wbar_bf16) return epipipe::launch<2>(w, e, scratch, st);
    return epipipe::launch<1>(w, e, scratch, st);
}

}  // namespace ctb
