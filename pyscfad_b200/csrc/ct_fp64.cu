// Float64 path of the B200 CCSD(T) energy + VJP.
//
// Per wave of sorted jobs (a>=b>=c) the host runs:
//   F1  G_sigma[p,qr]   = sum_f vvop[x,y,p,o+f] t2T[z,f,qr]        (get_wv dgemm 1, ccsd_t.c:137-139)
//   F2  G_sigma[pq,r]  -= sum_l vooo[x,pq,l] t2T[z,y,l,r]           (get_wv dgemm 2, ccsd_t.c:140-142)
//   EPI orbit epilogue: W, V, r3, D, energy, zbar/d3bar/wbar/vbar, mo_energy_bar
//                                                                   (ccsd_t_vjp.c:9-117, lno_ccsd_t.c:6-29)
//   VT  V-term bars of t1T, fvo, vvop[:,:,:,:o], t2T                (ccsd_t_vjp.c:171-246 gemv parts)
//   VB  vvop_bar[x,y,p,o+f] += sum_qr t2T[z,f,qr] Wbar_sigma[p,qr]  (get_vvov_bar, :139-152)
//   TB  t2T_bar[z,f,qr]     += sum_{terms with z} vvop[x,y,p,o+f] Wbar[p,qr]  (get_t2T_bar dgemm 1)
//   OB1 vooo_bar[x,pq,l]    -= sum_r t2T[z,y,l,r] Wbar[pq,r]        (get_vooo_bar, :154-169)
//   OB2 t2T_bar[z,y,l,r]    -= sum_pq vooo[x,pq,l] Wbar[pq,r]       (get_t2T_bar dgemm 2)
// The GEMMs run on the float64 tensor pipe (DMMA, mma.sync m8n8k4 .f64).
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cstdio>
#include "ct_common.cuh"
#include "ct_internal.h"
#include "ct_epi.cuh"

namespace ctb {

enum OutMode { OUT_STORE = 0, OUT_ADD = 1, OUT_ATOMIC = 2 };

struct GemmParams {
    const double *A, *B;
    double *C;
    long long sAm, sAk, sBn, sBk, sCm, sCn;
    int M, N, K;
    double alpha;
    int o, v, n;
    const int *jobs;
    const int *tb_entries;
    const int *tb_groups;
};

template <int KIND> struct KindTraits;
template <> struct KindTraits<K_F1>  { static constexpr bool A_MC = true,  B_NC = false; static constexpr int OUT = OUT_STORE; };
template <> struct KindTraits<K_F2>  { static constexpr bool A_MC = false, B_NC = true;  static constexpr int OUT = OUT_ADD; };
template <> struct KindTraits<K_VB>  { static constexpr bool A_MC = false, B_NC = false; static constexpr int OUT = OUT_ATOMIC; };
template <> struct KindTraits<K_TB>  { static constexpr bool A_MC = true,  B_NC = true;  static constexpr int OUT = OUT_ATOMIC; };
template <> struct KindTraits<K_OB1> { static constexpr bool A_MC = false, B_NC = false; static constexpr int OUT = OUT_ATOMIC; };
template <> struct KindTraits<K_OB2> { static constexpr bool A_MC = true,  B_NC = true;  static constexpr int OUT = OUT_ATOMIC; };

// element offsets of A, B and C for term id e = jl*6 + sigma of the wave
template <int KIND>
__device__ __forceinline__ void entry_offsets(const GemmParams &p, int e, long long &ao, long long &bo,
                                              long long &co) {
    const int jl = e / 6, sg = e - 6 * (e / 6);
    int a, b, c, x, y, z;
    unpack_job(p.jobs[jl], a, b, c);
    term_xyz(sg, a, b, c, x, y, z);
    const long long o = p.o, v = p.v, n = p.n, o2 = o * o, o3 = o2 * o;
    const long long slot = ((long long)jl * kSlots + sg) * o3;
    const long long vv_row = ((long long)(x * v + y) * o) * n + o;
    switch (KIND) {
    case K_F1:  ao = z * v * o2;       bo = vv_row;             co = slot; break;
    case K_F2:  ao = x * o3;           bo = (z * v + y) * o2;   co = slot; break;
    case K_VB:  ao = z * v * o2;       bo = slot;               co = vv_row; break;
    case K_TB:  ao = vv_row;           bo = slot;               co = z * v * o2; break;
    case K_OB1: ao = slot;             bo = (z * v + y) * o2;   co = x * o3; break;
    default:    ao = x * o3;           bo = slot;               co = (z * v + y) * o2; break;
    }
}

// C[m,n] (op)= alpha * sum_{entries} sum_k A_e[m,k] B_e[n,k]; CTA tile 64 x BN x 16,
// 4 warps of 32 x BN/2, double-buffered shared memory with register prefetch.
template <int BN, int KIND>
__global__ void __launch_bounds__(128) gemm_f64_kernel(const GemmParams p) {
    using T = KindTraits<KIND>;
    constexpr int BM = 64, BK = 16;
    constexpr int A_LD = T::A_MC ? (BM + 8) : (BK + 4);
    constexpr int A_SZ = T::A_MC ? BK * A_LD : BM * A_LD;
    constexpr int B_LD = T::B_NC ? (BN + 8) : (BK + 4);
    constexpr int B_SZ = T::B_NC ? BK * B_LD : BN * B_LD;
    constexpr int NT = BN / 16;
    constexpr int BPT = BN * BK / 128;
    __shared__ double As[2][A_SZ];
    __shared__ double Bs[2][B_SZ];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp & 1, wn = warp >> 1;
    const int tiles_n = (p.N + BN - 1) / BN;
    const int tm = blockIdx.y / tiles_n, tn = blockIdx.y - tm * tiles_n;
    const int m0 = tm * BM, n0 = tn * BN;

    int e_begin, e_end;
    long long coff = 0;
    if (KIND == K_TB) {
        const int z = p.tb_groups[3 * blockIdx.x];
        e_begin = p.tb_groups[3 * blockIdx.x + 1];
        e_end = p.tb_groups[3 * blockIdx.x + 2];
        coff = (long long)z * p.v * p.o * p.o;
    } else {
        e_begin = blockIdx.x;
        e_end = blockIdx.x + 1;
    }
    const int kt_per = (p.K + BK - 1) / BK;
    const int ntiles = (e_end - e_begin) * kt_per;

    double acc[4][NT][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < NT; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

    double ra[8], rb[BPT];
    int cur_e = -1;
    const double *Ae = nullptr, *Be = nullptr;

    auto load_tile = [&](int t) {
        const int e = e_begin + t / kt_per;
        const int k0 = (t - (t / kt_per) * kt_per) * BK;
        if (e != cur_e) {
            cur_e = e;
            const int eid = (KIND == K_TB) ? p.tb_entries[e] : e;
            long long ao, bo, co;
            entry_offsets<KIND>(p, eid, ao, bo, co);
            Ae = p.A + ao;
            Be = p.B + bo;
            if (KIND != K_TB) coff = co;
        }
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int idx = tid + i * 128;
            int m, k;
            if (T::A_MC) { k = idx >> 6; m = idx & 63; } else { m = idx >> 4; k = idx & 15; }
            const int gm = m0 + m, gk = k0 + k;
            ra[i] = (gm < p.M && gk < p.K) ? __ldg(Ae + gm * p.sAm + gk * p.sAk) : 0.0;
        }
#pragma unroll
        for (int i = 0; i < BPT; ++i) {
            const int idx = tid + i * 128;
            int nn, k;
            if (T::B_NC) { k = idx / BN; nn = idx - k * BN; } else { nn = idx >> 4; k = idx & 15; }
            const int gn = n0 + nn, gk = k0 + k;
            rb[i] = (gn < p.N && gk < p.K) ? __ldg(Be + gn * p.sBn + gk * p.sBk) : 0.0;
        }
    };
    auto store_tile = [&](int buf) {
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int idx = tid + i * 128;
            if (T::A_MC) { const int k = idx >> 6, m = idx & 63; As[buf][k * A_LD + m] = ra[i]; }
            else { const int m = idx >> 4, k = idx & 15; As[buf][m * A_LD + k] = ra[i]; }
        }
#pragma unroll
        for (int i = 0; i < BPT; ++i) {
            const int idx = tid + i * 128;
            if (T::B_NC) { const int k = idx / BN, nn = idx - k * BN; Bs[buf][k * B_LD + nn] = rb[i]; }
            else { const int nn = idx >> 4, k = idx & 15; Bs[buf][nn * B_LD + k] = rb[i]; }
        }
    };

    if (ntiles > 0) {
        load_tile(0);
        store_tile(0);
        __syncthreads();
        for (int t = 0; t < ntiles; ++t) {
            const int buf = t & 1;
            if (t + 1 < ntiles) load_tile(t + 1);
#pragma unroll
            for (int ks = 0; ks < 4; ++ks) {
                double af[4], bf[NT];
                const int kk = ks * 4 + (lane & 3);
#pragma unroll
                for (int mt = 0; mt < 4; ++mt) {
                    const int m = wm * 32 + mt * 8 + (lane >> 2);
                    af[mt] = T::A_MC ? As[buf][kk * A_LD + m] : As[buf][m * A_LD + kk];
                }
#pragma unroll
                for (int nt = 0; nt < NT; ++nt) {
                    const int nn = wn * (BN / 2) + nt * 8 + (lane >> 2);
                    bf[nt] = T::B_NC ? Bs[buf][kk * B_LD + nn] : Bs[buf][nn * B_LD + kk];
                }
#pragma unroll
                for (int mt = 0; mt < 4; ++mt)
#pragma unroll
                    for (int nt = 0; nt < NT; ++nt) dmma(acc[mt][nt], af[mt], bf[nt]);
            }
            if (t + 1 < ntiles) store_tile(buf ^ 1);
            __syncthreads();
        }
    }

    double *C = p.C + coff;
#pragma unroll
    for (int mt = 0; mt < 4; ++mt) {
        const int m = m0 + wm * 32 + mt * 8 + (lane >> 2);
        if (m >= p.M) continue;
#pragma unroll
        for (int nt = 0; nt < NT; ++nt)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int nn = n0 + wn * (BN / 2) + nt * 8 + (lane & 3) * 2 + h;
                if (nn >= p.N) continue;
                double *c = C + m * p.sCm + nn * p.sCn;
                const double val = p.alpha * acc[mt][nt][h];
                if (T::OUT == OUT_STORE) *c = val;
                else if (T::OUT == OUT_ADD) *c += val;
                else atomicAdd(c, val);
            }
    }
}

template <int KIND>
static cudaError_t launch_kind(const GemmParams &p, int groups, cudaStream_t st) {
    const int bn = p.N <= 16 ? 16 : (p.N <= 32 ? 32 : (p.N <= 48 ? 48 : 64));
    const int tiles = ((p.M + 63) / 64) * ((p.N + bn - 1) / bn);
    if (groups <= 0) return cudaSuccess;
    if (tiles > 65535) return cudaErrorInvalidConfiguration;
    dim3 grid(groups, tiles);
    switch (bn) {
    case 16: gemm_f64_kernel<16, KIND><<<grid, 128, 0, st>>>(p); break;
    case 32: gemm_f64_kernel<32, KIND><<<grid, 128, 0, st>>>(p); break;
    case 48: gemm_f64_kernel<48, KIND><<<grid, 128, 0, st>>>(p); break;
    default: gemm_f64_kernel<64, KIND><<<grid, 128, 0, st>>>(p); break;
    }
    return cudaGetLastError();
}

cudaError_t f64_gemm(GemmKind kind, const WaveView &w, const double *A, const double *B, double *C,
                     double *scratch, cudaStream_t st) {
    (void)scratch;
    GemmParams p{};
    p.A = A; p.B = B; p.C = C;
    p.o = w.o; p.v = w.v; p.n = w.n;
    p.jobs = w.jobs; p.tb_entries = w.tb_entries; p.tb_groups = w.tb_groups;
    const long long o = w.o, v = w.v, n = w.n, o2 = o * o;
    const int terms = w.n_jobs * 6;
    switch (kind) {
    case K_F1:
        p.sAm = 1; p.sAk = o2; p.sBn = n; p.sBk = 1; p.sCm = 1; p.sCn = o2;
        p.M = (int)o2; p.N = (int)o; p.K = (int)v; p.alpha = 1.0;
        return launch_kind<K_F1>(p, terms, st);
    case K_F2:
        p.sAm = o; p.sAk = 1; p.sBn = 1; p.sBk = o; p.sCm = o; p.sCn = 1;
        p.M = (int)o2; p.N = (int)o; p.K = (int)o; p.alpha = -1.0;
        return launch_kind<K_F2>(p, terms, st);
    case K_VB:
        p.sAm = o2; p.sAk = 1; p.sBn = o2; p.sBk = 1; p.sCm = 1; p.sCn = n;
        p.M = (int)v; p.N = (int)o; p.K = (int)o2; p.alpha = 1.0;
        return launch_kind<K_VB>(p, terms, st);
    case K_TB:
        p.sAm = 1; p.sAk = n; p.sBn = 1; p.sBk = o2; p.sCm = o2; p.sCn = 1;
        p.M = (int)v; p.N = (int)o2; p.K = (int)o; p.alpha = 1.0;
        return launch_kind<K_TB>(p, w.n_tb_groups, st);
    case K_OB1:
        p.sAm = o; p.sAk = 1; p.sBn = o; p.sBk = 1; p.sCm = o; p.sCn = 1;
        p.M = (int)o2; p.N = (int)o; p.K = (int)o; p.alpha = -1.0;
        return launch_kind<K_OB1>(p, terms, st);
    default:
        p.sAm = 1; p.sAk = o; p.sBn = 1; p.sBk = o; p.sCm = o; p.sCn = 1;
        p.M = (int)o; p.N = (int)o; p.K = (int)o2; p.alpha = -1.0;
        return launch_kind<K_OB2>(p, terms, st);
    }
}

// ---------------------------------------------------------------------------
// Orbit epilogue, tiled.  One CTA per job.  The occupied cube is cut into
// T^3 blocks; a block-orbit is a sorted block triple I>=J>=K together with
// its (up to 6) permuted blocks.  For each block-orbit the CTA stages, with
// coalesced T-element rows, the permuted blocks of all six G slots and the
// V-term tiles in shared memory; each thread then owns whole element orbits
// {perm(i,j,k)}, so W, V, r3, the denominator and the backward quantities
// never leave registers; W-bar is written back block by block and ybar
// straight to its slot.
// ---------------------------------------------------------------------------
template <typename ST, int T, typename VT>
struct EpiSmem {
    static constexpr int T3 = T * T * T, T2 = T * T;
    // tile layout: element (u, w, t) of a staged block at u*TP + w*T + t.  For
    // T = 8 each u-plane is padded by 4 elements, which (with the thread
    // mapping of loc_of) keeps the six permuted access patterns of a warp at
    // most 2-way bank-conflicted.
    static constexpr int TP = T2 + (T == 8 ? 4 : 0), BLK = T * TP;
    static constexpr size_t g_off = 0;                                       // ST[6][6][BLK]
    static constexpr size_t va_off = g_off + sizeof(ST) * 36 * BLK;          // VT[6][6][T2]
    static constexpr size_t vb_off = va_off + sizeof(VT) * 36 * T2;          // VT[6][6][T2]
    static constexpr size_t u_off = vb_off + sizeof(VT) * 36 * T2;           // VT[6][64]
    static constexpr size_t w_off = u_off + sizeof(VT) * 6 * 64;             // VT[6][64]
    static constexpr size_t occ_off = w_off + sizeof(VT) * 6 * 64;           // double[64]
    static constexpr size_t eocc_off = occ_off + sizeof(double) * 64;        // double[64]
    static constexpr size_t tmp_off = eocc_off + sizeof(double) * 64;        // double[T3]
    static size_t bytes(int nthr) {
        (void)nthr;  // the final reduction reuses the G-tile area
        return tmp_off + sizeof(double) * T3;
    }
    __device__ static int pidx(int e3) { return (e3 / T2) * TP + e3 % T2; }
};

// T3M: the iterative (T) seed build (orbit_t3), a separate instance so the
// other modes keep their register allocation
template <typename ST, int T, typename VT, int NTHR, int WB, bool T3M = false>
__global__ void __launch_bounds__(NTHR, (NTHR >= 256 ? 2 : 4)) epi_kernel(const WaveView w, const EpiArgs e, ST *scratch) {
    using L = EpiSmem<ST, T, VT>;
    constexpr int T3 = L::T3, T2 = L::T2, TP = L::TP, BLK = L::BLK;
    extern __shared__ __align__(16) uint8_t esm[];
    ST *Gs = reinterpret_cast<ST *>(esm + L::g_off);
    VT *VA = reinterpret_cast<VT *>(esm + L::va_off);
    VT *VB = reinterpret_cast<VT *>(esm + L::vb_off);
    VT *Us = reinterpret_cast<VT *>(esm + L::u_off);
    VT *Ws = reinterpret_cast<VT *>(esm + L::w_off);
    double *occ_acc = reinterpret_cast<double *>(esm + L::occ_off);
    double *tmp_s = reinterpret_cast<double *>(esm + L::tmp_off);
    double *eocc = reinterpret_cast<double *>(esm + L::eocc_off);
    double *red = reinterpret_cast<double *>(esm + L::g_off);  // used after the last block-orbit
    static_assert(sizeof(ST) * 36 * BLK >= sizeof(double) * 3 * NTHR, "reduction area");

    const int o = e.o, v = e.v, n = e.n;
    const long long o3 = (long long)o * o * o;
    const int jl = blockIdx.x, tid = threadIdx.x;
    int a, b, c;
    unpack_job(w.jobs[jl], a, b, c);
    const double fac = job_fac(a, b, c);
    const double eabc = e.mo_energy[o + a] + e.mo_energy[o + b] + e.mo_energy[o + c];
    ST *S = scratch + (long long)jl * kSlots * o3;
    const bool vjp = e.with_vjp != 0;
    const bool lno = e.lno_phase == 1 && !vjp;    // LNO forward: W and z/D cubes
    const bool lbar = e.lno_phase == 2 && vjp;    // LNO backward pass
    const bool t3m = T3M && !vjp;                 // iterative (T) seed: 6-D arrays

    // per-term offsets of the V-term operand rows vvop[x,y] and t2T[y,x]
    // (shared memory: read with a runtime term index, no local-memory array)
    __shared__ long long vv_off[6], tt_off[6];
    if (tid < 6) {
        int x, y, z;
        term_xyz(tid, a, b, c, x, y, z);
        vv_off[tid] = ((long long)(x * v + y) * o) * n;
        tt_off[tid] = ((long long)(y * v + x) * o) * o;
    }
    for (int i = tid; i < o; i += NTHR) { occ_acc[i] = 0.0; eocc[i] = e.mo_energy[i]; }
    for (int i = tid; i < 6 * o; i += NTHR) {
        const int sg = i / o, r = i - sg * o;
        int x, y, z;
        term_xyz(sg, a, b, c, x, y, z);
        Us[sg * 64 + r] = (VT)e.t1T[z * o + r];
        Ws[sg * 64 + r] = (VT)e.fvo[z * o + r];
    }

    KSum eacc;
    double vir_acc = 0.0;
    const double eb = e.et_bar;
    const int nb = (o + T - 1) / T;
    int BI = 0, BJ = 0, BK = 0;
    const int nbo = nb * (nb + 1) * (nb + 2) / 6;
    for (int bo = 0; bo < nbo; ++bo) {
        if (bo > 0) {  // next sorted block triple (I >= J >= K), K fastest
            if (BK < BJ) ++BK;
            else if (BJ < BI) { ++BJ; BK = 0; }
            else { ++BI; BJ = 0; BK = 0; }
        }
        const int blk[3] = {BI, BJ, BK};
        // permuted blocks of the orbit; dmap[s]: staging buffer of slot s's block,
        // fresh[s]: slot s is the first with that block (all indices compile-time)
        int bs[6][3], dmap[6], nd = 0;
        bool fresh[6];
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
        __syncthreads();  // previous block-orbit fully written back
        // stage G blocks of the six slots (T-element rows, full-row vector loads)
        const bool full = (BI + 1) * T <= o;  // every block of this orbit lies inside the cube
#pragma unroll
        for (int s = 0; s < 6; ++s) {
            if (!fresh[s]) continue;
            const int d = dmap[s];
            const int p0 = bs[s][0] * T, q0 = bs[s][1] * T, r0 = bs[s][2] * T;
            // LNO backward: the z/D cube and the two parts of A and B (slots 1-5)
            // into tile groups 0-4
            for (int sg = 0; sg < (lbar ? 5 : 6); ++sg) {
                const ST *src = S + (sg + (lbar ? 1 : 0)) * o3;
                ST *dst = Gs + (sg * 6 + d) * BLK;
                if (full && sizeof(ST) * T % 16 == 0 && (sizeof(ST) * o) % 16 == 0) {
                    constexpr int VEC = 16 / sizeof(ST), NV = T3 / VEC;
                    for (int i = tid; i < NV; i += NTHR) {
                        const int e3 = i * VEC;
                        const int u = e3 / T2, ww = (e3 / T) % T, t = e3 % T;
                        cp_async16(dst + L::pidx(e3), src + ((long long)(p0 + u) * o + q0 + ww) * o + r0 + t);
                    }
                } else {
                    for (int e3 = tid; e3 < T3; e3 += NTHR) {
                        const int p = p0 + e3 / T2, q = q0 + (e3 / T) % T, r = r0 + e3 % T;
                        dst[L::pidx(e3)] = (p < o && q < o && r < o) ? src[((long long)p * o + q) * o + r] : ST(0);
                    }
                }
            }
        }
        // stage V-term tiles: A = vvop[x,y,P,Q], B = t2T[y,x,P,Q] on the block pair of each
        // slot; all loads of a thread are issued before its shared-memory stores
        if (!lbar) {
            constexpr int NV = (36 * T2 + NTHR - 1) / NTHR;
            double la[NV], lb[NV];
#pragma unroll
            for (int k = 0; k < NV; ++k) {
                const int idx = tid + k * NTHR;
                la[k] = lb[k] = 0.0;
                if (idx < 36 * T2) {
                    const int sg = idx / (6 * T2), cc = (idx / T2) % 6, uw = idx % T2;
                    // blocks of slot cc's first two axes: blk[kR(cc,0)], blk[kR(cc,1)]
                    constexpr unsigned int KR01 = (0u | 1u << 2) | (0u | 2u << 2) << 4 | (1u | 0u << 2) << 8 |
                                                  (1u | 2u << 2) << 12 | (2u | 0u << 2) << 16 | (2u | 1u << 2) << 20;
                    const int k0 = (KR01 >> (4 * cc)) & 3, k1 = (KR01 >> (4 * cc + 2)) & 3;
                    const int P = (k0 == 0 ? BI : (k0 == 1 ? BJ : BK)) * T + uw / T;
                    const int Q = (k1 == 0 ? BI : (k1 == 1 ? BJ : BK)) * T + uw % T;
                    if (P < o && Q < o) {
                        la[k] = __ldg(e.vvop + vv_off[sg] + (long long)P * n + Q);
                        lb[k] = __ldg(e.t2T + tt_off[sg] + (long long)P * o + Q);
                    }
                }
            }
#pragma unroll
            for (int k = 0; k < NV; ++k) {
                const int idx = tid + k * NTHR;
                if (idx < 36 * T2) {
                    VA[idx] = (VT)la[k];
                    VB[idx] = (VT)lb[k];
                }
            }
        }
        cp_async_wait_all();
        __syncthreads();
        for (int q = tid; q < T3; q += NTHR) {
            int loc[3];
            loc_of<T, NTHR>(q, loc);
            if (lbar)
                orbit_lno_bar<ST, T, TP, BLK>(loc, BI, BJ, BK, dmap, Gs, eocc, tmp_s, S + 6 * o3, o, eabc, eb,
                                              vir_acc);
            else if (t3m)
                orbit_t3<ST, VT, T, TP, BLK>(loc, BI, BJ, BK, dmap, Gs, VA, VB, Us, Ws, eocc, o, v, eabc, a, b, c,
                                             e.t3_c, e.t3_x);
            else
                orbit_element<double, ST, VT, T, TP, BLK, WB>(loc, BI, BJ, BK, dmap, Gs, VA, VB, Us, Ws, eocc, tmp_s,
                                                              S + 6 * o3, o, fac, eabc, eb, vjp, eacc, vir_acc, true,
                                                              nullptr, nullptr, lno);
        }
        if (vjp || lno) {
            __syncthreads();
            // occupied-energy bar: orbit partials summed per block row (no contended atomics)
            if (vjp && tid < 3 * T) {
                const int axis = tid / T, u = tid % T;
                const int gi = blk[axis] * T + u;
                double acc = 0.0;
                for (int r2 = 0; r2 < T2; ++r2) {
                    const int qq = axis == 0 ? u * T2 + r2 : (axis == 1 ? (r2 / T) * T2 + u * T + r2 % T
                                                                      : r2 * T + u);
                    acc += tmp_s[qq];
                }
                if (gi < o) atomicAdd(&occ_acc[gi], -acc);
            }
#pragma unroll
            for (int s = 0; s < 6; ++s) {
                if (!fresh[s]) continue;
                const int d = dmap[s];
                const int p0 = bs[s][0] * T, q0 = bs[s][1] * T, r0 = bs[s][2] * T;
                for (int sg = 0; sg < (vjp ? 6 : 2); ++sg) {   // LNO: the W and z/D cubes only
                    ST *dstg = S + sg * o3;
                    const ST *srcs = Gs + (sg * 6 + d) * BLK;
                    if (full && sizeof(ST) * T % 16 == 0 && (sizeof(ST) * o) % 16 == 0) {
                        constexpr int VEC = 16 / sizeof(ST), NV = T3 / VEC;
                        for (int i = tid; i < NV; i += NTHR) {
                            const int e3 = i * VEC;
                            const int u = e3 / T2, ww = (e3 / T) % T, t = e3 % T;
                            *reinterpret_cast<float4 *>(dstg + ((long long)(p0 + u) * o + q0 + ww) * o + r0 + t) =
                                *reinterpret_cast<const float4 *>(srcs + L::pidx(e3));
                        }
                    } else {
                        for (int e3 = tid; e3 < T3; e3 += NTHR) {
                            const int p = p0 + e3 / T2, q = q0 + (e3 / T) % T, r = r0 + e3 % T;
                            if (p < o && q < o && r < o) dstg[((long long)p * o + q) * o + r] = srcs[L::pidx(e3)];
                        }
                    }
                }
            }
        }
    }
    __syncthreads();  // last block-orbit done with the G tiles
    red[tid] = eacc.s;
    red[NTHR + tid] = eacc.c;
    red[2 * NTHR + tid] = vir_acc;
    __syncthreads();
    if (tid == 0) {
        KSum tot;
        double vt = 0.0;
        for (int t = 0; t < NTHR; ++t) {
            tot.add(red[t]);
            tot.add(red[NTHR + t]);
            vt += red[2 * NTHR + t];
        }
        const long long amaj = (long long)a * (a + 1) * (a + 2) / 6 + (long long)b * (b + 1) / 2 + c;
        if (!lbar) e.job_e[amaj] = 2.0 * tot.value();   // LNO: the projection kernel's energy stands
        if (vjp) {
            atomicAdd(&e.mo_energy_bar[o + a], vt);
            atomicAdd(&e.mo_energy_bar[o + b], vt);
            atomicAdd(&e.mo_energy_bar[o + c], vt);
        }
    }
    if (vjp)
        for (int i = tid; i < o; i += NTHR) atomicAdd(&e.mo_energy_bar[i], occ_acc[i]);
}

// V-term bars of one job.  With Vbar_sigma[p,q,r] = ybar[idx_sigma(p,q,r)]:
//   vvop_bar[x,y,p,q] += 1/2 sum_r Vbar t1T[z,r]     (get_vvoo_bar, ccsd_t_vjp.c:171-186)
//   t2T_bar[y,x,p,q]  += 1/2 sum_r Vbar fvo[z,r]     (get_t2T_bar gemv, :228-230)
//   t1T_bar[z,r]      += 1/2 sum_pq Vbar vvop[x,y,p,q]   (get_t1T_bar, :188-204)
//   fvo_bar[z,r]      += 1/2 sum_pq Vbar t2T[y,x,p,q]    (get_fvo_bar, :233-246)
// For each term the index r sits on one axis of ybar (two terms per axis), so
// the CTA makes one coalesced pass per axis: ybar contracted along that axis
// with the two terms' t1/fvo vectors, and along the other two with their
// vvop/t2T matrices.
__device__ __forceinline__ double ldg_st(const double *p) { return __ldg(p); }
__device__ __forceinline__ float ldg_st(const float *p) { return __ldg(p); }

struct VtTerm {
    int x, y, z, mp, mq;
};

__device__ __forceinline__ VtTerm vt_term(int sg, int a, int b, int c) {
    VtTerm t;
    term_xyz(sg, a, b, c, t.x, t.y, t.z);
    const int ri = kInv(sg);
    t.mp = kR(ri, 0) == 0 ? 0 : (kR(ri, 1) == 0 ? 1 : 2);
    t.mq = kR(ri, 0) == 1 ? 0 : (kR(ri, 1) == 1 ? 1 : 2);
    return t;
}

// One axis pass per CTA (blockIdx.x = 3 * job + axis).  The o^2 pairs of the
// two other axes are processed in chunks of VT_CH: the chunk's ybar values
// (all r) are staged in shared memory as Ys[r][pair]; then each thread
// contracts one pair along r with the two terms' t1/fvo rows (vvop-bar and
// t2T-bar updates), and 4 * o threads contract one r along the chunk's pairs
// with the terms' vvop/t2T values (t1T-bar / fvo-bar partials, kept in
// registers across chunks).  No warp shuffles.
constexpr int VT_CH = 256;

// QRT: ybar (slot 6) is qr-tiled (the mixed path's slot layout): element
// (i,j,k) at i o^2 + (j/8) 8o + (k/8) 64 + (j%8) 8 + k%8
template <typename ST, bool QRT>
__global__ void __launch_bounds__(VT_CH) vterm_kernel(const WaveView w, const EpiArgs e, const ST *scratch) {
    constexpr int NTHR = VT_CH, LD = VT_CH + 1;
    extern __shared__ __align__(16) uint8_t vsm[];
    ST *Ys = reinterpret_cast<ST *>(vsm);                                 // [o][LD]
    double *AB = reinterpret_cast<double *>(vsm + sizeof(ST) * 64 * LD);  // [4][VT_CH]: A_t0, A_t1, B_t0, B_t1
    double *UW = AB + 4 * VT_CH;                                         // [4][64]: u_t0, u_t1, w_t0, w_t1
    const int o = e.o, v = e.v, n = e.n, oo = o * o;
    const long long o3 = (long long)oo * o;
    const int jl = blockIdx.x / 3, ax = blockIdx.x - 3 * (blockIdx.x / 3), tid = threadIdx.x;
    int a, b, c;
    unpack_job(w.jobs[jl], a, b, c);
    const ST *Yb = scratch + ((long long)jl * kSlots + 6) * o3;
    // terms per axis of r: axis 0 -> sigma 3,5; axis 1 -> sigma 1,4; axis 2 -> sigma 0,2
    const int s0 = ax == 0 ? 3 : (ax == 1 ? 1 : 0), s1 = ax == 0 ? 5 : (ax == 1 ? 4 : 2);
    const VtTerm T0 = vt_term(s0, a, b, c), T1 = vt_term(s1, a, b, c);
    // coordinate m of pair (f0, f1) with r's axis set to 0, without indexed arrays
    auto coord = [&](int m, int f0, int f1) {
        const int c0 = ax == 0 ? 0 : f0, c1 = ax == 0 ? f0 : (ax == 1 ? 0 : f1), c2 = ax == 2 ? 0 : f1;
        return m == 0 ? c0 : (m == 1 ? c1 : c2);
    };
    const long long rstep = ax == 0 ? (long long)oo : (ax == 1 ? (long long)o : 1LL);
    // x / o by multiply-high with ceil(2^32 / o): exact for x < 2^32 / o^2 (x < o^2 * 4 here)
    const unsigned omag = (unsigned)(((1ull << 32) + o - 1) / o);
    auto divo = [&](int x) { return (int)__umulhi((unsigned)x, omag); };
    int fvo_nz = 0;
    for (int i = tid; i < 2 * o; i += NTHR) {
        const int t = i / o, r = i - t * o;
        const int z = t ? T1.z : T0.z;
        UW[t * 64 + r] = e.t1T[z * o + r];
        const double f = e.fvo[z * o + r];
        UW[(2 + t) * 64 + r] = f;
        fvo_nz |= (f != 0.0);
    }
    // with both terms' fvo rows zero the t2T-bar updates of this pass add zeros: skipped
    const bool with_fvo = __syncthreads_or(fvo_nz) != 0;
    // (r, q4) of this thread's r-contraction: q4 = 0,1 -> A of term 0,1; 2,3 -> B
    const int rr = tid % 64, q4 = tid / 64;
    const bool rowner = rr < o && q4 < 4;
    double racc = 0.0;
    for (int base = 0; base < oo; base += VT_CH) {
        const int cnt = min(VT_CH, oo - base);
        __syncthreads();  // previous chunk consumed
        // stage ybar: Ys[r][j] = ybar(pair base + j, r); consecutive threads take
        // consecutive memory (pairs for axes 0/1, r for axis 2)
        auto tile = [&](int j, int k) { return (j >> 3) * 8 * o + (k >> 3) * 64 + (j & 7) * 8 + (k & 7); };
        if (ax < 2) {
            if (tid < cnt) {
                const int pr = base + tid, f0 = divo(pr), f1 = pr - f0 * o;
                if (QRT) {
                    if (ax == 0) {
                        const ST *src = Yb + tile(f0, f1);
#pragma unroll 8
                        for (int r = 0; r < o; ++r) Ys[r * LD + tid] = src[(long long)r * oo];
                    } else {
                        const ST *src = Yb + (long long)f0 * oo;
#pragma unroll 8
                        for (int r = 0; r < o; ++r) Ys[r * LD + tid] = src[tile(r, f1)];
                    }
                } else {
                    const ST *src = Yb + (ax == 0 ? (long long)pr : (long long)f0 * oo + f1);
#pragma unroll 8
                    for (int r = 0; r < o; ++r) Ys[r * LD + tid] = src[r * rstep];
                }
            }
        } else {
            for (int i = tid; i < cnt * o; i += NTHR) {
                const int j = divo(i), r = i - j * o;
                if (QRT) {
                    const int pr = base + j, f0 = divo(pr), f1 = pr - f0 * o;
                    Ys[r * LD + j] = Yb[(long long)f0 * oo + tile(f1, r)];
                } else {
                    Ys[r * LD + j] = Yb[(long long)(base + j) * o + r];
                }
            }
        }
        // the chunk's vvop / t2T values of both terms at (P, Q) of each pair
        for (int i = tid; i < cnt * 2; i += NTHR) {
            const int t = i >= cnt ? 1 : 0, j = i - t * cnt;
            const int pr = base + j, f0 = divo(pr), f1 = pr - f0 * o;
            const int tx = t ? T1.x : T0.x, ty = t ? T1.y : T0.y;
            const int P = coord(t ? T1.mp : T0.mp, f0, f1), Q = coord(t ? T1.mq : T0.mq, f0, f1);
            AB[t * VT_CH + j] = e.vvop[((long long)(tx * v + ty) * o + P) * n + Q];
            AB[(2 + t) * VT_CH + j] = e.t2T[((long long)(ty * v + tx) * o + P) * o + Q];
        }
        __syncthreads();
        // pair contraction along r -> vvop-bar / t2T-bar
        if (tid < cnt) {
            double su0 = 0, su1 = 0, sw0 = 0, sw1 = 0;
            for (int r = 0; r < o; ++r) {
                const double val = (double)Ys[r * LD + tid];
                su0 += val * UW[r]; su1 += val * UW[64 + r];
                sw0 += val * UW[128 + r]; sw1 += val * UW[192 + r];
            }
            const int pr = base + tid, f0 = divo(pr), f1 = pr - f0 * o;
#pragma unroll
            for (int t = 0; t < 2; ++t) {
                const int tx = t ? T1.x : T0.x, ty = t ? T1.y : T0.y;
                const int P = coord(t ? T1.mp : T0.mp, f0, f1), Q = coord(t ? T1.mq : T0.mq, f0, f1);
                atomicAdd(e.vvop_bar + ((long long)(tx * v + ty) * o + P) * n + Q, 0.5 * (t ? su1 : su0));
                if (with_fvo) atomicAdd(e.t2T_bar + ((long long)(ty * v + tx) * o + P) * o + Q, 0.5 * (t ? sw1 : sw0));
            }
        }
        // r contraction along the chunk's pairs -> t1T-bar / fvo-bar partials
        // (four independent partial sums hide the add latency)
        if (rowner) {
            const ST *row = Ys + rr * LD;
            const double *vec = AB + q4 * VT_CH;
            double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
            int j = 0;
            for (; j + 4 <= cnt; j += 4) {
                a0 += (double)row[j] * vec[j];
                a1 += (double)row[j + 1] * vec[j + 1];
                a2 += (double)row[j + 2] * vec[j + 2];
                a3 += (double)row[j + 3] * vec[j + 3];
            }
            for (; j < cnt; ++j) a0 += (double)row[j] * vec[j];
            racc += (a0 + a1) + (a2 + a3);
        }
    }
    if (rowner) {
        const int z = (q4 & 1) ? T1.z : T0.z;
        double *dst = (q4 < 2 ? e.t1T_bar : e.fvo_bar) + z * o + rr;
        atomicAdd(dst, 0.5 * racc);
    }
}

template <typename ST>
static size_t vterm_smem() {
    return sizeof(ST) * 64 * (VT_CH + 1) + sizeof(double) * (4 * VT_CH + 4 * 64);
}

template <typename ST, bool QRT>
static cudaError_t launch_vterm(const WaveView &w, const EpiArgs &e, const ST *scratch, cudaStream_t st) {
    if (w.n_jobs <= 0) return cudaSuccess;
    if (e.o > 64) return cudaErrorInvalidValue;
    {
        cudaError_t ce = smem_optin(reinterpret_cast<const void *>(vterm_kernel<ST, QRT>), (int)vterm_smem<ST>());
        if (ce != cudaSuccess) return ce;
    }
    vterm_kernel<ST, QRT><<<w.n_jobs * 3, VT_CH, vterm_smem<ST>(), st>>>(w, e, scratch);
    return cudaGetLastError();
}

template <typename ST, int T, typename VT, int NTHR, int WB, bool T3M>
static cudaError_t launch_epi(const WaveView &w, const EpiArgs &e, ST *scratch, cudaStream_t st) {
    if (w.n_jobs <= 0) return cudaSuccess;
    if (e.o > 64) return cudaErrorInvalidValue;
    const size_t smem = EpiSmem<ST, T, VT>::bytes(NTHR);
    {
        cudaError_t ce = smem_optin(reinterpret_cast<const void *>(epi_kernel<ST, T, VT, NTHR, WB, T3M>), (int)smem);
        if (ce != cudaSuccess) return ce;
    }
    epi_kernel<ST, T, VT, NTHR, WB, T3M><<<w.n_jobs, NTHR, smem, st>>>(w, e, scratch);
    return cudaGetLastError();
}

cudaError_t f64_epilogue(const WaveView &w, const EpiArgs &e, double *scratch, cudaStream_t st) {
    if (e.t3_c) {
        if (!e.t3_x || e.with_vjp) return cudaErrorInvalidValue;
        return launch_epi<double, 4, double, 64, 0, true>(w, e, scratch, st);
    }
    return launch_epi<double, 4, double, 64, 0, false>(w, e, scratch, st);
}

cudaError_t f64_vterm(const WaveView &w, const EpiArgs &e, const double *scratch, cudaStream_t st) {
    return launch_vterm<double, false>(w, e, scratch, st);
}

// V-term bars of the mixed path (float ybar, qr-tiled slots): the same four
// contractions as vterm_kernel, one CTA per (job, axis), restructured for
// shared-memory throughput.  A chunk of 256 pairs (pair index f0*o + f1 of
// the two axes other than r's) is staged r-major as Ys[r][j] (row stride
// 260 floats: 16-byte rows, and 65 16-byte units per row so that 8 threads
// reading 8 consecutive rows hit 8 distinct bank groups): with 16-byte
// cp.async pieces of 4 pairs for axes 0 and 1 (4 consecutive f1 lie in one
// 8-run of the tiled slot), and through registers for axis 2, whose runs
// are along r.  Then
//   U: one thread per pair: sum_r Ys[r][j] * (t1_z0, t1_z1, fvo_z0, fvo_z1)[r]
//      (one float4 broadcast per r) -> vvop_bar / t2T_bar;
//   B: thread (r, quarter): sum over its 64 pairs of Ys[r][j..j+3] (float4)
//      times the pair's (vvop_t0, vvop_t1, t2T_t0, t2T_t1) (float4 broadcast),
//      float partials per chunk added into float64 -> t1T_bar / fvo_bar.
// Products and per-chunk sums are float (the ybar operand is float on this
// path), chunk sums and the output reductions float64.
constexpr int V2_NT = 256, V2_CH = 256, V2_LD = V2_CH + 4;

static size_t vterm2_smem(int o) {
    return sizeof(float) * (size_t)o * V2_LD + sizeof(float4) * (V2_CH + 64) + sizeof(double) * 4 * 4 * 64;
}

template <int AX>
__device__ __forceinline__ void vterm2_axis(const WaveView &w, const EpiArgs &e, const float *Yb, int a, int b,
                                            int c, uint8_t *sm) {
    const int o = e.o, v = e.v, n = e.n, oo = o * o, tid = threadIdx.x;
    float *Ys = reinterpret_cast<float *>(sm);                  // [o][V2_LD]
    float4 *AB = reinterpret_cast<float4 *>(Ys + o * V2_LD);     // [V2_CH]
    float4 *UW = AB + V2_CH;                                     // [64]
    double *Bq = reinterpret_cast<double *>(UW + 64);            // [4 quarters][4 combos][64]
    // terms per axis of r: axis 0 -> sigma 3,5; axis 1 -> sigma 1,4; axis 2 -> sigma 0,2
    constexpr int S0 = AX == 0 ? 3 : (AX == 1 ? 1 : 0), S1 = AX == 0 ? 5 : (AX == 1 ? 4 : 2);
    const VtTerm T0 = vt_term(S0, a, b, c), T1 = vt_term(S1, a, b, c);
    auto coord = [](int m, int f0, int f1) {
        const int c0 = AX == 0 ? 0 : f0, c1 = AX == 0 ? f0 : (AX == 1 ? 0 : f1), c2 = AX == 2 ? 0 : f1;
        return m == 0 ? c0 : (m == 1 ? c1 : c2);
    };
    auto tile = [o](int j, int k) { return (j >> 3) * 8 * o + (k >> 3) * 64 + (j & 7) * 8 + (k & 7); };
    const unsigned omag = (unsigned)(((1ull << 32) + o - 1) / o);
    auto divo = [omag](int x) { return (int)__umulhi((unsigned)x, omag); };
    int fvo_nz = 0;
    if (tid < o) {
        const int r = tid;
        const float f0 = (float)e.fvo[T0.z * o + r], f1 = (float)e.fvo[T1.z * o + r];
        UW[r] = make_float4((float)e.t1T[T0.z * o + r], (float)e.t1T[T1.z * o + r], f0, f1);
        fvo_nz = (e.fvo[T0.z * o + r] != 0.0) || (e.fvo[T1.z * o + r] != 0.0);
    }
    // with both terms' fvo rows zero the t2T-bar updates of this pass add zeros: skipped
    const bool with_fvo = __syncthreads_or(fvo_nz) != 0;
    const int br = tid & 63, qd = tid >> 6;   // B role: row r, quarter of the chunk's pairs
    double bacc0 = 0.0, bacc1 = 0.0, bacc2 = 0.0, bacc3 = 0.0;
    for (int base = 0; base < oo; base += V2_CH) {
        const int cnt = min(V2_CH, oo - base);   // a multiple of 4 (o % 8 == 0)
        __syncthreads();                         // previous chunk consumed
        if (AX != 2) {
            const int npc = cnt >> 2;
            for (int i = tid; i < o * npc; i += V2_NT) {
                const int r = i / npc, q4 = i - r * npc;
                const int pr = base + 4 * q4, f0 = divo(pr), f1 = pr - f0 * o;
                const float *src = AX == 0 ? Yb + (long long)r * oo + tile(f0, f1) : Yb + (long long)f0 * oo + tile(r, f1);
                cp_async16(Ys + r * V2_LD + 4 * q4, src);
            }
            cp_async_commit();
        } else if (tid < cnt) {
            const int pr = base + tid, f0 = divo(pr), f1 = pr - f0 * o;
            const float *src = Yb + (long long)f0 * oo + tile(f1, 0);
#pragma unroll 4
            for (int r0 = 0; r0 < o; r0 += 8) {
                const float4 y0 = __ldg(reinterpret_cast<const float4 *>(src + r0 * 8));
                const float4 y1 = __ldg(reinterpret_cast<const float4 *>(src + r0 * 8 + 4));
                float *d = Ys + r0 * V2_LD + tid;
                d[0] = y0.x; d[V2_LD] = y0.y; d[2 * V2_LD] = y0.z; d[3 * V2_LD] = y0.w;
                d[4 * V2_LD] = y1.x; d[5 * V2_LD] = y1.y; d[6 * V2_LD] = y1.z; d[7 * V2_LD] = y1.w;
            }
        }
        // the chunk's vvop / t2T values of both terms at (P, Q) of each pair
        if (tid < cnt) {
            const int pr = base + tid, f0 = divo(pr), f1 = pr - f0 * o;
            const int P0 = coord(T0.mp, f0, f1), Q0 = coord(T0.mq, f0, f1);
            const int P1 = coord(T1.mp, f0, f1), Q1 = coord(T1.mq, f0, f1);
            AB[tid] = make_float4((float)e.vvop[((long long)(T0.x * v + T0.y) * o + P0) * n + Q0],
                                  (float)e.vvop[((long long)(T1.x * v + T1.y) * o + P1) * n + Q1],
                                  (float)e.t2T[((long long)(T0.y * v + T0.x) * o + P0) * o + Q0],
                                  (float)e.t2T[((long long)(T1.y * v + T1.x) * o + P1) * o + Q1]);
        }
        if (AX != 2) cp_async_wait_all();
        __syncthreads();
        // U: pair contraction along r -> vvop-bar / t2T-bar
        if (tid < cnt) {
            float su0 = 0.f, su1 = 0.f, sw0 = 0.f, sw1 = 0.f;
#pragma unroll 8
            for (int r = 0; r < o; ++r) {
                const float y = Ys[r * V2_LD + tid];
                const float4 u = UW[r];
                su0 = fmaf(y, u.x, su0); su1 = fmaf(y, u.y, su1);
                sw0 = fmaf(y, u.z, sw0); sw1 = fmaf(y, u.w, sw1);
            }
            const int pr = base + tid, f0 = divo(pr), f1 = pr - f0 * o;
            const int P0 = coord(T0.mp, f0, f1), Q0 = coord(T0.mq, f0, f1);
            const int P1 = coord(T1.mp, f0, f1), Q1 = coord(T1.mq, f0, f1);
            atomicAdd(e.vvop_bar + ((long long)(T0.x * v + T0.y) * o + P0) * n + Q0, 0.5 * (double)su0);
            atomicAdd(e.vvop_bar + ((long long)(T1.x * v + T1.y) * o + P1) * n + Q1, 0.5 * (double)su1);
            if (with_fvo) {
                atomicAdd(e.t2T_bar + ((long long)(T0.y * v + T0.x) * o + P0) * o + Q0, 0.5 * (double)sw0);
                atomicAdd(e.t2T_bar + ((long long)(T1.y * v + T1.x) * o + P1) * o + Q1, 0.5 * (double)sw1);
            }
        }
        // B: r contraction along the quarter's pairs -> t1T-bar / fvo-bar partials
        if (br < o) {
            float p0 = 0.f, p1 = 0.f, p2 = 0.f, p3 = 0.f;
            const int j1 = min(qd * (V2_CH / 4) + V2_CH / 4, cnt);
            const float *row = Ys + br * V2_LD;
            for (int j = qd * (V2_CH / 4); j < j1; j += 4) {
                const float4 y4 = *reinterpret_cast<const float4 *>(row + j);
                const float yy[4] = {y4.x, y4.y, y4.z, y4.w};
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const float4 m = AB[j + u];
                    p0 = fmaf(yy[u], m.x, p0); p1 = fmaf(yy[u], m.y, p1);
                    p2 = fmaf(yy[u], m.z, p2); p3 = fmaf(yy[u], m.w, p3);
                }
            }
            bacc0 += p0; bacc1 += p1; bacc2 += p2; bacc3 += p3;
        }
    }
    if (br < o) {
        Bq[(qd * 4 + 0) * 64 + br] = bacc0;
        Bq[(qd * 4 + 1) * 64 + br] = bacc1;
        Bq[(qd * 4 + 2) * 64 + br] = bacc2;
        Bq[(qd * 4 + 3) * 64 + br] = bacc3;
    }
    __syncthreads();
    {
        // combo k = tid / 64: 0, 1 -> t1T-bar of term 0, 1; 2, 3 -> fvo-bar of term 0, 1
        const int k = tid >> 6, r = tid & 63;
        if (r < o) {
            const double s = Bq[k * 64 + r] + Bq[(4 + k) * 64 + r] + Bq[(8 + k) * 64 + r] + Bq[(12 + k) * 64 + r];
            const int z = (k & 1) ? T1.z : T0.z;
            atomicAdd((k < 2 ? e.t1T_bar : e.fvo_bar) + z * o + r, 0.5 * s);
        }
    }
}

__global__ void __launch_bounds__(V2_NT) vterm2_kernel(const WaveView w, const EpiArgs e, const float *scratch) {
    extern __shared__ __align__(16) uint8_t vsm2[];
    const int o = e.o;
    const long long o3 = (long long)o * o * o;
    const int jl = blockIdx.x / 3, ax = blockIdx.x - 3 * (blockIdx.x / 3);
    int a, b, c;
    unpack_job(w.jobs[jl], a, b, c);
    const float *Yb = scratch + ((long long)jl * kSlots + 6) * o3;
    if (ax == 0) vterm2_axis<0>(w, e, Yb, a, b, c, vsm2);
    else if (ax == 1) vterm2_axis<1>(w, e, Yb, a, b, c, vsm2);
    else vterm2_axis<2>(w, e, Yb, a, b, c, vsm2);
}

cudaError_t f32_vterm(const WaveView &w, const EpiArgs &e, const float *scratch, cudaStream_t st) {
    if (w.n_jobs <= 0) return cudaSuccess;
    if (e.o > 64 || e.o % 8 != 0) return cudaErrorInvalidValue;
    const size_t smem = vterm2_smem(e.o);
    {
        cudaError_t ce = smem_optin(reinterpret_cast<const void *>(vterm2_kernel), (int)vterm2_smem(64));
        if (ce != cudaSuccess) return ce;
    }
    vterm2_kernel<<<w.n_jobs * 3, V2_NT, smem, st>>>(w, e, scratch);
    return cudaGetLastError();
}

// Deterministic compensated sum of the per-job energies, fixed order: each of
// kRedBlocks CTAs sums a fixed contiguous chunk (Neumaier), then one CTA sums
// the partials in block order.
constexpr int kRedBlocks = kReduceParts;

__global__ void __launch_bounds__(1024) reduce_energy_part_kernel(const double *job_e, long long n, double *part) {
    __shared__ double ss[1024], cc[1024];
    const long long chunk = (n + gridDim.x - 1) / gridDim.x;
    const long long lo = blockIdx.x * chunk, hi = lo + chunk < n ? lo + chunk : n;
    KSum k;
    for (long long i = lo + threadIdx.x; i < hi; i += blockDim.x) k.add(job_e[i]);
    ss[threadIdx.x] = k.s;
    cc[threadIdx.x] = k.c;
    __syncthreads();
    if (threadIdx.x == 0) {
        KSum t;
        for (int i = 0; i < blockDim.x; ++i) { t.add(ss[i]); t.add(cc[i]); }
        part[2 * blockIdx.x] = t.s;
        part[2 * blockIdx.x + 1] = t.c;
    }
}

__global__ void reduce_energy_final_kernel(const double *part, int nparts, double *out) {
    KSum t;
    for (int i = 0; i < 2 * nparts; ++i) t.add(part[i]);
    out[0] = t.value();
}

// single-CTA variant (no work buffer)
__global__ void __launch_bounds__(1024) reduce_energy_kernel(const double *job_e, long long n, double *out) {
    __shared__ double ss[1024], cc[1024];
    KSum k;
    for (long long i = threadIdx.x; i < n; i += blockDim.x) k.add(job_e[i]);
    ss[threadIdx.x] = k.s;
    cc[threadIdx.x] = k.c;
    __syncthreads();
    if (threadIdx.x == 0) {
        KSum t;
        for (int i = 0; i < blockDim.x; ++i) { t.add(ss[i]); t.add(cc[i]); }
        out[0] = t.value();
    }
}

cudaError_t reduce_energy_1cta(const double *job_e, long long n, double *e_out, cudaStream_t st) {
    reduce_energy_kernel<<<1, 1024, 0, st>>>(job_e, n, e_out);
    return cudaGetLastError();
}

cudaError_t reduce_energy(const double *job_e, long long n, double *e_out, double *work, cudaStream_t st) {
    reduce_energy_part_kernel<<<kRedBlocks, 1024, 0, st>>>(job_e, n, work);
    reduce_energy_final_kernel<<<1, 1, 0, st>>>(work, kRedBlocks, e_out);
    return cudaGetLastError();
}

}  // namespace ctb
