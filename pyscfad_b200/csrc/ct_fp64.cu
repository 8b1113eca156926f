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
#include <cstdio>
#include "ct_common.cuh"
#include "ct_internal.h"

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

__device__ __forceinline__ void dmma(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
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

// Value stored into a W-bar slot: float scratch feeds tf32 tensor-core GEMMs,
// so it is rounded to the nearest tf32 (the MMA itself would truncate).
template <typename ST> __device__ __forceinline__ ST wbar_store(double x) { return (ST)x; }
template <> __device__ __forceinline__ float wbar_store<float>(double x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"((float)x));
    return __uint_as_float(r);
}

// ---------------------------------------------------------------------------
// Orbit epilogue.  One CTA per job; each thread owns whole occupied orbits
// {perm(i,j,k)} with i>=j>=k, so every scratch element is read once (G) and
// written once (Wbar, ybar) by the same thread, and r3 never leaves registers.
// ---------------------------------------------------------------------------
template <typename ST>
__global__ void __launch_bounds__(128) epi_kernel(const WaveView w, const EpiArgs e, ST *scratch) {
    const int o = e.o, v = e.v, n = e.n;
    const long long o3 = (long long)o * o * o;
    const int jl = blockIdx.x;
    int a, b, c;
    unpack_job(w.jobs[jl], a, b, c);
    const double fac = job_fac(a, b, c);
    const double eabc = e.mo_energy[o + a] + e.mo_energy[o + b] + e.mo_energy[o + c];
    ST *S = scratch + (long long)jl * kSlots * o3;

    const double *pv[6], *pt[6];
    int tz[6];
#pragma unroll
    for (int s = 0; s < 6; ++s) {
        int x, y, z;
        term_xyz(s, a, b, c, x, y, z);
        pv[s] = e.vvop + ((long long)(x * v + y) * o) * n;
        pt[s] = e.t2T + ((long long)(y * v + x) * o) * o;
        tz[s] = z * o;
    }

    __shared__ double occ_acc[256];
    __shared__ double red_s[128], red_c[128], red_v[128];
    for (int i = threadIdx.x; i < o; i += blockDim.x) occ_acc[i] = 0.0;
    __syncthreads();

    KSum eacc;
    double vir_acc = 0.0;
    const double eb = e.et_bar;
    for (int q = threadIdx.x; q < e.n_orb; q += blockDim.x) {
        const int pk = e.orbits[q];
        const int ijk[3] = {pk & 255, (pk >> 8) & 255, (pk >> 16) & 255};
        int pp[6][3];
        long long pos[6];
#pragma unroll
        for (int s = 0; s < 6; ++s) {
#pragma unroll
            for (int m = 0; m < 3; ++m) pp[s][m] = ijk[kR(s, m)];
            pos[s] = ((long long)pp[s][0] * o + pp[s][1]) * o + pp[s][2];
        }
        bool first[6];
#pragma unroll
        for (int s = 0; s < 6; ++s) {
            bool f = true;
#pragma unroll
            for (int t = 0; t < s; ++t) f = f && (pos[t] != pos[s]);
            first[s] = f;
        }
        double W[6];
#pragma unroll
        for (int s = 0; s < 6; ++s) W[s] = 0.0;
#pragma unroll
        for (int sg = 0; sg < 6; ++sg) {
            double g[6];
#pragma unroll
            for (int s = 0; s < 6; ++s) g[s] = (double)S[sg * o3 + pos[s]];
#pragma unroll
            for (int s = 0; s < 6; ++s) W[s] += g[kComp(s, sg)];
        }
        double Y[6];
#pragma unroll
        for (int s = 0; s < 6; ++s) {
            double vs = 0.0;
#pragma unroll
            for (int sg = 0; sg < 6; ++sg) {
                const int cs = kComp(s, sg);
                const int P = pp[cs][0], Q = pp[cs][1], R = pp[cs][2];
                vs += __ldg(pv[sg] + (long long)P * n + Q) * __ldg(e.t1T + tz[sg] + R)
                    + __ldg(pt[sg] + P * o + Q) * __ldg(e.fvo + tz[sg] + R);
            }
            Y[s] = W[s] + 0.5 * vs;
        }
        double Z[6];
#pragma unroll
        for (int s = 0; s < 6; ++s) {
            double zz = 0.0;
#pragma unroll
            for (int t = 0; t < 6; ++t) zz += kR3C(t) * Y[kComp(s, t)];
            Z[s] = zz;
        }
        const double d3 = fac / (e.mo_energy[ijk[0]] + e.mo_energy[ijk[1]] + e.mo_energy[ijk[2]] - eabc);
#pragma unroll
        for (int s = 0; s < 6; ++s)
            if (first[s]) eacc.add(W[s] * Z[s] * d3);
        if (e.with_vjp) {
            double zb[6], wb[6], tmp = 0.0;
#pragma unroll
            for (int s = 0; s < 6; ++s) {
                zb[s] = eb * W[s] * d3;
                wb[s] = eb * Z[s] * d3;
                if (first[s]) tmp += eb * W[s] * Z[s] * d3 * d3 / fac;
            }
            double yb[6];
#pragma unroll
            for (int s = 0; s < 6; ++s) {
                double t = 0.0;
#pragma unroll
                for (int u = 0; u < 6; ++u) t += kR3C(u) * zb[kComp(s, u)];
                yb[s] = t;
            }
#pragma unroll
            for (int s = 0; s < 6; ++s) wb[s] += yb[s];
            atomicAdd(&occ_acc[ijk[0]], -tmp);
            atomicAdd(&occ_acc[ijk[1]], -tmp);
            atomicAdd(&occ_acc[ijk[2]], -tmp);
            vir_acc += tmp;
#pragma unroll
            for (int sg = 0; sg < 6; ++sg)
#pragma unroll
                for (int s = 0; s < 6; ++s) S[sg * o3 + pos[s]] = wbar_store<ST>(wb[kComp(s, kInv(sg))]);
#pragma unroll
            for (int s = 0; s < 6; ++s) S[6 * o3 + pos[s]] = (ST)yb[s];
        }
    }
    red_s[threadIdx.x] = eacc.s;
    red_c[threadIdx.x] = eacc.c;
    red_v[threadIdx.x] = vir_acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        KSum tot;
        double vt = 0.0;
        for (int t = 0; t < blockDim.x; ++t) {
            tot.add(red_s[t]);
            tot.add(red_c[t]);
            vt += red_v[t];
        }
        const long long amaj = (long long)a * (a + 1) * (a + 2) / 6 + (long long)b * (b + 1) / 2 + c;
        e.job_e[amaj] = 2.0 * tot.value();
        if (e.with_vjp) {
            atomicAdd(&e.mo_energy_bar[o + a], vt);
            atomicAdd(&e.mo_energy_bar[o + b], vt);
            atomicAdd(&e.mo_energy_bar[o + c], vt);
        }
    }
    if (e.with_vjp)
        for (int i = threadIdx.x; i < o; i += blockDim.x) atomicAdd(&e.mo_energy_bar[i], occ_acc[i]);
}

// V-term bars of one (job, sigma): with Vbar_sigma[p,q,r] = ybar[idx_sigma(p,q,r)],
//   vvop_bar[x,y,p,q] += 1/2 sum_r Vbar t1T[z,r]     (get_vvoo_bar, ccsd_t_vjp.c:171-186)
//   t2T_bar[y,x,p,q]  += 1/2 sum_r Vbar fvo[z,r]     (get_t2T_bar gemv, :228-230)
//   t1T_bar[z,r]      += 1/2 sum_pq Vbar vvop[x,y,p,q]   (get_t1T_bar, :188-204)
//   fvo_bar[z,r]      += 1/2 sum_pq Vbar t2T[y,x,p,q]    (get_fvo_bar, :233-246)
template <typename ST>
__global__ void __launch_bounds__(256) vterm_kernel(const WaveView w, const EpiArgs e, const ST *scratch) {
    const int o = e.o, v = e.v, n = e.n;
    const long long o3 = (long long)o * o * o;
    const int jl = blockIdx.x / 6, sg = blockIdx.x - 6 * (blockIdx.x / 6);
    int a, b, c, x, y, z;
    unpack_job(w.jobs[jl], a, b, c);
    term_xyz(sg, a, b, c, x, y, z);
    const ST *Yb = scratch + ((long long)jl * kSlots + 6) * o3;
    const int ri = kInv(sg);
    const int r0 = kR(ri, 0), r1 = kR(ri, 1), r2 = kR(ri, 2);
    const double *vv = e.vvop + ((long long)(x * v + y) * o) * n;
    const double *tt = e.t2T + ((long long)(y * v + x) * o) * o;
    double *vvb = e.vvop_bar + ((long long)(x * v + y) * o) * n;
    double *ttb = e.t2T_bar + ((long long)(y * v + x) * o) * o;
    const double *t1z = e.t1T + z * o, *fz = e.fvo + z * o;
    const int oo = o * o;
    for (int pq = threadIdx.x; pq < oo; pq += blockDim.x) {
        const int p_ = pq / o, q_ = pq - p_ * o;
        double sa = 0.0, sb = 0.0;
        for (int r = 0; r < o; ++r) {
            const int t3[3] = {p_, q_, r};
            const double vb = (double)Yb[((long long)t3[r0] * o + t3[r1]) * o + t3[r2]];
            sa += vb * __ldg(t1z + r);
            sb += vb * __ldg(fz + r);
        }
        atomicAdd(vvb + (long long)p_ * n + q_, 0.5 * sa);
        atomicAdd(ttb + pq, 0.5 * sb);
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int r = wid; r < o; r += nw) {
        double sc = 0.0, sd = 0.0;
        for (int pq = lane; pq < oo; pq += 32) {
            const int p_ = pq / o, q_ = pq - p_ * o;
            const int t3[3] = {p_, q_, r};
            const double vb = (double)Yb[((long long)t3[r0] * o + t3[r1]) * o + t3[r2]];
            sc += vb * __ldg(vv + (long long)p_ * n + q_);
            sd += vb * __ldg(tt + pq);
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            sc += __shfl_xor_sync(0xffffffffu, sc, off);
            sd += __shfl_xor_sync(0xffffffffu, sd, off);
        }
        if (lane == 0) {
            atomicAdd(e.t1T_bar + z * o + r, 0.5 * sc);
            atomicAdd(e.fvo_bar + z * o + r, 0.5 * sd);
        }
    }
}

cudaError_t f64_epilogue(const WaveView &w, const EpiArgs &e, double *scratch, cudaStream_t st) {
    if (w.n_jobs <= 0) return cudaSuccess;
    epi_kernel<double><<<w.n_jobs, 128, 0, st>>>(w, e, scratch);
    return cudaGetLastError();
}

cudaError_t f64_vterm(const WaveView &w, const EpiArgs &e, const double *scratch, cudaStream_t st) {
    if (w.n_jobs <= 0) return cudaSuccess;
    vterm_kernel<double><<<w.n_jobs * 6, 256, 0, st>>>(w, e, scratch);
    return cudaGetLastError();
}

cudaError_t f32_epilogue(const WaveView &w, const EpiArgs &e, float *scratch, cudaStream_t st) {
    if (w.n_jobs <= 0) return cudaSuccess;
    epi_kernel<float><<<w.n_jobs, 128, 0, st>>>(w, e, scratch);
    return cudaGetLastError();
}

cudaError_t f32_vterm(const WaveView &w, const EpiArgs &e, const float *scratch, cudaStream_t st) {
    if (w.n_jobs <= 0) return cudaSuccess;
    vterm_kernel<float><<<w.n_jobs * 6, 256, 0, st>>>(w, e, scratch);
    return cudaGetLastError();
}

// Deterministic compensated sum of the per-job energies, fixed order.
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

cudaError_t reduce_energy(const double *job_e, long long n, double *e_out, cudaStream_t st) {
    reduce_energy_kernel<<<1, 1024, 0, st>>>(job_e, n, e_out);
    return cudaGetLastError();
}

}  // namespace ctb
