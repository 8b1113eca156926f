// Density-fitted ERI producer of the (T) inputs and its VJP, float64 on the
// tensor pipe (DMMA, mma.sync m8n8k4 .f64).
//
// pyscfad's DF-CCSD forms ovoo = Lov^T Loo, ovov = Lov^T Lov and
// ovvv = Lov^T Lvv from the three-index factors (pyscfad/cc/dfccsd.py:73-88);
// the (T) driver then transposes them into the kernel layouts vooo and vvop
// (pyscfad/cc/ccsd_t.py:88-106).  Here the kernel layouts come straight from
// the factors, with the transposes folded into the GEMMs' addressing:
//   vvop[a,y,i,p] = sum_P Lov[P,i,a] R[P,p,y],   R = [Lov ; Lvv] (naux, nmo, nvir)
//   vooo[a,i,k,j] = sum_P Lov[P,i,a] Loo[P,j,k]
// so neither ovvv nor any intermediate of vvop's size is formed.  The VJP
// pulls kernel-layout gradients back onto the factors by the transposed
// contractions (dLov, dLoo, and dR in the transposed order Rt = (naux, nvir, nmo)).
//
// All of these are one GEMM shape C = alpha A B (+ C) whose operands are
// addressed through two-level index maps: an index x of a row or column is
// split as (x / div, x % div) and weighted by two strides, which covers every
// permuted layout above.
#include <cuda_runtime.h>
#include <climits>
#include "ct_common.cuh"
#include "ct_internal.h"
#include "../../include/pyscfad_b200.h"

namespace ctb {
namespace df {

struct Ix {          // x -> (x / div) * s1 + (x % div) * s0
    int div;
    long long s1, s0;
};
struct Opd {
    const double *p;
    Ix r, c;         // row and column index maps
};

__host__ __device__ inline Ix ix_plain(long long s) { return Ix{INT_MAX, 0, s}; }
__host__ __device__ inline Ix ix_two(int div, long long s1, long long s0) { return Ix{div, s1, s0}; }

constexpr int BM = 64, BN = 64, BK = 16, NTHR = 256, LD = 64 + 4;

// One operand's slice of a K step: 4 loads per thread.  mn_fast: consecutive
// threads take consecutive rows (m or n), else consecutive k.  The k part of
// each load's address is kept as (quotient, remainder) and advanced by BK
// without divisions.
struct Loader {
    long long base[4];   // address part of the m (or n) index; -1 when out of range
    int kq[4], kr[4];    // k = kq * div + kr for this load
    int kl[4], ml[4];    // tile coordinates
    __device__ void init(const Ix &mix, const Ix &kix, int m0, int M, bool mn_fast) {
        const int t = threadIdx.x;
        for (int j = 0; j < 4; ++j) {
            int m, k;
            if (mn_fast) { m = t % 64; k = t / 64 + 4 * j; }
            else { k = t % 16; m = t / 16 + 16 * j; }
            ml[j] = m;
            kl[j] = k;
            const int gm = m0 + m;
            base[j] = gm < M ? (long long)(gm / mix.div) * mix.s1 + (long long)(gm % mix.div) * mix.s0 : -1;
            kq[j] = k / kix.div;
            kr[j] = k % kix.div;
        }
    }
    __device__ void load(const double *p, const Ix &kix, int kb, int K, double (&v)[4]) const {
        for (int j = 0; j < 4; ++j) {
            const bool ok = base[j] >= 0 && kb + kl[j] < K;
            v[j] = ok ? p[base[j] + (long long)kq[j] * kix.s1 + (long long)kr[j] * kix.s0] : 0.0;
        }
    }
    __device__ void advance(const Ix &kix) {
        for (int j = 0; j < 4; ++j) {
            kr[j] += BK;
            while (kr[j] >= kix.div) { kr[j] -= kix.div; ++kq[j]; }
        }
    }
};

// C[m,n] = alpha sum_k A[m,k] B[k,n] (+ C[m,n] when acc); 64 x 64 tiles, 8 warps
// of 32 x 16 (4 x 2 DMMA tiles), K steps of 16 staged in shared memory with a
// register prefetch of the next step.
__global__ void __launch_bounds__(NTHR) gemm_strided_kernel(int M, int N, int K, Opd A, Opd B, double *C, Ix cr,
                                                            Ix cc, double alpha, int acc, int a_mfast,
                                                            int b_nfast) {
    __shared__ double As[BK][LD], Bs[BK][LD];
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, c = lane & 3;
    const int wm = (warp >> 2) * 32, wn = (warp & 3) * 16;
    Loader la, lb;
    la.init(A.r, A.c, m0, M, a_mfast != 0);
    lb.init(B.c, B.r, n0, N, b_nfast != 0);
    double d[4][2][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) d[i][j][0] = d[i][j][1] = 0.0;
    double va[4], vb[4];
    la.load(A.p, A.c, 0, K, va);
    lb.load(B.p, B.r, 0, K, vb);
    for (int kb = 0; kb < K; kb += BK) {
        __syncthreads();
        for (int j = 0; j < 4; ++j) {
            As[la.kl[j]][la.ml[j]] = va[j];
            Bs[lb.kl[j]][lb.ml[j]] = vb[j];
        }
        __syncthreads();
        if (kb + BK < K) {
            la.advance(A.c);
            lb.advance(B.r);
            la.load(A.p, A.c, kb + BK, K, va);
            lb.load(B.p, B.r, kb + BK, K, vb);
        }
#pragma unroll
        for (int kk = 0; kk < BK; kk += 4) {
            double a[4], b[2];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = As[kk + c][wm + 8 * i + g];
#pragma unroll
            for (int j = 0; j < 2; ++j) b[j] = Bs[kk + c][wn + 8 * j + g];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 2; ++j) dmma(d[i][j], a[i], b[j]);
        }
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int m = m0 + wm + 8 * i + g;
        if (m >= M) continue;
        const long long rm = (long long)(m / cr.div) * cr.s1 + (long long)(m % cr.div) * cr.s0;
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int n = n0 + wn + 8 * j + 2 * c + h;
                if (n >= N) continue;
                double *dst = C + rm + (long long)(n / cc.div) * cc.s1 + (long long)(n % cc.div) * cc.s0;
                *dst = acc ? *dst + alpha * d[i][j][h] : alpha * d[i][j][h];
            }
    }
}

static cudaError_t gemm(int M, int N, int K, const Opd &A, const Opd &B, double *C, Ix cr, Ix cc, double alpha,
                        bool acc, cudaStream_t st) {
    if (M <= 0 || N <= 0 || K <= 0) return cudaSuccess;
    dim3 grid((N + BN - 1) / BN, (M + BM - 1) / BM);
    if (grid.y > 65535) return cudaErrorInvalidValue;
    const int a_mfast = A.r.s0 == 1 && A.r.div == INT_MAX ? 1 : (A.r.div != INT_MAX && A.r.s0 == 1 ? 1 : 0);
    const int b_nfast = B.c.s0 == 1 ? 1 : 0;
    gemm_strided_kernel<<<grid, NTHR, 0, st>>>(M, N, K, A, B, C, cr, cc, alpha, acc ? 1 : 0, a_mfast, b_nfast);
    return cudaGetLastError();
}

}  // namespace df
}  // namespace ctb

using namespace ctb::df;

extern "C" {

int ct_df_layouts(int nocc, int nvir, int naux, const double *Loo, const double *Lov, const double *R, double *vooo,
                  double *vvop, void *stream) {
    if (!Loo || !Lov || !R || !vooo || !vvop) return CT_ERR_NULL;
    if (nocc < 1 || nvir < 1 || naux < 1 || nocc > 255 || nvir > 1024) return CT_ERR_SHAPE;
    const long long o = nocc, v = nvir, n = o + v;
    cudaStream_t st = (cudaStream_t)stream;
    // rows m = (i, a) = i v + a: Lov[P, i, a] at P o v + m
    const Opd Alov{Lov, ix_plain(1), ix_plain(o * v)};
    // vvop[a, y, i, p]: columns (p, y) = p v + y of R[P, p, y]
    const Opd Br{R, ix_plain(n * v), ix_plain(1)};
    cudaError_t e = gemm((int)(o * v), (int)(n * v), naux, Alov, Br, vvop, ix_two((int)v, n, v * o * n),
                         ix_two((int)v, 1, o * n), 1.0, false, st);
    if (e != cudaSuccess) return CT_ERR_CUDA;
    // vooo[a, i, k, j]: columns (j, k) = j o + k of Loo[P, j, k]
    const Opd Bloo{Loo, ix_plain(o * o), ix_plain(1)};
    e = gemm((int)(o * v), (int)(o * o), naux, Alov, Bloo, vooo, ix_two((int)v, o * o, o * o * o),
             ix_two((int)o, 1, o), 1.0, false, st);
    return e == cudaSuccess ? CT_OK : CT_ERR_CUDA;
}

int ct_df_factor_bar(int nocc, int nvir, int naux, const double *Loo, const double *Lov, const double *Rt,
                     const double *vooo_bar, const double *vvop_bar, double *dLoo, double *dLov, double *dRt,
                     void *stream) {
    if (!Loo || !Lov || !Rt || !vooo_bar || !vvop_bar || !dLoo || !dLov || !dRt) return CT_ERR_NULL;
    if (nocc < 1 || nvir < 1 || naux < 1 || nocc > 255 || nvir > 1024) return CT_ERR_SHAPE;
    const long long o = nocc, v = nvir, n = o + v;
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e;
    // dLov[P, (i,a)] += sum_{(y,p)} Rt[P, y, p] vvop_bar[a, y, i, p]
    {
        const Opd A{Rt, ix_plain(v * n), ix_plain(1)};
        const Opd B{vvop_bar, ix_two((int)n, o * n, 1), ix_two((int)v, n, v * o * n)};
        e = gemm(naux, (int)(o * v), (int)(v * n), A, B, dLov, ix_plain(o * v), ix_plain(1), 1.0, true, st);
        if (e != cudaSuccess) return CT_ERR_CUDA;
    }
    // dRt[P, (y,p)] += sum_{(i,a)} Lov[P, i, a] vvop_bar[a, y, i, p]
    {
        const Opd A{Lov, ix_plain(o * v), ix_plain(1)};
        const Opd B{vvop_bar, ix_two((int)v, n, v * o * n), ix_two((int)n, o * n, 1)};
        e = gemm(naux, (int)(v * n), (int)(o * v), A, B, dRt, ix_plain(v * n), ix_plain(1), 1.0, true, st);
        if (e != cudaSuccess) return CT_ERR_CUDA;
    }
    // dLov[P, (i,a)] += sum_{(j,k)} Loo[P, j, k] vooo_bar[a, i, k, j]
    {
        const Opd A{Loo, ix_plain(o * o), ix_plain(1)};
        const Opd B{vooo_bar, ix_two((int)o, 1, o), ix_two((int)v, o * o, o * o * o)};
        e = gemm(naux, (int)(o * v), (int)(o * o), A, B, dLov, ix_plain(o * v), ix_plain(1), 1.0, true, st);
        if (e != cudaSuccess) return CT_ERR_CUDA;
    }
    // dLoo[P, (j,k)] += sum_{(i,a)} Lov[P, i, a] vooo_bar[a, i, k, j]
    {
        const Opd A{Lov, ix_plain(o * v), ix_plain(1)};
        const Opd B{vooo_bar, ix_two((int)v, o * o, o * o * o), ix_two((int)o, 1, o)};
        e = gemm(naux, (int)(o * o), (int)(o * v), A, B, dLoo, ix_plain(o * o), ix_plain(1), 1.0, true, st);
        if (e != cudaSuccess) return CT_ERR_CUDA;
    }
    return CT_OK;
}

}  // extern "C"
