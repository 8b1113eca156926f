// Iterative (T) on the full 6-D triples amplitudes (pyscfad/cc/ccsd_t_slow.py:
// 128-293): the update step of update_amps (:188-208) and the energy of
// energy (:210-220), on (v, v, v, o, o, o) arrays [a][b][c][i][j][k].
//
// The seed (t3_c = P6(W + V) / d3, t3_x = r3(P6(W)) / 3) comes from the
// F1/F2 GEMMs and the orbit epilogue (ct_t3_init in ct_host.cu).  A step is
//   t3_new = (P6(W + V) + P3(fvv' t3) - P3(foo' t3)) / d3
//          = t3_c + (P3(tvv) - P3(too)) / d3,
// P3(x)[abc][ijk] = x[abc][ijk] + x[bac][jik] + x[cba][kji] (:174-176), with
// fvv', foo' the Fock blocks without their diagonals.  The caller forms the
// two products as plain GEMMs: tvv = fvv' t3 on the first virtual index of
// the [a][b][c][i][j][k] array, too = foo' t3 on the first occupied index of
// an occupied-major copy [i][a][b][c][j][k], which this kernel also writes
// for the next step (t3_new_m).  It applies P3, divides by d3 and forms, in a
// fixed order, |t3_new - t3|^2 and the energy sum t3_new t3_x.
#include <cuda_runtime.h>
#include "ct_common.cuh"
#include "ct_internal.h"
#include "../../include/pyscfad_b200.h"

namespace ctb {
namespace t3it {

constexpr int kThreads = 256, kBlocks = 1024;

__global__ void __launch_bounds__(kThreads) update_kernel(int o, int v, const double *__restrict__ e,
                                                           const double *__restrict__ t3c,
                                                           const double *__restrict__ tvv,
                                                           const double *__restrict__ toom,
                                                           const double *__restrict__ t3,
                                                           const double *__restrict__ t3x,
                                                           double *__restrict__ t3n, double *__restrict__ t3nm,
                                                           double *__restrict__ part) {
    const long long o2 = (long long)o * o, o3 = o2 * o, v2 = (long long)v * v;
    const long long N = v2 * v * o3, mrow = v2 * v * o2;   // occupied-major row: [abc][jk]
    double s0 = 0.0, s1 = 0.0;
    for (long long idx = blockIdx.x * (long long)kThreads + threadIdx.x; idx < N;
         idx += (long long)kBlocks * kThreads) {
        const long long abc = idx / o3, ijk = idx - abc * o3;
        const int a = (int)(abc / v2), b = (int)((abc / v) % v), c = (int)(abc % v);
        const int i = (int)(ijk / o2), j = (int)((ijk / o) % o), k = (int)(ijk % o);
        const long long bac = ((long long)b * v + a) * v + c, jik = ((long long)j * o + i) * o + k;
        const long long cba = ((long long)c * v + b) * v + a, kji = ((long long)k * o + j) * o + i;
        // too at (abc, ijk), (bac, jik), (cba, kji) in the [i][abc][jk] layout
        const double p3 = (tvv[idx] + tvv[bac * o3 + jik] + tvv[cba * o3 + kji]) -
                          (toom[i * mrow + abc * o2 + j * o + k] + toom[j * mrow + bac * o2 + i * o + k] +
                           toom[k * mrow + cba * o2 + j * o + i]);
        const double d3 = e[i] + e[j] + e[k] - e[o + a] - e[o + b] - e[o + c];
        const double x = t3c[idx] + p3 / d3;
        t3n[idx] = x;
        if (t3nm) t3nm[i * mrow + abc * o2 + j * o + k] = x;
        const double d = x - t3[idx];
        s0 = fma(d, d, s0);
        s1 = fma(x, t3x[idx], s1);
    }
    // fixed-order block sum
    __shared__ double r0[kThreads], r1[kThreads];
    r0[threadIdx.x] = s0;
    r1[threadIdx.x] = s1;
    __syncthreads();
    for (int m = kThreads / 2; m >= 1; m >>= 1) {
        if ((int)threadIdx.x < m) {
            r0[threadIdx.x] += r0[threadIdx.x + m];
            r1[threadIdx.x] += r1[threadIdx.x + m];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = r0[0];
        part[2 * blockIdx.x + 1] = r1[0];
    }
}

__global__ void sum_kernel(const double *__restrict__ part, double *__restrict__ sums) {
    __shared__ double r0[kThreads], r1[kThreads];
    double s0 = 0.0, s1 = 0.0;
    for (int b = threadIdx.x; b < kBlocks; b += kThreads) {
        s0 += part[2 * b];
        s1 += part[2 * b + 1];
    }
    r0[threadIdx.x] = s0;
    r1[threadIdx.x] = s1;
    __syncthreads();
    for (int m = kThreads / 2; m >= 1; m >>= 1) {
        if ((int)threadIdx.x < m) {
            r0[threadIdx.x] += r0[threadIdx.x + m];
            r1[threadIdx.x] += r1[threadIdx.x + m];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        sums[0] = r0[0];
        sums[1] = r1[0];
    }
}

}  // namespace t3it
}  // namespace ctb

using namespace ctb;

extern "C" int ct_t3_update(int nocc, int nvir, const double *mo_energy, const double *t3_c, const double *tvv,
                            const double *too_m, const double *t3, const double *t3_x, double *t3_new,
                            double *t3_new_m, double *sums, void *stream) {
    if (nocc < 1 || nocc > 255 || nvir < 1 || nvir > 1024) return CT_ERR_SHAPE;
    if (!mo_energy || !t3_c || !tvv || !too_m || !t3 || !t3_x || !t3_new || !sums) return CT_ERR_NULL;
    // P3 reads other elements of tvv and too_m than the one written
    const double *ins[4] = {t3, tvv, too_m, t3_c};
    for (const double *q : ins)
        if (q == t3_new || (t3_new_m && q == t3_new_m)) return CT_ERR_SHAPE;
    cudaStream_t st = (cudaStream_t)stream;
    double *part = nullptr;
    if (cudaMallocAsync(&part, sizeof(double) * 2 * t3it::kBlocks, st) != cudaSuccess) return CT_ERR_NOMEM;
    t3it::update_kernel<<<t3it::kBlocks, t3it::kThreads, 0, st>>>(nocc, nvir, mo_energy, t3_c, tvv, too_m, t3, t3_x,
                                                                   t3_new, t3_new_m, part);
    t3it::sum_kernel<<<1, t3it::kThreads, 0, st>>>(part, sums);
    const cudaError_t ce = cudaGetLastError();
    cudaFreeAsync(part, st);
    return ce == cudaSuccess ? CT_OK : CT_ERR_CUDA;
}
