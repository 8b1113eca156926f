// Diagnostic self-test of the tcgen05 building blocks used by the mixed path:
// one CTA writes a 128x32 (A) and 32x32 (B) float tile in the 128-byte
// swizzled K-major layout by hand, issues tcgen05.mma (kind::tf32, M=128,
// N=32, 4 k-steps), and reads the accumulator back with tcgen05.ld.
#include <cuda_runtime.h>
#include "tc_ptx.cuh"
#include "../../include/pyscfad_b200.h"

namespace ctb {

__device__ __forceinline__ void mma_tf32_masked(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    uint32_t m0 = 0, m1 = 0, m2 = 0, m3 = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(m0), "r"(m1), "r"(m2), "r"(m3)
        : "memory");
}

// element (r, k) of a K-major tile with 128-B rows and 128-B swizzle
__device__ __forceinline__ int sw128(int r, int k) { return r * 32 + ((((k >> 2) ^ (r & 7)) << 2) | (k & 3)); }

// element (m, k) of an MN-major tf32 tile: chunks of 32 MN elements, each 32
// K-rows of 128 B; the four 32-B granules of a row are permuted by (k mod 4)
__device__ __forceinline__ int mn128(int m, int k) {
    const int c = m >> 5, mm = m & 31;
    return c * 1024 + k * 32 + ((((mm >> 3) ^ (k & 3)) << 3) | (mm & 7));
}

// variants: 0/1 K-major A, N=32 (two MMA forms); 2 MN-major A, N=32; 3 K-major, N=256
__global__ void __launch_bounds__(128) tc_selftest_kernel(const float *A, const float *B, float *D, int variant,
                                                          int *err) {
    extern __shared__ uint8_t raw[];
    uint8_t *sm = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(raw) + 1023) & ~uintptr_t(1023));
    const int N = variant == 3 ? 256 : 32;
    float *sA = reinterpret_cast<float *>(sm);           // 128 x 32
    float *sB = reinterpret_cast<float *>(sm + 16384);   // N x 32
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + 16384 + 32768);
    uint32_t *slot = reinterpret_cast<uint32_t *>(bar + 2);
    for (int i = threadIdx.x; i < 128 * 32; i += blockDim.x)
        sA[variant == 2 ? mn128(i / 32, i % 32) : sw128(i / 32, i % 32)] = A[i];
    for (int i = threadIdx.x; i < N * 32; i += blockDim.x) sB[sw128(i / 32, i % 32)] = B[i];
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (threadIdx.x == 0) { tc::mbar_init(tc::smem_u32(bar), 1); tc::fence_mbar_init(); }
    const int warp = threadIdx.x >> 5;
    if (warp == 0) { tc::tmem_alloc(tc::smem_u32(slot), 256); tc::tmem_relinquish(); }
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tmem = *slot;
    if (threadIdx.x == 0) {
        const uint32_t id = tc::idesc(2, 128, N, variant == 2, false);
        for (int kk = 0; kk < 4; ++kk) {
            const uint64_t da = variant == 2 ? tc::sdesc(tc::smem_u32(sA) + kk * 1024, 4096, 512, tc::kSw128Base32)
                                             : tc::sdesc(tc::smem_u32(sA) + kk * 32, 16, 1024);
            const uint64_t db = tc::sdesc(tc::smem_u32(sB) + kk * 32, 16, 1024);
            if (variant == 1) mma_tf32_masked(tmem, da, db, id, kk ? 1u : 0u);
            else tc::mma_tf32(tmem, da, db, id, kk ? 1u : 0u);
        }
        tc::mma_commit(tc::smem_u32(bar));
    }
    __syncwarp();
    tc::mbar_wait(tc::smem_u32(bar), 0, err);
    tc::fence_after();
    float v0[16];
    const uint32_t ta = tmem + ((uint32_t)(32 * warp) << 16);
    const int row = 32 * warp + (threadIdx.x & 31);
    for (int c0 = 0; c0 < N; c0 += 16) {
        tc::tmem_ld16(ta + c0, v0);
        for (int j = 0; j < 16; ++j) D[row * N + c0 + j] = v0[j];
    }
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    if (warp == 0) tc::tmem_dealloc(tmem, 256);
}

}  // namespace ctb

extern "C" int ct_tc_selftest(int variant, const float *A, const float *B, float *D) {
    using namespace ctb;
    int *err = nullptr;
    if (cudaMalloc(&err, sizeof(int)) != cudaSuccess) return CT_ERR_NOMEM;
    cudaMemset(err, 0, sizeof(int));
    const int smem = 16384 + 32768 + 64 + 1024;
    cudaFuncSetAttribute(tc_selftest_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    tc_selftest_kernel<<<1, 128, smem>>>(A, B, D, variant, err);
    cudaError_t e = cudaDeviceSynchronize();
    int h = 0;
    cudaMemcpy(&h, err, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(err);
    if (e != cudaSuccess) return CT_ERR_CUDA;
    return h ? CT_ERR_TIMEOUT : CT_OK;
}
