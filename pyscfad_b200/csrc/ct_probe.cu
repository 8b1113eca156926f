// Pipe-rate probes used as roofline denominators where no driver-measured
// peak exists (float64 DMMA and DFMA).  Register-resident loops: no memory
// traffic inside the timed region.
#include <cuda_runtime.h>
#include "../../include/pyscfad_b200.h"

namespace ctb {

__global__ void __launch_bounds__(256) probe_dmma(double *out, int iters) {
    double acc[8][2];
    double a = 1.0 + 1e-9 * threadIdx.x, b = 1.0 - 1e-9 * threadIdx.x;
#pragma unroll
    for (int i = 0; i < 8; ++i) acc[i][0] = acc[i][1] = 0.0;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int i = 0; i < 8; ++i)
            asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                         : "+d"(acc[i][0]), "+d"(acc[i][1])
                         : "d"(a), "d"(b));
    }
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < 8; ++i) s += acc[i][0] + acc[i][1];
    if (s == 12345.678) out[0] = s;
}

__global__ void __launch_bounds__(256) probe_dfma(double *out, int iters) {
    double acc[16];
    const double a = 1.0 + 1e-9 * threadIdx.x, b = 1.0 - 1e-12;
#pragma unroll
    for (int i = 0; i < 16; ++i) acc[i] = i;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int i = 0; i < 16; ++i) acc[i] = fma(acc[i], b, a);
    }
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < 16; ++i) s += acc[i];
    if (s == 12345.678) out[0] = s;
}

}  // namespace ctb

extern "C" int ct_peak_probe(int kind, double *tflops) {
    using namespace ctb;
    if (!tflops) return CT_ERR_NULL;
    if (kind < 0 || kind > 1) return CT_ERR_MODE;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return CT_ERR_NO_DEVICE;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    double *buf = nullptr;
    if (cudaMalloc(&buf, 8) != cudaSuccess) return CT_ERR_NOMEM;
    const int blocks = sms * 8, threads = 256, iters = 4096;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double flops = 0.0;
    for (int rep = 0; rep < 2; ++rep) {  // first pass warms up clocks
        cudaEventRecord(e0);
        if (kind == 0) {
            probe_dmma<<<blocks, threads>>>(buf, iters);
            flops = (double)blocks * (threads / 32) * iters * 8 * (8.0 * 8 * 4 * 2);
        } else {
            probe_dfma<<<blocks, threads>>>(buf, iters);
            flops = (double)blocks * threads * iters * 16 * 2.0;
        }
        cudaEventRecord(e1);
    }
    cudaError_t err = cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(buf);
    if (err != cudaSuccess || ms <= 0.f) return CT_ERR_CUDA;
    *tflops = flops / (ms * 1e-3) / 1e12;
    return CT_OK;
}
