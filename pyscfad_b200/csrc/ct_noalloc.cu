// Allocation-free variant of the float64 (T) energy.
//
// Some callers cannot let a library allocate device memory: an XLA/JAX FFI
// handler runs inside a framework that owns all device memory through its own
// allocator, and latency-sensitive callers avoid cudaMalloc/cudaFree because
// those calls synchronize the device.  For them ct_energy_noalloc computes the
// same float64 energy as ct_energy without any allocation: the wave scratch,
// the per-job energies and the job list live in the file-scope device array
// below, of fixed capacity, which every GPU that loads this library holds
// until the process exits.  Every call reuses (and overwrites) that array, so
// calls that overlap on the GPU, e.g. on two streams, race with each other.
#include <cuda_runtime.h>
#include <mutex>
#include "ct_common.cuh"
#include "ct_internal.h"
#include "../../include/pyscfad_b200.h"

namespace ctb {

static __device__ __align__(256) double g_noalloc_scratch[CT_NOALLOC_SCRATCH_DOUBLES];

namespace {
std::mutex g_noalloc_mu;
int g_noalloc_dev_ready[64] = {0};
double *g_noalloc_ptr[64] = {nullptr};
}  // namespace

// job index J (a-major order over a>=b>=c) -> packed job
__global__ void noalloc_jobs_kernel(int *jobs, long long first, int count, int v) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < count; t += gridDim.x * blockDim.x) {
        const long long J = first + t;
        int a = 0;
        while (a + 1 < v && (long long)(a + 1) * (a + 2) * (a + 3) / 6 <= J) ++a;
        long long r = J - (long long)a * (a + 1) * (a + 2) / 6;
        int b = 0;
        while (b + 1 <= a && (long long)(b + 1) * (b + 2) / 2 <= r) ++b;
        const int c = (int)(r - (long long)b * (b + 1) / 2);
        jobs[t] = pack_job(a, b, c);
    }
}

}  // namespace ctb

extern "C" int ct_energy_noalloc(const ct_problem *p, double *e_out, void *stream) {
    using namespace ctb;
    if (!p || !e_out) return CT_ERR_NULL;
    if (p->nocc < 1 || p->nocc > 64 || p->nvir < 1 || p->nvir > 1024) return CT_ERR_SHAPE;
    if (!p->mo_energy || !p->t1T || !p->t2T || !p->vooo || !p->fvo || !p->vvop) return CT_ERR_NULL;
    const long long o = p->nocc, v = p->nvir, o3 = o * o * o;
    const long long njobs = v * (v + 1) * (v + 2) / 6;
    // layout (doubles): [job energies: njobs][job list: ceil(wave/2)][scratch: wave * 7 o^3];
    // a wave of w jobs needs w (7 o^3 + 1) doubles (the +1 covers the job
    // list) after the energies and 64 doubles of alignment slack, so a
    // problem fits when njobs + 7 o^3 + 65 <= CT_NOALLOC_SCRATCH_DOUBLES
    const long long per_job = kSlots * o3 + 1;
    const long long avail = (long long)CT_NOALLOC_SCRATCH_DOUBLES - njobs - 64;
    if (avail < per_job) return CT_ERR_SIZE;
    const long long wave = avail / per_job < njobs ? avail / per_job : njobs;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return CT_ERR_NO_DEVICE;
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_dev_ready[dev]) {
        // once per device: check the architecture, then look up the array's
        // device address (host code only has a stand-in symbol for it)
        int major = 0;
        if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess || major != 10)
            return CT_ERR_NO_DEVICE;
        void *ptr = nullptr;
        if (cudaGetSymbolAddress(&ptr, g_noalloc_scratch) != cudaSuccess || !ptr) return CT_ERR_CUDA;
        g_noalloc_ptr[dev] = static_cast<double *>(ptr);
        g_noalloc_dev_ready[dev] = 1;
    }
    double *base = g_noalloc_ptr[dev];
    double *job_e = base;
    int *jobs = reinterpret_cast<int *>(base + njobs);
    double *scratch = base + njobs + (wave + 1) / 2 + 1;
    scratch = reinterpret_cast<double *>((reinterpret_cast<uintptr_t>(scratch) + 255) & ~uintptr_t(255));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // the array keeps the previous call's contents: clear the per-job energies
    if (cudaMemsetAsync(job_e, 0, njobs * sizeof(double), st) != cudaSuccess) return CT_ERR_CUDA;
    EpiArgs ea{};
    ea.o = (int)o; ea.v = (int)v; ea.n = (int)(o + v);
    ea.mo_energy = p->mo_energy; ea.t1T = p->t1T; ea.t2T = p->t2T; ea.fvo = p->fvo; ea.vvop = p->vvop;
    ea.with_vjp = 0;
    ea.job_e = job_e;
    for (long long first = 0; first < njobs; first += wave) {
        const int count = (int)(njobs - first < wave ? njobs - first : wave);
        noalloc_jobs_kernel<<<(count + 255) / 256, 256, 0, st>>>(jobs, first, count, (int)v);
        if (cudaGetLastError() != cudaSuccess) return CT_ERR_CUDA;
        WaveView wv{};
        wv.o = (int)o; wv.v = (int)v; wv.n = (int)(o + v);
        wv.n_jobs = count;
        wv.jobs = jobs;
        if (f64_gemm(K_F1, wv, p->t2T, p->vvop, scratch, scratch, st) != cudaSuccess) return CT_ERR_CUDA;
        if (f64_gemm(K_F2, wv, p->vooo, p->t2T, scratch, scratch, st) != cudaSuccess) return CT_ERR_CUDA;
        if (f64_epilogue(wv, ea, scratch, st) != cudaSuccess) return CT_ERR_CUDA;
    }
    if (reduce_energy_1cta(job_e, njobs, e_out, st) != cudaSuccess) return CT_ERR_CUDA;
    return CT_OK;
}
