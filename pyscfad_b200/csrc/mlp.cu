// Learned block surrogate: a 12-128-128-1 SiLU MLP over per-job features,
// trained on the GPU by the kernels below, and the feature kernels that feed
// it from the (T) inputs.
//
// A "block" is one sorted virtual triple (a >= b >= c): the unit of work of
// the (T) kernels, whose exact contribution the energy entries report per job.
//
// Parameters: one float32 vector of CT_MLP_NPARAM entries,
//   W1 [128][12] | b1 [128] | W2 [128][128] | b2 [128] | W3 [128] | b3
// Training: forward (keeps pre-activations) -> mse (loss, dL/dy) -> backward
// (per-sample deltas, then per-CTA partial gradients reduced in a fixed order,
// so gradients are deterministic) -> AdamW.  Inference: bf16 weights and
// activations on the tensor cores (mma.sync bf16), float32 accumulation.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cstdint>
#include "ct_common.cuh"
#include "ct_internal.h"
#include "../../include/pyscfad_b200.h"

namespace ctb {
namespace mlp {

constexpr int I = CT_MLP_IN, H = CT_MLP_HIDDEN;
constexpr int oW1 = 0, ob1 = H * I, oW2 = ob1 + H, ob2 = oW2 + H * H, oW3 = ob2 + H, ob3 = oW3 + H;
static_assert(ob3 + 1 == CT_MLP_NPARAM, "parameter layout");
constexpr int S = 32;               // samples per tile
constexpr int kGradCtas = 296;      // partial-gradient slots (2 per SM)

__device__ __forceinline__ float sigm(float z) { return 1.0f / (1.0f + __expf(-z)); }
__device__ __forceinline__ float silu(float z) { return z * sigm(z); }
__device__ __forceinline__ float dsilu(float z) {
    const float s = sigm(z);
    return s * (1.0f + z * (1.0f - s));
}

// ---------------------------------------------------------------- forward
// 128 threads (thread j = hidden unit j), persistent over 32-sample tiles.
__global__ void __launch_bounds__(128) forward_kernel(const float *__restrict__ P, const float *__restrict__ X,
                                                      int n, float *Z1, float *Z2, float *__restrict__ Y) {
    extern __shared__ float sm[];
    float *W2t = sm;                    // [k][j] = W2[j][k]
    float *A = W2t + H * H;             // [S][H] layer-1 activations, then W3-weighted layer-2 terms
    float *Xs = A + S * H;              // [S][I]
    const int j = threadIdx.x;
    for (int k = 0; k < H; ++k) W2t[k * H + j] = P[oW2 + j * H + k];
    float w1[I];
#pragma unroll
    for (int m = 0; m < I; ++m) w1[m] = P[oW1 + j * I + m];
    const float b1 = P[ob1 + j], b2 = P[ob2 + j], w3 = P[oW3 + j], b3 = P[ob3];
    const int ntile = (n + S - 1) / S;
    for (int tile = blockIdx.x; tile < ntile; tile += gridDim.x) {
        const int s0 = tile * S, ns = min(S, n - s0);
        __syncthreads();
        for (int e = j; e < S * I; e += H) Xs[e] = (e / I < ns) ? X[(size_t)s0 * I + e] : 0.0f;
        __syncthreads();
        for (int s = 0; s < S; ++s) {
            float z = b1;
#pragma unroll
            for (int m = 0; m < I; ++m) z = fmaf(w1[m], Xs[s * I + m], z);
            A[s * H + j] = silu(z);
            if (Z1 && s < ns) Z1[(size_t)(s0 + s) * H + j] = z;
        }
        __syncthreads();
        float acc[S];
#pragma unroll
        for (int s = 0; s < S; ++s) acc[s] = b2;
        for (int k = 0; k < H; ++k) {
            const float w = W2t[k * H + j];
#pragma unroll
            for (int s = 0; s < S; ++s) acc[s] = fmaf(w, A[s * H + k], acc[s]);
        }
        __syncthreads();
#pragma unroll
        for (int s = 0; s < S; ++s) {
            if (Z2 && s < ns) Z2[(size_t)(s0 + s) * H + j] = acc[s];
            A[s * H + j] = w3 * silu(acc[s]);
        }
        __syncthreads();
        // thread s (< 32) sums row s in a fixed order
        if (j < S && j < ns) {
            float y = b3;
            for (int k = 0; k < H; ++k) y += A[j * H + ((k + j) & (H - 1))];
            Y[s0 + j] = y;
        }
    }
}

// ---------------------------------------------------------------- loss
// L = (1/n) sum (y - t)^2, dY = 2 (y - t) / n; one CTA, fixed-order reduction.
__global__ void __launch_bounds__(1024) mse_kernel(const float *Y, const float *T, int n, float *dY, double *loss) {
    __shared__ double red[1024];
    double acc = 0.0;
    const float inv = 1.0f / (float)n;
    for (int s = threadIdx.x; s < n; s += blockDim.x) {
        const float d = Y[s] - T[s];
        if (dY) dY[s] = 2.0f * d * inv;
        acc += (double)d * d;
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int w = 512; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0 && loss) *loss = red[0] / n;
}

// ---------------------------------------------------------------- backward
// per-sample deltas: D2[s][j] = dY[s] W3[j] silu'(Z2[s][j]);
//                    D1[s][k] = silu'(Z1[s][k]) sum_j D2[s][j] W2[j][k]
__global__ void __launch_bounds__(128) delta_kernel(const float *__restrict__ P, const float *__restrict__ Z1,
                                                    const float *__restrict__ Z2, const float *__restrict__ dY,
                                                    int n, float *__restrict__ D1, float *__restrict__ D2) {
    extern __shared__ float sm[];
    float *W2s = sm;               // [j][k], natural layout
    float *Ds = W2s + H * H;       // [S][H]
    const int k = threadIdx.x;
    for (int jj = 0; jj < H; ++jj) W2s[jj * H + k] = P[oW2 + jj * H + k];
    const float w3 = P[oW3 + k];
    const int ntile = (n + S - 1) / S;
    for (int tile = blockIdx.x; tile < ntile; tile += gridDim.x) {
        const int s0 = tile * S, ns = min(S, n - s0);
        __syncthreads();
        for (int s = 0; s < S; ++s) {
            float d = 0.0f;
            if (s < ns) {
                d = dY[s0 + s] * w3 * dsilu(Z2[(size_t)(s0 + s) * H + k]);
                D2[(size_t)(s0 + s) * H + k] = d;
            }
            Ds[s * H + k] = d;
        }
        __syncthreads();
        float acc[S];
#pragma unroll
        for (int s = 0; s < S; ++s) acc[s] = 0.0f;
        for (int jj = 0; jj < H; ++jj) {
            const float w = W2s[jj * H + k];
#pragma unroll
            for (int s = 0; s < S; ++s) acc[s] = fmaf(w, Ds[s * H + jj], acc[s]);
        }
#pragma unroll
        for (int s = 0; s < S; ++s)
            if (s < ns) D1[(size_t)(s0 + s) * H + k] = acc[s] * dsilu(Z1[(size_t)(s0 + s) * H + k]);
    }
}

// per-CTA partial parameter gradients over a strided set of tiles, written to
// part[blockIdx.x][NPARAM] (256 threads)
__global__ void __launch_bounds__(256) grad_kernel(const float *__restrict__ X, const float *__restrict__ Z1,
                                                   const float *__restrict__ Z2, const float *__restrict__ dY,
                                                   const float *__restrict__ D1, const float *__restrict__ D2,
                                                   int n, float *__restrict__ part) {
    extern __shared__ float sm[];
    float *D2s = sm;                 // [S][H]
    float *A1s = D2s + S * H;        // [S][H]
    float *D1s = A1s + S * H;        // [S][H]
    float *A2s = D1s + S * H;        // [S][H]
    float *Xs = A2s + S * H;         // [S][I]
    float *dYs = Xs + S * I;         // [S]
    const int t = threadIdx.x;
    const int jr = t >> 1, kp = t & 1;   // gW2 rows jr, columns kp + 2 kk
    float g2[64];
#pragma unroll
    for (int kk = 0; kk < 64; ++kk) g2[kk] = 0.0f;
    float g1[6] = {0, 0, 0, 0, 0, 0};    // gW1 entries t + 256 q (of 1536)
    float gsmall = 0.0f, gb3 = 0.0f;     // t < 128: gb1[t]; else gW3[t-128]
    float gb2 = 0.0f;                    // t < 128: gb2[t]
    const int ntile = (n + S - 1) / S;
    for (int tile = blockIdx.x; tile < ntile; tile += gridDim.x) {
        const int s0 = tile * S, ns = min(S, n - s0);
        __syncthreads();
        for (int e = t; e < S * H; e += 256) {
            const int s = e / H;
            const size_t g = (size_t)s0 * H + e;
            const bool ok = s < ns;
            D2s[e] = ok ? D2[g] : 0.0f;
            A1s[e] = ok ? silu(Z1[g]) : 0.0f;
            D1s[e] = ok ? D1[g] : 0.0f;
            A2s[e] = ok ? silu(Z2[g]) : 0.0f;
        }
        for (int e = t; e < S * I; e += 256) Xs[e] = (e / I < ns) ? X[(size_t)s0 * I + e] : 0.0f;
        if (t < S) dYs[t] = t < ns ? dY[s0 + t] : 0.0f;
        __syncthreads();
        for (int s = 0; s < S; ++s) {
            const float d = D2s[s * H + jr];
#pragma unroll
            for (int kk = 0; kk < 64; ++kk) g2[kk] = fmaf(d, A1s[s * H + kp + 2 * kk], g2[kk]);
        }
#pragma unroll
        for (int q = 0; q < 6; ++q) {
            const int e = t + 256 * q, kr = e / I, m = e % I;
            float acc = g1[q];
            for (int s = 0; s < S; ++s) acc = fmaf(D1s[s * H + kr], Xs[s * I + m], acc);
            g1[q] = acc;
        }
        if (t < H) {
            for (int s = 0; s < S; ++s) { gsmall += D1s[s * H + t]; gb2 += D2s[s * H + t]; }
        } else {
            for (int s = 0; s < S; ++s) gsmall = fmaf(dYs[s], A2s[s * H + t - H], gsmall);
        }
        if (t == 0)
            for (int s = 0; s < S; ++s) gb3 += dYs[s];
    }
    float *out = part + (size_t)blockIdx.x * CT_MLP_NPARAM;
#pragma unroll
    for (int kk = 0; kk < 64; ++kk) out[oW2 + jr * H + kp + 2 * kk] = g2[kk];
#pragma unroll
    for (int q = 0; q < 6; ++q) out[oW1 + t + 256 * q] = g1[q];
    if (t < H) { out[ob1 + t] = gsmall; out[ob2 + t] = gb2; }
    else out[oW3 + t - H] = gsmall;
    if (t == 0) out[ob3] = gb3;
}

__global__ void reduce_parts_kernel(const float *part, int nparts, float *grad) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= CT_MLP_NPARAM) return;
    float acc = 0.0f;
    for (int c = 0; c < nparts; ++c) acc += part[(size_t)c * CT_MLP_NPARAM + e];
    grad[e] = acc;
}

// ---------------------------------------------------------------- AdamW
__global__ void adam_kernel(float *P, const float *G, float *M, float *V, int step, float lr, float b1, float b2,
                            float eps, float wd) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= CT_MLP_NPARAM) return;
    const float g = G[e];
    const float m = b1 * M[e] + (1.0f - b1) * g;
    const float v = b2 * V[e] + (1.0f - b2) * g * g;
    M[e] = m;
    V[e] = v;
    const float mh = m / (1.0f - powf(b1, (float)step));
    const float vh = v / (1.0f - powf(b2, (float)step));
    float p = P[e];
    p -= lr * (mh / (sqrtf(vh) + eps) + wd * p);
    P[e] = p;
}

// ---------------------------------------------------------------- bf16 inference
__global__ void to_bf16_kernel(const float *P, __nv_bfloat16 *Q) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < CT_MLP_NPARAM) Q[e] = __float2bfloat16_rn(P[e]);
}

__device__ __forceinline__ float rbf(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// bf16 tensor-core inference (mma.sync m16n8k16, float32 accumulation): each
// warp takes 16 samples; layer 1 (K = 12, padded to 16) and layer 2 (K = 128)
// run as MMAs, and the layer-1 accumulators, after SiLU and rounding to bf16,
// are already the A fragments of layer 2 (two 8-column C tiles = one 16-wide
// K step), so activations never touch shared memory.  Layer 3 is a dot
// product reduced over the four lanes that share a row.
constexpr int kInferWarps = 4;
constexpr int kW2Ld = H + 8;     // padded bf16 row of W2 in shared memory (conflict-free B fragments)
constexpr int kW1Ld = 16 + 8;    // W1 rows padded to K = 16 (+8 against bank conflicts)

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t *>(&v);
}

__device__ __forceinline__ void mma_bf16_16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__global__ void __launch_bounds__(32 * kInferWarps) infer_bf16_kernel(const __nv_bfloat16 *__restrict__ Q,
                                                                      const float *__restrict__ X, int n,
                                                                      float *__restrict__ Y) {
    extern __shared__ float sm[];
    __nv_bfloat16 *W2s = reinterpret_cast<__nv_bfloat16 *>(sm);   // [j][kW2Ld]: W2[j][k]
    __nv_bfloat16 *W1s = W2s + H * kW2Ld;                         // [j][kW1Ld]: W1[j][m], m >= 12 zero
    float *bias = reinterpret_cast<float *>(W1s + H * kW1Ld);     // b1[128] | b2[128] | W3[128]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int e = tid; e < H * H; e += blockDim.x) W2s[(e / H) * kW2Ld + e % H] = Q[oW2 + e];
    for (int e = tid; e < H * 16; e += blockDim.x) {
        const int j = e / 16, m = e % 16;
        W1s[j * kW1Ld + m] = m < I ? Q[oW1 + j * I + m] : __float2bfloat16_rn(0.0f);
    }
    for (int e = tid; e < H; e += blockDim.x) {
        bias[e] = __bfloat162float(Q[ob1 + e]);
        bias[H + e] = __bfloat162float(Q[ob2 + e]);
        bias[2 * H + e] = __bfloat162float(Q[oW3 + e]);
    }
    const float b3 = __bfloat162float(Q[ob3]);
    __syncthreads();
    const int g = lane >> 2, c2 = (lane & 3) * 2;   // fragment row group, column pair
    const int ntile = (n + 16 * kInferWarps - 1) / (16 * kInferWarps);
    for (int tile = blockIdx.x; tile < ntile; tile += gridDim.x) {
        const int s0 = tile * 16 * kInferWarps + warp * 16;
        // layer-1 A fragment: rows g, g+8 of the warp's 16 samples; features c2, c2+1 (+8)
        uint32_t a1[4];
        {
            float x[2][4];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int s = s0 + g + 8 * h;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int m = c2 + (q & 1) + 8 * (q >> 1);
                    x[h][q] = (s < n && m < I) ? X[(size_t)s * I + m] : 0.0f;
                }
            }
            a1[0] = pack_bf16(x[0][0], x[0][1]);
            a1[1] = pack_bf16(x[1][0], x[1][1]);
            a1[2] = pack_bf16(x[0][2], x[0][3]);
            a1[3] = pack_bf16(x[1][2], x[1][3]);
        }
        // layer 1 -> SiLU -> bf16 A fragments of layer 2 (k-step t = C tiles 2t, 2t+1)
        uint32_t a2[H / 16][4];
#pragma unroll
        for (int nt = 0; nt < H / 8; ++nt) {
            const int j = nt * 8 + g;   // B fragment column
            const uint32_t b0 = *reinterpret_cast<const uint32_t *>(W1s + j * kW1Ld + c2);
            const uint32_t b1 = *reinterpret_cast<const uint32_t *>(W1s + j * kW1Ld + c2 + 8);
            const int col = nt * 8 + c2;
            float d[4] = {bias[col], bias[col + 1], bias[col], bias[col + 1]};
            mma_bf16_16816(d, a1, b0, b1);
            const uint32_t lo = pack_bf16(silu(d[0]), silu(d[1])), hi = pack_bf16(silu(d[2]), silu(d[3]));
            a2[nt >> 1][(nt & 1) * 2 + 0] = lo;
            a2[nt >> 1][(nt & 1) * 2 + 1] = hi;
        }
        // layer 2 and the layer-3 dot product
        float y0 = 0.0f, y1 = 0.0f;   // rows g and g + 8
#pragma unroll
        for (int nt = 0; nt < H / 8; ++nt) {
            const int j = nt * 8 + g, col = nt * 8 + c2;
            float d[4] = {bias[H + col], bias[H + col + 1], bias[H + col], bias[H + col + 1]};
#pragma unroll
            for (int kt = 0; kt < H / 16; ++kt) {
                const uint32_t b0 = *reinterpret_cast<const uint32_t *>(W2s + j * kW2Ld + kt * 16 + c2);
                const uint32_t b1 = *reinterpret_cast<const uint32_t *>(W2s + j * kW2Ld + kt * 16 + c2 + 8);
                mma_bf16_16816(d, a2[kt], b0, b1);
            }
            const float w0 = bias[2 * H + col], w1 = bias[2 * H + col + 1];
            y0 += w0 * rbf(silu(d[0])) + w1 * rbf(silu(d[1]));
            y1 += w0 * rbf(silu(d[2])) + w1 * rbf(silu(d[3]));
        }
        // the four lanes of a row group hold disjoint columns: fixed-order butterfly
        y0 += __shfl_xor_sync(0xffffffffu, y0, 1);
        y0 += __shfl_xor_sync(0xffffffffu, y0, 2);
        y1 += __shfl_xor_sync(0xffffffffu, y1, 1);
        y1 += __shfl_xor_sync(0xffffffffu, y1, 2);
        if ((lane & 3) == 0) {
            if (s0 + g < n) Y[s0 + g] = y0 + b3;
            if (s0 + g + 8 < n) Y[s0 + g + 8] = y1 + b3;
        }
    }
}

// ---------------------------------------------------------------- features
// Pair statistics of virtual pair (x, y), one CTA each (128 threads):
//   st[0][x][y] = ||t2T[x,y]||_F                       (t2 block norm)
//   st[1][x][y] = sum_ij t2T[x,y,j,i] (2 vvop[x,y,i,j] - vvop[y,x,i,j])
//                                                       (MP2 pair energy of x,y)
//   st[2][x][y] = ||vvop[x,y,:,o:]||_F                  (vvov block norm)
__global__ void __launch_bounds__(128) pair_stats_kernel(int o, int v, const double *__restrict__ t2T,
                                                         const double *__restrict__ vvop, float *st) {
    const int x = blockIdx.x / v, y = blockIdx.x % v, n = o + v;
    const double *T = t2T + ((size_t)x * v + y) * o * o;
    const double *Kxy = vvop + ((size_t)x * v + y) * o * n;
    const double *Kyx = vvop + ((size_t)y * v + x) * o * n;
    double tn = 0.0, e2 = 0.0, vn = 0.0;
    for (int e = threadIdx.x; e < o * o; e += blockDim.x) {
        const int j = e / o, i = e % o;
        const double t = T[e];   // t2T[x,y,j,i]
        tn += t * t;
        e2 += t * (2.0 * Kxy[(size_t)i * n + j] - Kyx[(size_t)i * n + j]);
    }
    for (int e = threadIdx.x; e < o * v; e += blockDim.x) {
        const double q = Kxy[(size_t)(e / v) * n + o + e % v];
        vn += q * q;
    }
    __shared__ double red[3][128];
    red[0][threadIdx.x] = tn; red[1][threadIdx.x] = e2; red[2][threadIdx.x] = vn;
    __syncthreads();
    for (int w = 64; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int q = 0; q < 3; ++q) red[q][threadIdx.x] += red[q][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const size_t vv = (size_t)v * v, xy = (size_t)x * v + y;
        st[xy] = (float)sqrt(red[0][0]);
        st[vv + xy] = (float)red[1][0];
        st[2 * vv + xy] = (float)sqrt(red[2][0]);
    }
}

// 12 features of each packed job (a >= b >= c); pairs in the order (a,b), (a,c), (b,c):
//   f0-2  log(t2 block norm of the pair, 1e-30 floor)
//   f3-5  asinh(MP2 pair energy / 1e-4)
//   f6-8  log(vvov block norms of (x,y) and (y,x) in quadrature)
//   f9    e_a + e_b + e_c - 3 e_homo         (smallest denominator of the job)
//   f10   e_a + e_b + e_c - 3 mean(e_occ)    (mean denominator)
//   f11   log of the job's orbit size (6, 3 or 1 orderings)
__global__ void job_features_kernel(int o, int v, const double *__restrict__ mo_energy, const int *__restrict__ jobs,
                                    long long njobs, const float *__restrict__ st, float *__restrict__ F) {
    __shared__ double occ_stats[2];
    if (threadIdx.x == 0) {
        double mx = mo_energy[0], sum = 0.0;
        for (int i = 0; i < o; ++i) { mx = fmax(mx, mo_energy[i]); sum += mo_energy[i]; }
        occ_stats[0] = mx; occ_stats[1] = sum / o;
    }
    __syncthreads();
    const size_t vv = (size_t)v * v;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < njobs;
         t += (long long)gridDim.x * blockDim.x) {
        int a, b, c;
        unpack_job(jobs[t], a, b, c);
        const int px[3] = {a, a, b}, py[3] = {b, c, c};
        float f[CT_MLP_IN];
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            const size_t xy = (size_t)px[q] * v + py[q], yx = (size_t)py[q] * v + px[q];
            f[q] = logf(fmaxf(st[xy], 1e-30f));
            f[3 + q] = asinhf(st[vv + xy] * 1e4f);
            const float n1 = st[2 * vv + xy], n2 = st[2 * vv + yx];
            f[6 + q] = 0.5f * logf(fmaxf(n1 * n1 + n2 * n2, 1e-30f));
        }
        const double eabc = mo_energy[o + a] + mo_energy[o + b] + mo_energy[o + c];
        f[9] = (float)(eabc - 3.0 * occ_stats[0]);
        f[10] = (float)(eabc - 3.0 * occ_stats[1]);
        f[11] = logf(a == c ? 1.0f : ((a == b || b == c) ? 3.0f : 6.0f));
#pragma unroll
        for (int q = 0; q < CT_MLP_IN; ++q) F[(size_t)t * CT_MLP_IN + q] = f[q];
    }
}

static int grid_for(int n, int per_sm) {
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int tiles = (n + S - 1) / S;
    return tiles < sms * per_sm ? (tiles > 0 ? tiles : 1) : sms * per_sm;
}

constexpr size_t kFwdSmem = (size_t)(H * H + S * H + S * I) * sizeof(float);
constexpr size_t kDeltaSmem = (size_t)(H * H + S * H) * sizeof(float);
constexpr size_t kGradSmem = (size_t)(4 * S * H + S * I + S) * sizeof(float);
constexpr size_t kInferSmem = (size_t)(H * kW2Ld + H * kW1Ld) * sizeof(__nv_bfloat16) + 3 * H * sizeof(float);

// the limits are per device context: smem_optin applies each once per device
static cudaError_t set_smem() {
    cudaError_t e;
    if ((e = smem_optin(reinterpret_cast<const void *>(forward_kernel), (int)kFwdSmem))) return e;
    if ((e = smem_optin(reinterpret_cast<const void *>(delta_kernel), (int)kDeltaSmem))) return e;
    if ((e = smem_optin(reinterpret_cast<const void *>(grad_kernel), (int)kGradSmem))) return e;
    if ((e = smem_optin(reinterpret_cast<const void *>(infer_bf16_kernel), (int)kInferSmem))) return e;
    return cudaSuccess;
}

static int status(cudaError_t e) { return e == cudaSuccess ? CT_OK : CT_ERR_CUDA; }

}  // namespace mlp
}  // namespace ctb

using namespace ctb::mlp;

extern "C" {

long long ct_mlp_work_floats(int n) {
    if (n < 1) return -1;
    return 2LL * n * H + (long long)kGradCtas * CT_MLP_NPARAM;
}

int ct_mlp_forward(const float *params, const float *X, int n, float *Z1, float *Z2, float *Y, void *stream) {
    if (!params || !X || !Y) return CT_ERR_NULL;
    if (n < 1) return CT_ERR_SHAPE;
    if (set_smem() != cudaSuccess) return CT_ERR_CUDA;
    forward_kernel<<<grid_for(n, 2), 128, kFwdSmem, (cudaStream_t)stream>>>(params, X, n, Z1, Z2, Y);
    return status(cudaGetLastError());
}

int ct_mlp_mse(const float *Y, const float *T, int n, float *dY, double *loss, void *stream) {
    if (!Y || !T) return CT_ERR_NULL;
    if (n < 1) return CT_ERR_SHAPE;
    mse_kernel<<<1, 1024, 0, (cudaStream_t)stream>>>(Y, T, n, dY, loss);
    return status(cudaGetLastError());
}

int ct_mlp_backward(const float *params, const float *X, const float *Z1, const float *Z2, const float *dY, int n,
                    float *grad, float *work, void *stream) {
    if (!params || !X || !Z1 || !Z2 || !dY || !grad || !work) return CT_ERR_NULL;
    if (n < 1) return CT_ERR_SHAPE;
    if (set_smem() != cudaSuccess) return CT_ERR_CUDA;
    cudaStream_t st = (cudaStream_t)stream;
    float *D1 = work, *D2 = work + (size_t)n * H, *part = work + 2 * (size_t)n * H;
    delta_kernel<<<grid_for(n, 2), 128, kDeltaSmem, st>>>(params, Z1, Z2, dY, n, D1, D2);
    const int g = grid_for(n, 2) < kGradCtas ? grid_for(n, 2) : kGradCtas;
    grad_kernel<<<g, 256, kGradSmem, st>>>(X, Z1, Z2, dY, D1, D2, n, part);
    reduce_parts_kernel<<<(CT_MLP_NPARAM + 255) / 256, 256, 0, st>>>(part, g, grad);
    return status(cudaGetLastError());
}

int ct_mlp_adam(float *params, const float *grad, float *m, float *v, int step, float lr, float beta1, float beta2,
                float eps, float weight_decay, void *stream) {
    if (!params || !grad || !m || !v) return CT_ERR_NULL;
    if (step < 1) return CT_ERR_SHAPE;
    adam_kernel<<<(CT_MLP_NPARAM + 255) / 256, 256, 0, (cudaStream_t)stream>>>(params, grad, m, v, step, lr, beta1,
                                                                               beta2, eps, weight_decay);
    return status(cudaGetLastError());
}

int ct_mlp_to_bf16(const float *params, void *params_bf16, void *stream) {
    if (!params || !params_bf16) return CT_ERR_NULL;
    to_bf16_kernel<<<(CT_MLP_NPARAM + 255) / 256, 256, 0, (cudaStream_t)stream>>>(
        params, static_cast<__nv_bfloat16 *>(params_bf16));
    return status(cudaGetLastError());
}

int ct_mlp_infer_bf16(const void *params_bf16, const float *X, int n, float *Y, void *stream) {
    if (!params_bf16 || !X || !Y) return CT_ERR_NULL;
    if (n < 1) return CT_ERR_SHAPE;
    if (set_smem() != cudaSuccess) return CT_ERR_CUDA;
    const int tiles = (n + 16 * kInferWarps - 1) / (16 * kInferWarps);
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int grid = tiles < 4 * sms ? tiles : 4 * sms;
    infer_bf16_kernel<<<grid, 32 * kInferWarps, kInferSmem, (cudaStream_t)stream>>>(
        static_cast<const __nv_bfloat16 *>(params_bf16), X, n, Y);
    return status(cudaGetLastError());
}

int ct_surrogate_features(const ct_problem *p, const int *jobs, long long njobs, float *pair_work, float *F,
                          void *stream) {
    if (!p || !jobs || !pair_work || !F || !p->mo_energy || !p->t2T || !p->vvop) return CT_ERR_NULL;
    if (p->nocc < 1 || p->nocc > 255 || p->nvir < 1 || p->nvir > 1024 || njobs < 1) return CT_ERR_SHAPE;
    cudaStream_t st = (cudaStream_t)stream;
    pair_stats_kernel<<<p->nvir * p->nvir, 128, 0, st>>>(p->nocc, p->nvir, p->t2T, p->vvop, pair_work);
    const long long blocks = (njobs + 255) / 256;
    job_features_kernel<<<(int)(blocks < 4096 ? blocks : 4096), 256, 0, st>>>(p->nocc, p->nvir, p->mo_energy, jobs,
                                                                              njobs, pair_work, F);
    return status(cudaGetLastError());
}

}  // extern "C"
