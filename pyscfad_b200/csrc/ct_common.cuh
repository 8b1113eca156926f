// Shared definitions for the B200 CCSD(T) kernels.
//
// Notation: o = nocc, v = nvir, n = nmo = o + v.  A "job" is one sorted virtual
// triple a >= b >= c (the reference's job list, pyscfadlib/.../vjp/cc/ccsd_t.c:6-72).
// Each job has six "terms" sigma = 0..5 with ordered triples
//   (x,y,z) = (a,b,c), (a,c,b), (b,a,c), (b,c,a), (c,a,b), (c,b,a)
// (get_wz, ccsd_t_vjp.c:32-37).  Term sigma's o^3 block
//   P[p,q,r] = sum_f vvop[x,y,p,o+f] t2T[z,f,q,r] - sum_l vooo[x,p,q,l] t2T[z,y,l,r]
// is scattered into the job's W through the permutation idx_sigma
// (_make_permute_indices, ccsd_t.c:74-96).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace ctb {

// packed job: a | b << 10 | c << 20 (nvir <= 1024)
__host__ __device__ inline int pack_job(int a, int b, int c) { return a | (b << 10) | (c << 20); }
__host__ __device__ inline void unpack_job(int j, int &a, int &b, int &c) {
    a = j & 1023; b = (j >> 10) & 1023; c = (j >> 20) & 1023;
}

// ordered triple of term sigma for job (a,b,c)
__host__ __device__ inline void term_xyz(int sigma, int a, int b, int c, int &x, int &y, int &z) {
    switch (sigma) {
    case 0: x = a; y = b; z = c; break;
    case 1: x = a; y = c; z = b; break;
    case 2: x = b; y = a; z = c; break;
    case 3: x = b; y = c; z = a; break;
    case 4: x = c; y = a; z = b; break;
    default: x = c; y = b; z = a; break;
    }
}

// Orbit slots: for a sorted occupied triple (i>=j>=k), slot s is the position
// (ijk[R(s,0)], ijk[R(s,1)], ijk[R(s,2)]),
//   R = (0,1,2) (0,2,1) (1,0,2) (1,2,0) (2,0,1) (2,1,0).
// COMP(s,t) is the slot of rearrangement R_t applied to slot s's position.
// With it, inside one orbit:
//   W[slot s]     = sum_sigma G_sigma[slot COMP(s,sigma)]     (w[idx_sigma(n)] += P_sigma[n])
//   z[slot s]     = sum_t R3C(t) y[slot COMP(s,t)]             (add_and_permute)
//   Wbar_sigma[s] = wbar[slot COMP(s,INV(sigma))]              (wabc_bar[n] = w0_bar[idx[n]])
__host__ __device__ constexpr int kR(int s, int m) {
    constexpr int T[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
    return T[s][m];
}
__host__ __device__ constexpr int kComp(int s, int t) {
    constexpr int T[6][6] = {{0, 1, 2, 3, 4, 5}, {1, 0, 4, 5, 2, 3}, {2, 3, 0, 1, 5, 4},
                             {3, 2, 5, 4, 0, 1}, {4, 5, 1, 0, 3, 2}, {5, 4, 3, 2, 1, 0}};
    return T[s][t];
}
__host__ __device__ constexpr int kInv(int s) {
    constexpr int T[6] = {0, 1, 2, 4, 3, 5};
    return T[s];
}
// r3 weights over R_t: identity 4, transpositions -2, 3-cycles 1 (ccsd_t.c:112-117)
__host__ __device__ constexpr double kR3C(int t) {
    constexpr double T[6] = {4.0, -2.0, -2.0, 1.0, 1.0, -2.0};
    return T[t];
}

// symmetry factor of a sorted job (get_d3 callers, ccsd_t_vjp.c:298-304)
__host__ __device__ inline double job_fac(int a, int b, int c) {
    return (a == c) ? (1.0 / 6.0) : ((a == b || b == c) ? 0.5 : 1.0);
}

// Neumaier compensated accumulation
struct KSum {
    double s = 0.0, c = 0.0;
    __host__ __device__ inline void add(double x) {
        double t = s + x;
        if (fabs(s) >= fabs(x)) c += (s - t) + x; else c += (x - t) + s;
        s = t;
    }
    __host__ __device__ inline double value() const { return s + c; }
};

#ifdef __CUDACC__
// d += a b on the float64 tensor pipe: one m8n8k4 MMA (row-major A, column-major
// B).  Fragments: lane i holds A[i/4][i%4], B[i%4][i/4] and D[i/4][2(i%4)..+1].
__device__ __forceinline__ void dmma(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}
#endif

}  // namespace ctb
