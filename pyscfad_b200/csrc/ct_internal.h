// Internal interfaces between the host orchestration (ct_host.cu) and the
// kernel translation units.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace ctb {

// GEMM kinds of one wave (offsets per (job, sigma) term; see entry_offsets)
enum GemmKind { K_F1 = 0, K_F2 = 1, K_VB = 2, K_TB = 3, K_OB1 = 4, K_OB2 = 5 };

struct WaveView {
    int o, v, n;
    int n_jobs;             // jobs in this wave
    const int *jobs;        // device, packed (a | b<<10 | c<<20), wave-local
    int n_tb_groups;        // K_TB groups (one per distinct z in the wave)
    const int *tb_entries;  // device, local term ids jl*6+sigma sorted by z
    const int *tb_groups;   // device, (z, e_begin, e_end) per group
    // mixed path: z-groups cut into chunks of <= 256/o terms, and the same
    // structure keyed by x (index ranges point into tb_entries / x_entries)
    int n_zchunks;
    const int *zchunks;
    const int *x_entries;
    int n_xgroups;
    const int *xgroups;
    int n_xchunks;
    const int *xchunks;
    int n_ochunks;        // x-sorted terms in chunks of <= 256 / o (OB2)
    const int *ochunks;
};

struct EpiArgs {
    int o, v, n;
    const double *mo_energy, *t1T, *t2T, *fvo, *vvop;
    double et_bar;
    int with_vjp;
    double *job_e;          // indexed by a-major job index a(a+1)(a+2)/6 + b(b+1)/2 + c
    double *mo_energy_bar;
    double *t1T_bar, *t2T_bar, *fvo_bar, *vvop_bar;
    const int *orbits;      // packed i | j<<8 | k<<16, i>=j>=k
    int n_orb;
    // BF16x3: W-bar goes to bf16 hi/lo planes here (plane jl*6+sigma of the
    // wave's 6 n_jobs planes: every hi plane, then every lo plane) instead of
    // the float slots; else null
    void *wbar_bf16;
    // mixed path: float copies of vvop[:,:,:,:o] (v,v,o,o) and t2T (v,v,o,o)
    // for the V-term tiles of the pipelined epilogue; null on the float64 path
    const float *vvoo_f, *t2_f;
    // LNO-projected energy (float64 path, no VJP): projector mat (o,o) on the
    // device, or null for the canonical energy; only orderings whose first
    // virtual index lies in [lno_a0, lno_a1) contribute
    const double *lno_mat;
    int lno_a0, lno_a1;
    // VJP slab block (lno_ccsd_t_vjp.c:355-398): an ordering (x, y, z) counts
    // when y in [lno_b0, lno_b1) and z in [lno_c0, lno_c1) (full ranges otherwise)
    int lno_b0, lno_b1, lno_c0, lno_c1;
    // 0: canonical; 1: LNO forward pass (W cube to slot 0, z/D to slot 1);
    // 2: LNO backward pass (reads z/D and the two parts of A and B from slots
    // 1-5, writes W-bar to slots 0-5 and ybar to slot 6)
    int lno_phase;
    double *lno_mat_bar_part;   // LNO VJP: per-job (o, o) partials of mat_bar
    // iterative (T) seed (float64 path, no VJP; null otherwise): each element
    // orbit writes P6(W + V) / D to t3_c and r3(P6(W)) / 3 to t3_x, both
    // (v, v, v, o, o, o) arrays [a][b][c][i][j][k], at every simultaneous
    // permutation of (a, b, c) and of the element's (i, j, k)
    double *t3_c, *t3_x;
};

// Raises a kernel's dynamic shared-memory limit to `bytes` on the current
// device.  The attribute belongs to each device's context, so it is applied
// once per (kernel, device), not once per process; thread-safe.
cudaError_t smem_optin(const void *kernel, int bytes);

// profiled kernel kinds (ct_profile_read)
enum ProfKind { PK_F1 = 0, PK_F2, PK_EPI, PK_VT, PK_VB, PK_TB, PK_OB1, PK_OB2, PK_RED,
                PK_MPREP, PK_MF, PK_MVB, PK_MTB, PK_MOO, PK_MOB1, PK_MOB2, kProfKinds };

// scratch layout per job: 7 slots of o^3 (slots 0..5: G_sigma then Wbar_sigma,
// slot 6: ybar = r3^T(zbar))
constexpr int kSlots = 7;

// float64 path (ct_fp64.cu)
cudaError_t f64_gemm(GemmKind kind, const WaveView &w, const double *A, const double *B, double *C,
                     double *scratch, cudaStream_t st);
cudaError_t f64_epilogue(const WaveView &w, const EpiArgs &e, double *scratch, cudaStream_t st);
cudaError_t f64_vterm(const WaveView &w, const EpiArgs &e, const double *scratch, cudaStream_t st);
// LNO projections (ct_lno.cu).  The energy of each job of the wave from the
// W and z/D cubes the epilogue leaves in slots 0 and 1 (writes e.job_e)
cudaError_t f64_lno_contract(const WaveView &w, const EpiArgs &e, const double *scratch, cudaStream_t st);
// LNO VJP: from slots 0-1 the projected cubes A, B in two parts each (axes
// 1-2 into slots 2, 3; axis 0 into slots 4, 5), each job's energy into
// e.job_e and its mat_bar partial into e.lno_mat_bar_part
cudaError_t f64_lno_vjp_project(const WaveView &w, const EpiArgs &e, double *scratch, cudaStream_t st);
// mat_bar += sum over the wave's jobs of the partials (fixed order)
cudaError_t f64_lno_mat_bar(const WaveView &w, const EpiArgs &e, double *mat_bar, cudaStream_t st);
// work: 2 * kReduceParts doubles of device scratch
constexpr int kReduceParts = 256;
cudaError_t reduce_energy(const double *job_e, long long n, double *e_out, double *work, cudaStream_t st);
// the same sum in one CTA (no work buffer; the allocation-free entry uses it)
cudaError_t reduce_energy_1cta(const double *job_e, long long n, double *e_out, cudaStream_t st);
// mixed path: the pipelined orbit epilogue (ct_epi_f32.cu) and the V-term kernel on float scratch
cudaError_t f32_epilogue(const WaveView &w, const EpiArgs &e, float *scratch, cudaStream_t st);
cudaError_t f32_vterm(const WaveView &w, const EpiArgs &e, const float *scratch, cudaStream_t st);
// the same two on the mixed path's float, qr-tiled slots
cudaError_t f32_lno_contract(const WaveView &w, const EpiArgs &e, const float *scratch, cudaStream_t st);
cudaError_t f32_lno_vjp_project(const WaveView &w, const EpiArgs &e, float *scratch, cudaStream_t st);

}  // namespace ctb
