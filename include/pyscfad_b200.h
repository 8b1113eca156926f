/*
 * pyscfad_b200 C-ABI: B200 (sm_100a) CCSD(T) perturbative-triples energy and
 * its hand-written vector-Jacobian product.
 *
 * Every entry point is extern "C" with plain pointers and sizes.  Tensors use
 * the layouts pyscfad's (T) VJP driver builds (pyscfad/cc/ccsd_t.py:88-106):
 *
 *   mo_energy (nmo)                 orbital energies, occupied first
 *   t1T       (nvir, nocc)          t1 transposed
 *   t2T       (nvir, nvir, nocc, nocc)  t2[i,j,a,b] stored at [a,b,j,i]
 *   vooo      (nvir, nocc, nocc, nocc)  ovoo.transpose(1,0,3,2)
 *   fvo       (nvir, nocc)          fock[nocc:, :nocc]
 *   vvop      (nvir, nvir, nocc, nmo)   [ovov | ovvv] transposed (1,3,0,2)
 *
 * all C-contiguous float64.  Gradient buffers ACCUMULATE (+=), as the
 * reference's do (ccsd_t_vjp.c:332-497): callers zero them first.
 *
 * Status codes: 0 on success, a negative CT_ERR_* otherwise; nothing throws
 * across the ABI.  Device-pointer entry points are stream-ordered: they
 * enqueue work on `stream` (a cudaStream_t, NULL = legacy default stream) and
 * return; host-pointer entry points block until their results are on the host.
 */
#ifndef PYSCFAD_B200_H
#define PYSCFAD_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define CT_OK               0
#define CT_ERR_SHAPE       -1   /* nocc/nvir/slab bounds out of range */
#define CT_ERR_NOMEM       -2   /* device or pinned allocation failed */
#define CT_ERR_CUDA        -3   /* a CUDA call or kernel launch failed */
#define CT_ERR_MODE        -4   /* unknown precision mode */
#define CT_ERR_NULL        -5   /* a required pointer is NULL */
#define CT_ERR_NO_DEVICE   -6   /* no sm_100 device visible */
#define CT_ERR_TIMEOUT     -7   /* a bounded device-side wait gave up */
#define CT_ERR_NONFINITE   -8   /* the energy came out NaN/Inf */
#define CT_ERR_SIZE        -9   /* request exceeds a fixed capacity */

/* contraction precision of the W/V build and the backward GEMMs; orbital-energy
 * denominators, per-job energies and the final reduction are float64 in every
 * mode */
#define CT_MODE_FP64    0   /* float64 throughout (the drop-in path) */
#define CT_MODE_TF32    1   /* tcgen05 kind::tf32 tiles, float32 accumulate */
#define CT_MODE_BF16X3  2   /* tcgen05 bf16 hi/lo split, 3 products, float32 accumulate */
/* the tcgen05 modes need nocc % 8 == 0 and nocc <= 64 (else CT_ERR_SHAPE) */

typedef struct {
    int nocc;
    int nvir;
    const double *mo_energy;
    const double *t1T;
    const double *t2T;
    const double *vooo;
    const double *fvo;
    const double *vvop;
} ct_problem;

typedef struct {
    double *mo_energy;
    double *t1T;
    double *t2T;
    double *vooo;
    double *fvo;
    double *vvop;
} ct_grads;

/* Library / device information. */
int ct_version(void);
const char *ct_status_string(int status);

/*
 * Canonical (T) energy on the device.
 *   e_out      device pointer to one double, receives E(T)
 *   job_e_out  nullable device pointer to nvir(nvir+1)(nvir+2)/6 doubles, receives the
 *              per-(a>=b>=c) job contributions in a-major order (they sum to E(T))
 * Replaces the forward energy of pyscfad/cc/ccsd_t.py:41 (PySCF's kernel) and
 * lnoccsdt_contract with mat = I (pyscfadlib/pyscfadlib/vjp/cc/lno_ccsd_t.c:96-138,
 * x2/3 as pyscfad/lno/ccsd_t.py:111 applies).
 */
int ct_energy(const ct_problem *p, int mode, double *e_out, double *job_e_out, void *stream);

/*
 * Energy and VJP in one pass (W/V recomputed per job, never stored beyond the
 * current wave).  et_bar follows the C kernel's convention: the value the
 * reference's ccsd_t_energy_vjp receives, i.e. twice the cotangent of E(T)
 * (pyscfad/cc/ccsd_t.py:86).  e_out (device, nullable) receives E(T).
 * Replaces ccsd_t_energy_vjp (pyscfadlib/pyscfadlib/vjp/cc/ccsd_t_vjp.c:332-497)
 * over the full (0,nvir,0,nvir) block.
 */
int ct_energy_vjp(const ct_problem *p, int mode, double et_bar, const ct_grads *g,
                  double *e_out, void *stream);

/*
 * Host-pointer drop-in with the exact argument list of the reference's
 * ccsd_t_energy_vjp (ccsd_t_vjp.c:332-346), including the (a0,a1,b0,b1) slab
 * block and its row/col caches (pyscfad/cc/ccsd_t.py:108-177).  Runs the FP64
 * path on the current device; blocks until the accumulated gradients are back.
 * Returns a status instead of void.
 */
int ctb_ccsd_t_energy_vjp(double *mo_energy, double *t1T, double *t2T,
                          double *vooo, double *fvo, double et_bar,
                          int nocc, int nvir, int a0, int a1, int b0, int b1,
                          void *cache_row_a, void *cache_col_a,
                          void *cache_row_b, void *cache_col_b,
                          double *mo_energy_bar, double *t1T_bar, double *t2T_bar,
                          double *vooo_bar, double *fvo_bar,
                          double *cache_row_a_bar, double *cache_col_a_bar,
                          double *cache_row_b_bar, double *cache_col_b_bar);

/* Same, with a precision mode. */
int ctb_ccsd_t_energy_vjp_mode(double *mo_energy, double *t1T, double *t2T,
                               double *vooo, double *fvo, double et_bar,
                               int nocc, int nvir, int a0, int a1, int b0, int b1,
                               void *cache_row_a, void *cache_col_a,
                               void *cache_row_b, void *cache_col_b,
                               double *mo_energy_bar, double *t1T_bar, double *t2T_bar,
                               double *vooo_bar, double *fvo_bar,
                               double *cache_row_a_bar, double *cache_col_a_bar,
                               double *cache_row_b_bar, double *cache_col_b_bar, int mode);

/*
 * Host-pointer canonical energy over the jobs a0 <= a < a1 (all b, c with
 * a>=b>=c); (0, nvir) gives E(T).  vvop is the full (nvir,nvir,nocc,nmo) array.
 * Mirrors the forward call of pyscfad/cc/ccsd_t.py:41 (whole array) and
 * lnoccsdt_contract's a-slab argument (lno_ccsd_t.c:96-100) with mat = I.
 */
int ctb_ccsd_t_energy(double *e_tot, double *mo_energy, double *t1T, double *t2T,
                      double *vooo, double *fvo, int nocc, int nvir, int a0, int a1,
                      double *vvop, int mode);

/*
 * Host-pointer drop-in for lnoccsdt_contract (lno_ccsd_t.c:96-100): the same
 * argument list with the slab cache replaced by the full vvop array; adds the
 * LNO-projected energy of the a-slab [a0, a1) to *e_tot (float64 path).
 */
int ctb_lnoccsdt_contract(double *e_tot, double *mat, double *mo_energy, double *t1T,
                          double *t2T, double *vooo, double *fvo, int nocc, int nvir,
                          int a0, int a1, double *vvop);

/*
 * Host-pointer drop-in with the exact argument list of lnoccsdt_energy_vjp
 * (lno_ccsd_t_vjp.c:400-414): the slab block (b0, b1, c0, c1) and the caches
 * pyscfad's LNO backward cuts (pyscfad/lno/ccsd_t.py:194-220: rows
 * vvop[s0:s1, :], columns vvop[:, s0:s1], one array for the slab [0, nvir)).
 * mat_bar and the other gradients accumulate.  Each vvop pair's gradient is
 * added to exactly one cache gradient (the driver only uses their sums).
 * Float64 path; blocks until the gradients are back.
 */
int ctb_lnoccsdt_energy_vjp(double *mat, double *mo_energy, double *t1T, double *t2T,
                            double *vooo, double *fvo, double et_bar, int nocc, int nvir,
                            int b0, int b1, int c0, int c1,
                            void *cache_row_a, void *cache_col_a,
                            void *cache_row_b, void *cache_col_b,
                            double *mat_bar, double *mo_energy_bar, double *t1T_bar,
                            double *t2T_bar, double *vooo_bar, double *fvo_bar,
                            double *cache_row_a_bar, double *cache_col_a_bar,
                            double *cache_row_b_bar, double *cache_col_b_bar);

/*
 * Device-pointer block calls, the reference's slab interface on device memory:
 * ct_energy_vjp_block runs the jobs _ccsd_t_gen_jobs enumerates for
 * (a0,a1,b0,b1) (pyscfadlib/pyscfadlib/vjp/cc/ccsd_t.c:6-72; either b1 <= a0 or
 * (b0,b1) == (a0,a1)) with vvop the full array, and e_out (device, nullable)
 * receives that block's share of E(T).  ct_energy_block covers the jobs
 * a0 <= a < a1 (lnoccsdt_contract's a-slab, lno_ccsd_t.c:96-100, mat = I).
 */
int ct_energy_vjp_block(const ct_problem *p, int mode, double et_bar, const ct_grads *g,
                        int a0, int a1, int b0, int b1, double *e_out, void *stream);
int ct_energy_block(const ct_problem *p, int mode, int a0, int a1, double *e_out,
                    double *job_e_out, void *stream);

/*
 * LNO-projected (T) energy, the sum lnoccsdt_contract (lno_ccsd_t.c:96-138)
 * accumulates: over the ordered jobs (x, y, z), y >= z, a0 <= x < a1, of
 * fac * sum_ijk (sum_l mat[l,i] w[l,j,k]) z[i,j,k] / D (fac 1/2 when y == z;
 * lno_ccsd_t.c:6-29), without the driver's 2/3 (pyscfad/lno/ccsd_t.py:111).
 * mat: DEVICE (nocc, nocc) float64, C-contiguous.  Float64 path only; nocc <= 64.
 * e_out (device, nullable) receives the sum; job_e_out (device, nullable,
 * v(v+1)(v+2)/6 doubles) each sorted job's share at its a-major index.
 * mat = identity gives 3/2 of the canonical E(T) of the same slab's jobs.
 */
int ct_lno_energy(const ct_problem *p, const double *mat, int a0, int a1, double *e_out,
                  double *job_e_out, void *stream);

/*
 * The same LNO-projected energy in a chosen precision mode (no reference
 * counterpart: lnoccsdt_contract is float64).  CT_MODE_FP64 is ct_lno_energy;
 * CT_MODE_TF32 / CT_MODE_BF16X3 run the F1/F2 contractions on the tensor
 * cores as the canonical mixed path does (nocc % 8 == 0, nocc <= 64), keep the
 * W and z/D cubes as float and form the projection in float64 from them.
 */
int ct_lno_energy_mode(const ct_problem *p, int mode, const double *mat, int a0, int a1,
                       double *e_out, double *job_e_out, void *stream);

/*
 * VJP of the LNO-projected sum over every LNO job: lnoccsdt_energy_vjp
 * (lno_ccsd_t_vjp.c:400-566) with the full block (0, nvir, 0, nvir).  et_bar
 * as the reference kernel takes it (pyscfad/lno/ccsd_t.py:127 applies the 2/3
 * before the call; no doubling).  Gradients (device, kernel layouts) and
 * mat_bar (device, (nocc, nocc)) accumulate (+=); e_out (device, nullable)
 * receives the sum.  Float64 path only; nocc <= 64.
 */
int ct_lno_energy_vjp(const ct_problem *p, const double *mat, double et_bar, const ct_grads *g,
                      double *mat_bar, double *e_out, void *stream);

/*
 * One slab block (b0, b1, c0, c1) of the same: the orderings (x, y, z) with y
 * in [b0, b1) and z in [c0, c1) (lno_ccsd_t_vjp.c:355-398); either
 * (c0, c1) == (b0, b1) or c1 <= b0.  vvop is the full array on the device.
 */
int ct_lno_energy_vjp_block(const ct_problem *p, const double *mat, double et_bar, int b0, int b1,
                            int c0, int c1, const ct_grads *g, double *mat_bar, double *e_out,
                            void *stream);

/*
 * The same slab block in a chosen precision mode (no reference counterpart:
 * lnoccsdt_energy_vjp is float64).  CT_MODE_FP64 is ct_lno_energy_vjp_block;
 * CT_MODE_TF32 / CT_MODE_BF16X3 (nocc % 8 == 0, nocc <= 64) run the F1/F2 and
 * bar GEMMs on the tensor cores as the canonical mixed VJP does, keep the W,
 * z/D, A and B cubes as float and form the projections, energies and mat_bar
 * in float64 from them.  (0, nvir, 0, nvir) covers every LNO job.
 */
int ct_lno_energy_vjp_mode(const ct_problem *p, int mode, const double *mat, double et_bar,
                           int b0, int b1, int c0, int c1, const ct_grads *g, double *mat_bar,
                           double *e_out, void *stream);

/*
 * Iterative (T) on the full 6-D triples amplitudes (pyscfad/cc/ccsd_t_slow.py:
 * 128-293), two steps.  ct_t3_init fills t3_c = P6(w + v) / d3 (the initial
 * guess of update_amps, :188-208) and t3_x = r3_6d(P6(w)) / 3 (so that
 * energy(t2, t3) of :210-220 is sum t3 * t3_x), both DEVICE (v, v, v, o, o, o)
 * float64 arrays laid out [a][b][c][i][j][k] (the reference's t3[i,j,k,a,b,c]
 * transposed); float64 path.  ct_t3_update forms one update,
 * t3_new = t3_c + (P3(tvv) - P3(too)) / d3, from tvv = fvv' t3 (the virtual
 * Fock block without its diagonal on the first virtual index, [a][b][c][i][j][k])
 * and too_m = foo' t3 on the first occupied index of the occupied-major copy
 * [i][a][b][c][j][k] (both formed by the caller, e.g. as one GEMM each); it
 * writes t3_new, its occupied-major copy t3_new_m (nullable) and
 * sums[0] = |t3_new - t3|^2, sums[1] = the energy of t3_new (device, 2
 * doubles).  The outputs must not alias the inputs.
 */
int ct_t3_init(const ct_problem *p, double *t3_c, double *t3_x, void *stream);
int ct_t3_update(int nocc, int nvir, const double *mo_energy, const double *t3_c, const double *tvv,
                 const double *too_m, const double *t3, const double *t3_x, double *t3_new,
                 double *t3_new_m, double *sums, void *stream);

/*
 * E(T) restricted to an explicit list of sorted virtual triples (no reference
 * counterpart; it is the exact pass of a surrogate-screened energy).
 * jobs_abc: HOST array of njobs triples (a, b, c), nvir > a >= b >= c >= 0,
 * each listed once.  e_out (device, nullable) receives the sum over the
 * listed jobs; job_e_out (device, nullable, v(v+1)(v+2)/6 doubles) receives
 * each listed job's contribution at its a-major sorted index and zero
 * elsewhere.  A job outside the sorted range returns CT_ERR_SHAPE.
 */
int ct_energy_jobs(const ct_problem *p, int mode, const int *jobs_abc, int njobs, double *e_out,
                   double *job_e_out, void *stream);

/*
 * Measurement hooks (no reference counterpart): when enabled, every kernel
 * launch of the library is bracketed by CUDA events on its stream;
 * ct_profile_read sums the durations of one kernel kind (0 W-build GEMM,
 * 1 vooo W term, 2 epilogue, 3 V-term bars, 4 vvop bar GEMM, 5 t2 bar GEMM,
 * 6 vooo bar GEMM, 7 t2 vooo-bar GEMM, 8 energy reduction, 9.. mixed-path kinds).
 * ct_peak_probe measures a pipe's sustained rate in TFLOP/s with a
 * register-resident loop (kind 0 float64 DMMA, 1 float64 DFMA).
 */
int ct_profile_enable(int on);
int ct_profile_read(int kind, double *total_ms, int *launches);
int ct_profile_reset(void);
int ct_peak_probe(int kind, double *tflops);

/*
 * Allocation-free float64 energy.  No counterpart in the reference: it exists
 * for callers that must not have the library allocate device memory, such as
 * an XLA/JAX FFI handler whose framework owns all device memory, or callers
 * avoiding the device-wide synchronization of cudaMalloc/cudaFree.  Same
 * inputs, result and float64 arithmetic as ct_energy (e_out: device pointer to
 * one double), but all scratch lives in one file-scope device array of
 * CT_NOALLOC_SCRATCH_DOUBLES doubles (32 MiB), held by every GPU that loads
 * the library until exit; no cudaMalloc/cudaFree or allocating routine is
 * called.  Problems need nvir(nvir+1)(nvir+2)/6 + 7 nocc^3 + 65 doubles of it
 * (nocc <= 64); larger ones return CT_ERR_SIZE.  The first call on a device
 * looks up the array's device address (once per device, with that device
 * current), so it should come before any stream capture.  Every call reuses
 * the same array: calls that overlap on the GPU (e.g. on two streams) race.
 */
#define CT_NOALLOC_SCRATCH_DOUBLES (4 * 1024 * 1024)
int ct_energy_noalloc(const ct_problem *p, double *e_out, void *stream);

/*
 * Learned block surrogate (no reference counterpart).  A 12-128-128-1 SiLU MLP
 * maps cheap per-job features of a sorted virtual triple (a >= b >= c) to that
 * job's (T) contribution; it ranks jobs and estimates the unscreened ones in a
 * screened pass, with ct_energy_jobs computing the kept jobs exactly.
 * All pointers are device pointers; all work is stream-ordered.
 *
 * Parameters: float32[CT_MLP_NPARAM] = W1[128][12] | b1[128] | W2[128][128] |
 * b2[128] | W3[128] | b3.  X: float32[n][12] row-major features; Y: float32[n].
 */
#define CT_MLP_IN 12
#define CT_MLP_HIDDEN 128
#define CT_MLP_NPARAM (CT_MLP_HIDDEN * CT_MLP_IN + CT_MLP_HIDDEN + CT_MLP_HIDDEN * CT_MLP_HIDDEN + CT_MLP_HIDDEN + CT_MLP_HIDDEN + 1)

/* float32 forward; Z1, Z2 (nullable, float32[n][128]) receive the hidden
 * pre-activations that ct_mlp_backward needs. */
int ct_mlp_forward(const float *params, const float *X, int n, float *Z1, float *Z2, float *Y, void *stream);
/* loss = mean (Y - T)^2 (double, nullable); dY = dloss/dY (nullable). */
int ct_mlp_mse(const float *Y, const float *T, int n, float *dY, double *loss, void *stream);
/* Floats of the work buffer ct_mlp_backward needs for n samples. */
long long ct_mlp_work_floats(int n);
/* grad (overwritten) = dloss/dparams given dY, from the saved pre-activations;
 * deterministic (fixed-order reduction of per-CTA partial sums). */
int ct_mlp_backward(const float *params, const float *X, const float *Z1, const float *Z2, const float *dY, int n,
                    float *grad, float *work, void *stream);
/* One AdamW step (bias-corrected moments m, v; decoupled weight decay). */
int ct_mlp_adam(float *params, const float *grad, float *m, float *v, int step, float lr, float beta1, float beta2,
                float eps, float weight_decay, void *stream);
/* params -> bf16 copy (round to nearest even), for ct_mlp_infer_bf16. */
int ct_mlp_to_bf16(const float *params, void *params_bf16, void *stream);
/* Inference with bf16 weights and activations, float32 accumulation. */
int ct_mlp_infer_bf16(const void *params_bf16, const float *X, int n, float *Y, void *stream);
/*
 * Features of njobs packed jobs (a | b << 10 | c << 20, a >= b >= c) of
 * problem p into F (float32[njobs][12]); pair_work holds 3 nvir^2 floats of
 * per-virtual-pair statistics (t2 block norms, MP2 pair energies, vvov block
 * norms).  Reads mo_energy, t2T and vvop.
 */
int ct_surrogate_features(const ct_problem *p, const int *jobs, long long njobs, float *pair_work, float *F,
                          void *stream);

/* Frees the cached device workspace (scratch waves, job plans). */
/*
 * Density-fitted ERI producer (pyscfad/cc/dfccsd.py:73-88 forms ovoo, ovov,
 * ovvv from the three-index factors; pyscfad/cc/ccsd_t.py:88-106 transposes
 * them into vooo and vvop): the kernel layouts straight from the factors on
 * device pointers, float64 tensor-core GEMMs with the transposes folded into
 * their addressing.  Loo (naux, nocc, nocc), Lov (naux, nocc, nvir),
 * R = [Lov ; Lvv] (naux, nmo, nvir) with Lvv unpacked; writes
 * vooo (nvir, nocc, nocc, nocc) and vvop (nvir, nvir, nocc, nmo).
 */
int ct_df_layouts(int nocc, int nvir, int naux, const double *Loo, const double *Lov, const double *R,
                  double *vooo, double *vvop, void *stream);
/*
 * Its VJP: accumulates (+=) the factor gradients of kernel-layout gradients
 * vooo_bar and vvop_bar into dLoo (naux, nocc, nocc), dLov (naux, nocc, nvir)
 * and dRt (naux, nvir, nmo), the gradient of Rt = R transposed in its last two
 * axes (Rt is passed too); the caller splits dRt into the Lov and Lvv parts.
 */
int ct_df_factor_bar(int nocc, int nvir, int naux, const double *Loo, const double *Lov, const double *Rt,
                     const double *vooo_bar, const double *vvop_bar, double *dLoo, double *dLov, double *dRt,
                     void *stream);

int ct_release_workspace(void);

/* Device bytes the workspace of one call at (nocc, nvir, mode) would hold. */
long long ct_workspace_bytes(int nocc, int nvir, int mode, int with_vjp);

#ifdef __cplusplus
}
#endif
#endif /* PYSCFAD_B200_H */
