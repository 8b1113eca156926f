// Interface of the mixed-precision (tcgen05) path to the host orchestration.
#pragma once
#include <cuda_runtime.h>
#include "ct_internal.h"
#include "../../include/pyscfad_b200.h"

namespace ctb {

// Low-precision operand copies prepared once per call (converted from the
// float64 inputs on the device).
struct MixedOperands {
    void *t2 = nullptr;      // t2T as float32 (tf32) or its bf16 hi plane
    void *vvop = nullptr;    // vvop virtual block as float32 / bf16 hi plane
    void *vooo = nullptr;    // vooo as float32 / bf16 hi plane
    void *t2q = nullptr;     // t2T with each (q,r) plane qr-tiled (as the scratch slots), for VB
    void *t2k = nullptr;     // t2T transposed to [z][tiled qr][f] (rows padded to vp), F1's K-major A
    void *t2_lo = nullptr;   // bf16 lo planes (BF16x3 only)
    void *t2q_lo = nullptr;
    void *t2k_lo = nullptr;
    void *vvop_lo = nullptr;
    void *vooo_lo = nullptr;
    float *vvoo_f = nullptr;  // float vvop[:,:,:,:o] as (v,v,o,o), for the epilogue's V tiles
    float *t2_f = nullptr;    // float t2T (v,v,o,o), for the epilogue's V tiles
    size_t bytes = 0;
    int mode = 0;
    int vp = 0;              // padded nvir of the vvop copy (16-byte rows)
};

// The rows of the inputs one conversion covers: t2T rows z in [z0, z1)
// (t2, t2q, t2k, t2_f), vooo rows x in [x0, x1), and vvop pair rectangles
// x in [r[0], r[1]), y in [r[2], r[3]) (vvop, vvoo_f).  Staged callers convert
// each stage's rows once they are on the device.
struct MixedRegion {
    int z0 = 0, z1 = 0, x0 = 0, x1 = 0;
    int nrect = 0;
    int rect[4][4] = {};
};

// extra scratch bytes per job the mixed path needs beyond the 7 o^3 slots
double mixed_extra_bytes_per_job(int o, int mode);
// operand buffer and pointers, no conversion
int mixed_setup(const ct_problem *p, int mode, MixedOperands *mo, cudaStream_t st);
// converts the rows of one region (after mixed_setup)
int mixed_convert(const ct_problem *p, const MixedOperands &mo, const MixedRegion &r, cudaStream_t st);
// mixed_setup and the conversion of every row
int mixed_prepare(const ct_problem *p, int mode, MixedOperands *mo, cudaStream_t st);
// prof(kind, 0/1, ctx) brackets each launch for the optional per-kernel timing
int mixed_wave(const WaveView &w, const EpiArgs &e, const ct_problem *p, const ct_grads *g,
               const MixedOperands &mo, int mode, bool vjp, void *scratch, cudaStream_t st,
               int (*prof)(int, int, void *), void *pctx);
void mixed_release(MixedOperands *mo, cudaStream_t st);
// frees the operand buffer kept across calls
void mixed_free_cache();
// bytes of that buffer for (nocc, nvir, mode)
size_t mixed_operand_bytes(int o, int v, int mode);
// reads (and synchronizes on) the device-side timeout flag of the tcgen05 kernels
int mixed_check_error(cudaStream_t st);

}  // namespace ctb
