// Mixed-precision path (tcgen05 kind::tf32 / bf16x3).  Placeholder until the
// tensor-memory kernels land: reports CT_ERR_MODE.
#include "ct_mixed.h"

namespace ctb {

double mixed_extra_bytes_per_job(int o, int mode) {
    (void)o; (void)mode;
    return 0.0;
}

int mixed_prepare(const ct_problem *p, int mode, MixedOperands *mo, cudaStream_t st) {
    (void)p; (void)mode; (void)mo; (void)st;
    return CT_ERR_MODE;
}

int mixed_wave(const WaveView &w, const EpiArgs &e, const ct_problem *p, const ct_grads *g,
               const MixedOperands &mo, int mode, bool vjp, void *scratch, cudaStream_t st) {
    (void)w; (void)e; (void)p; (void)g; (void)mo; (void)mode; (void)vjp; (void)scratch; (void)st;
    return CT_ERR_MODE;
}

void mixed_release(MixedOperands *mo, cudaStream_t st) { (void)mo; (void)st; }

}  // namespace ctb
