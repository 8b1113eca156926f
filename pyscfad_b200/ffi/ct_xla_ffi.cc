// XLA FFI handlers over the C-ABI, for a JAX build of pyscfad.
//
// pyscfad drives the (T) path from a jax.custom_vjp (pyscfad/cc/ccsd_t.py:36-80):
// the forward is the canonical energy (:41), the backward the hand-written VJP
// (_ccsd_t_energy_vjp, :82-192, reaching ccsd_t_energy_vjp of
// pyscfadlib/vjp/cc/ccsd_t_vjp.c:332-346 through ctypes).  These handlers put
// the same two calls on XLA's stream with XLA-owned device buffers, in the
// kernel layouts the driver builds (:88-106): t1T (v,o), t2T (v,v,o,o),
// vooo (v,o,o,o), fvo (v,o), vvop (v,v,o,nmo), mo_energy (nmo).
//
//   ct_energy_ffi      (mode attr)          -> e (scalar)
//   ct_energy_vjp_ffi  (mode, et_bar attrs) -> e, mo_energy_bar, t1T_bar,
//                                              t2T_bar, vooo_bar, fvo_bar, vvop_bar
//
// et_bar is the cotangent of E(T); the kernel convention is twice it
// (pyscfad/cc/ccsd_t.py:86), applied here.  The gradient results are zeroed
// on the stream before the kernel accumulates into them.
//
// Compiled only where jaxlib's FFI headers are on the include path
// (python -m pyscfad_b200._build --ffi <dir holding xla/ffi/api/ffi.h>); the
// guard leaves an empty translation unit otherwise.
#if defined(__has_include)
#if __has_include("xla/ffi/api/ffi.h")
#define CTB_HAVE_XLA_FFI 1
#endif
#endif

#ifdef CTB_HAVE_XLA_FFI
#include <cuda_runtime.h>
#include <string>
#include "xla/ffi/api/ffi.h"
#include "pyscfad_b200.h"

namespace ffi = xla::ffi;

namespace {

ffi::Error status_error(const char *what, int s) {
    if (s == CT_OK) return ffi::Error::Success();
    std::string msg = std::string(what) + ": " + ct_status_string(s);
    return ffi::Error(ffi::ErrorCode::kInternal, msg);
}

ct_problem problem_of(ffi::Buffer<ffi::F64> &mo, ffi::Buffer<ffi::F64> &t1T, ffi::Buffer<ffi::F64> &t2T,
                      ffi::Buffer<ffi::F64> &vooo, ffi::Buffer<ffi::F64> &fvo, ffi::Buffer<ffi::F64> &vvop) {
    const auto dims = t1T.dimensions();
    ct_problem p{};
    p.nvir = static_cast<int>(dims[0]);
    p.nocc = static_cast<int>(dims[1]);
    p.mo_energy = mo.typed_data();
    p.t1T = t1T.typed_data();
    p.t2T = t2T.typed_data();
    p.vooo = vooo.typed_data();
    p.fvo = fvo.typed_data();
    p.vvop = vvop.typed_data();
    return p;
}

ffi::Error CtEnergy(cudaStream_t st, int64_t mode, ffi::Buffer<ffi::F64> mo, ffi::Buffer<ffi::F64> t1T,
                    ffi::Buffer<ffi::F64> t2T, ffi::Buffer<ffi::F64> vooo, ffi::Buffer<ffi::F64> fvo,
                    ffi::Buffer<ffi::F64> vvop, ffi::ResultBuffer<ffi::F64> e) {
    ct_problem p = problem_of(mo, t1T, t2T, vooo, fvo, vvop);
    return status_error("ct_energy", ct_energy(&p, static_cast<int>(mode), e->typed_data(), nullptr, st));
}

ffi::Error CtEnergyVjp(cudaStream_t st, int64_t mode, double et_bar, ffi::Buffer<ffi::F64> mo,
                       ffi::Buffer<ffi::F64> t1T, ffi::Buffer<ffi::F64> t2T, ffi::Buffer<ffi::F64> vooo,
                       ffi::Buffer<ffi::F64> fvo, ffi::Buffer<ffi::F64> vvop, ffi::ResultBuffer<ffi::F64> e,
                       ffi::ResultBuffer<ffi::F64> mo_b, ffi::ResultBuffer<ffi::F64> t1_b,
                       ffi::ResultBuffer<ffi::F64> t2_b, ffi::ResultBuffer<ffi::F64> vooo_b,
                       ffi::ResultBuffer<ffi::F64> fvo_b, ffi::ResultBuffer<ffi::F64> vvop_b) {
    ct_problem p = problem_of(mo, t1T, t2T, vooo, fvo, vvop);
    for (auto *r : {&mo_b, &t1_b, &t2_b, &vooo_b, &fvo_b, &vvop_b})
        if (cudaMemsetAsync((*r)->untyped_data(), 0, (*r)->size_bytes(), st) != cudaSuccess)
            return status_error("ct_energy_vjp", CT_ERR_CUDA);
    ct_grads g{mo_b->typed_data(), t1_b->typed_data(), t2_b->typed_data(),
               vooo_b->typed_data(), fvo_b->typed_data(), vvop_b->typed_data()};
    return status_error("ct_energy_vjp",
                        ct_energy_vjp(&p, static_cast<int>(mode), 2.0 * et_bar, &g, e->typed_data(), st));
}

}  // namespace

XLA_FFI_DEFINE_HANDLER_SYMBOL(ct_energy_ffi, CtEnergy,
                              ffi::Ffi::Bind()
                                  .Ctx<ffi::PlatformStream<cudaStream_t>>()
                                  .Attr<int64_t>("mode")
                                  .Arg<ffi::Buffer<ffi::F64>>()
                                  .Arg<ffi::Buffer<ffi::F64>>()
                                  .Arg<ffi::Buffer<ffi::F64>>()
                                  .Arg<ffi::Buffer<ffi::F64>>()
                                  .Arg<ffi::Buffer<ffi::F64>>()
                                  .Arg<ffi::Buffer<ffi::F64>>()
                                  .Ret<ffi::Buffer<ffi::F64>>());

XLA_FFI_DEFINE_HANDLER_SYMBOL(ct_energy_vjp_ffi, CtEnergyVjp,
                              ffi::Ffi::Bind()
                                  .Ctx<ffi::PlatformStream<cudaStream_t>>()
                                  .Attr<int64_t>("mode")
                                  .Attr<double>("et_bar")
                                  .Arg<ffi::Buffer<ffi::F64>>()
                                  .Arg<ffi::Buffer<ffi::F64>>()
                                  .Arg<ffi::Buffer<ffi::F64>>()
                                  .Arg<ffi::Buffer<ffi::F64>>()
                                  .Arg<ffi::Buffer<ffi::F64>>()
                                  .Arg<ffi::Buffer<ffi::F64>>()
                                  .Ret<ffi::Buffer<ffi::F64>>()
                                  .Ret<ffi::Buffer<ffi::F64>>()
                                  .Ret<ffi::Buffer<ffi::F64>>()
                                  .Ret<ffi::Buffer<ffi::F64>>()
                                  .Ret<ffi::Buffer<ffi::F64>>()
                                  .Ret<ffi::Buffer<ffi::F64>>()
                                  .Ret<ffi::Buffer<ffi::F64>>());
#endif  // CTB_HAVE_XLA_FFI
