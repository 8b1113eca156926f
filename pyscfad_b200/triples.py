"""Device-level (T) energy and VJP on torch CUDA tensors in the kernel layouts.

Tensors are float64, C-contiguous, on one CUDA device, in the layouts of
pyscfad's (T) VJP driver (pyscfad/cc/ccsd_t.py:88-106):
mo_energy (nmo), t1T (v,o), t2T (v,v,o,o) [a,b,j,i], vooo (v,o,o,o),
fvo (v,o), vvop (v,v,o,nmo).  All work is enqueued on the current torch stream.
"""
from __future__ import annotations

import ctypes

import torch

from . import native

KEYS = ("mo_energy", "t1T", "t2T", "vooo", "fvo", "vvop")


def _check_layouts(L: dict):
    t1T = L["t1T"]
    nvir, nocc = t1T.shape
    nmo = nocc + nvir
    shapes = dict(mo_energy=(nmo,), t1T=(nvir, nocc), t2T=(nvir, nvir, nocc, nocc),
                  vooo=(nvir, nocc, nocc, nocc), fvo=(nvir, nocc), vvop=(nvir, nvir, nocc, nmo))
    dev = t1T.device
    if dev.type != "cuda":
        raise native.CtError("pyscfad_b200 kernels need CUDA tensors")
    for k in KEYS:
        t = L[k]
        if tuple(t.shape) != shapes[k]:
            raise native.CtError(f"{k}: shape {tuple(t.shape)} != {shapes[k]}")
        if t.dtype != torch.float64 or not t.is_contiguous() or t.device != dev:
            raise native.CtError(f"{k}: need a contiguous float64 tensor on {dev}")
    return nocc, nvir, dev


def _problem(L: dict, nocc: int, nvir: int) -> native.CtProblem:
    return native.CtProblem(nocc, nvir, *[ctypes.c_void_p(L[k].data_ptr()) for k in KEYS])


def _stream(dev) -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)


def energy(L: dict, mode="fp64", job_e: torch.Tensor | None = None) -> torch.Tensor:
    """E(T) as a 0-d device tensor.  ``job_e`` (optional, float64, length
    v(v+1)(v+2)/6) receives the per-job (a>=b>=c, a-major) contributions."""
    nocc, nvir, dev = _check_layouts(L)
    out = torch.empty((), dtype=torch.float64, device=dev)
    je = None
    if job_e is not None:
        if job_e.numel() != nvir * (nvir + 1) * (nvir + 2) // 6 or job_e.dtype != torch.float64:
            raise native.CtError("job_e: need v(v+1)(v+2)/6 float64 elements")
        je = ctypes.c_void_p(job_e.data_ptr())
    prob = _problem(L, nocc, nvir)
    with torch.cuda.device(dev):
        st = native.lib().ct_energy(ctypes.byref(prob), native.mode_id(mode),
                                    ctypes.c_void_p(out.data_ptr()), je, _stream(dev))
    native.check(st, "ct_energy")
    return out


def lno_energy(L: dict, mat: torch.Tensor, a0: int = 0, a1: int | None = None,
               job_e: torch.Tensor | None = None, mode="fp64") -> torch.Tensor:
    """LNO-projected (T) sum of lnoccsdt_contract (lno_ccsd_t.c:96-138) over
    the a-slab [a0, a1) as a 0-d device tensor: ordered jobs (x, y>=z) with x
    in the slab, occupied index of x projected by ``mat`` (nocc, nocc).
    pyscfad's LNO driver scales the full-range sum by 2/3
    (pyscfad/lno/ccsd_t.py:111); mat = I gives 3/2 of E(T).  ``mode`` "tf32"
    or "bf16x3" runs the contractions on the tensor cores (nocc % 8 == 0)."""
    nocc, nvir, dev = _check_layouts(L)
    if a1 is None:
        a1 = nvir
    if mat.shape != (nocc, nocc) or mat.dtype != torch.float64 or mat.device != dev:
        raise native.CtError("mat: need a (nocc, nocc) float64 tensor on the inputs' device")
    mat = mat.contiguous()
    out = torch.empty((), dtype=torch.float64, device=dev)
    je = None
    if job_e is not None:
        if job_e.numel() != nvir * (nvir + 1) * (nvir + 2) // 6 or job_e.dtype != torch.float64:
            raise native.CtError("job_e: need v(v+1)(v+2)/6 float64 elements")
        je = ctypes.c_void_p(job_e.data_ptr())
    prob = _problem(L, nocc, nvir)
    with torch.cuda.device(dev):
        st = native.lib().ct_lno_energy_mode(ctypes.byref(prob), native.mode_id(mode),
                                             ctypes.c_void_p(mat.data_ptr()), int(a0), int(a1),
                                             ctypes.c_void_p(out.data_ptr()), je, _stream(dev))
    native.check(st, "ct_lno_energy_mode")
    return out


def lno_energy_vjp(L: dict, mat: torch.Tensor, et_bar: float, grads: dict | None = None,
                   mat_bar: torch.Tensor | None = None, block: tuple | None = None, mode="fp64"):
    """VJP of the full-range LNO sum (lnoccsdt_energy_vjp over every LNO job).
    ``et_bar`` is the reference kernel's cotangent as passed
    (pyscfad/lno/ccsd_t.py:127 scales by 2/3 first; no doubling).  Accumulates
    into ``grads`` and ``mat_bar`` (created zeroed when None); returns
    (sum device tensor, mat_bar, grads).  ``block`` = (b0, b1, c0, c1) runs one
    block of the reference driver's slab loop instead of every LNO job.
    ``mode`` "tf32" or "bf16x3" runs the GEMMs on the tensor cores
    (nocc % 8 == 0)."""
    nocc, nvir, dev = _check_layouts(L)
    if mat.shape != (nocc, nocc) or mat.dtype != torch.float64 or mat.device != dev:
        raise native.CtError("mat: need a (nocc, nocc) float64 tensor on the inputs' device")
    mat = mat.contiguous()
    b0, b1, c0, c1 = block if block is not None else (0, nvir, 0, nvir)
    if grads is None:
        grads = {k: torch.zeros_like(L[k]) for k in KEYS}
    if mat_bar is None:
        mat_bar = torch.zeros_like(mat)
    for k in KEYS:
        g = grads[k]
        if g.shape != L[k].shape or g.dtype != torch.float64 or not g.is_contiguous() or g.device != dev:
            raise native.CtError(f"grad {k}: need a contiguous float64 tensor like the input")
    if mat_bar.shape != mat.shape or mat_bar.dtype != torch.float64 or not mat_bar.is_contiguous():
        raise native.CtError("mat_bar: need a contiguous (nocc, nocc) float64 tensor")
    prob = _problem(L, nocc, nvir)
    gr = native.CtGrads(*[ctypes.c_void_p(grads[k].data_ptr()) for k in KEYS])
    out = torch.empty((), dtype=torch.float64, device=dev)
    with torch.cuda.device(dev):
        st = native.lib().ct_lno_energy_vjp_mode(ctypes.byref(prob), native.mode_id(mode),
                                                 ctypes.c_void_p(mat.data_ptr()), float(et_bar), int(b0), int(b1),
                                                 int(c0), int(c1), ctypes.byref(gr),
                                                 ctypes.c_void_p(mat_bar.data_ptr()),
                                                 ctypes.c_void_p(out.data_ptr()), _stream(dev))
    native.check(st, "ct_lno_energy_vjp_mode")
    return out, mat_bar, grads


def energy_vjp(L: dict, et_bar: float, grads: dict | None = None, mode="fp64"):
    """Accumulates the VJP into ``grads`` (created zeroed when None) and returns
    (E(T) device tensor, grads).  ``et_bar`` follows the C kernel's convention
    (twice the cotangent of E(T), pyscfad/cc/ccsd_t.py:86)."""
    nocc, nvir, dev = _check_layouts(L)
    if grads is None:
        grads = {k: torch.zeros_like(L[k]) for k in KEYS}
    for k in KEYS:
        g = grads[k]
        if g.shape != L[k].shape or g.dtype != torch.float64 or not g.is_contiguous() or g.device != dev:
            raise native.CtError(f"grad {k}: need a contiguous float64 tensor like the input")
    prob = _problem(L, nocc, nvir)
    gr = native.CtGrads(*[ctypes.c_void_p(grads[k].data_ptr()) for k in KEYS])
    out = torch.empty((), dtype=torch.float64, device=dev)
    with torch.cuda.device(dev):
        st = native.lib().ct_energy_vjp(ctypes.byref(prob), native.mode_id(mode), float(et_bar),
                                        ctypes.byref(gr), ctypes.c_void_p(out.data_ptr()), _stream(dev))
    native.check(st, "ct_energy_vjp")
    return out, grads


class TriplesEnergy(torch.autograd.Function):
    """E(T) over kernel-layout tensors; backward runs the hand-written VJP
    (W/V recomputed, never stored).  mode is not differentiable."""

    @staticmethod
    def forward(ctx, mo_energy, t1T, t2T, vooo, fvo, vvop, mode="fp64"):
        L = dict(mo_energy=mo_energy.contiguous(), t1T=t1T.contiguous(), t2T=t2T.contiguous(),
                 vooo=vooo.contiguous(), fvo=fvo.contiguous(), vvop=vvop.contiguous())
        ctx.save_for_backward(*[L[k] for k in KEYS])
        ctx.mode = mode
        return energy(L, mode)

    @staticmethod
    def backward(ctx, gE):
        L = dict(zip(KEYS, ctx.saved_tensors))
        # the C kernel's et_bar is twice the cotangent (pyscfad/cc/ccsd_t.py:86)
        _, g = energy_vjp(L, 2.0 * float(gE), None, ctx.mode)
        return tuple(g[k] for k in KEYS) + (None,)


def triples_energy(mo_energy, t1T, t2T, vooo, fvo, vvop, mode="fp64"):
    return TriplesEnergy.apply(mo_energy, t1T, t2T, vooo, fvo, vvop, mode)
