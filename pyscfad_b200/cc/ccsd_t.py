"""CCSD(T) energy with a hand-written VJP on B200 — drop-in for pyscfad.cc.ccsd_t.

Mirrors pyscfad/cc/ccsd_t.py:
  * ``kernel(mycc, eris, t1, t2, verbose)`` (:28-80): returns E(T); when the
    inputs are torch tensors that require grad, the result is differentiable
    and its backward is ``_ccsd_t_energy_vjp`` (the reference's custom_vjp bwd).
  * ``_ccsd_t_energy_vjp(eris, t1, t2, et_bar, max_memory)`` (:82-192): returns
    (t1_bar, t2_bar, fock_bar, mo_energy_bar, ovoo_bar, ovov_bar, ovvv_bar) with
    the same layout transforms, the et_bar doubling (:86), and the packed-tril
    ovvv gradient (:186-191) when eris.ovvv is stored packed.

Both forward and backward run on the CUDA kernels of this package (FP64 by
default; ``mode='tf32'`` / ``'bf16x3'`` select the mixed-precision
contractions).  max_memory is accepted for signature compatibility: the B200
path keeps vvop resident instead of streaming slabs.
"""
from __future__ import annotations

import numpy as np
import torch

from .. import triples
from .eris import pack_tril

__all__ = ["kernel", "_ccsd_t_energy_vjp", "kernel_layouts", "CCSDTKernel"]


def _dev(device=None):
    if device is not None:
        return torch.device(device)
    if not torch.cuda.is_available():
        raise RuntimeError("pyscfad_b200: no CUDA device available")
    return torch.device("cuda", torch.cuda.current_device())


def _t(x, dev):
    if isinstance(x, torch.Tensor):
        return x.to(device=dev, dtype=torch.float64)
    return torch.as_tensor(np.asarray(x, dtype=np.float64), device=dev)


def kernel_layouts(t1, t2, mo_energy, fock, ovoo, ovov, ovvv_full, device=None) -> dict:
    """Kernel-layout tensors from pyscf-layout inputs (pyscfad/cc/ccsd_t.py:88-106)."""
    dev = _dev(device)
    t1, t2 = _t(t1, dev), _t(t2, dev)
    nocc, nvir = t1.shape
    fock = _t(fock, dev)
    ovov, ovoo, ovvv_full = _t(ovov, dev), _t(ovoo, dev), _t(ovvv_full, dev)
    vvop = torch.empty((nvir, nvir, nocc, nocc + nvir), dtype=torch.float64, device=dev)
    vvop[:, :, :, :nocc] = ovov.permute(1, 3, 0, 2)
    vvop[:, :, :, nocc:] = ovvv_full.permute(1, 3, 0, 2)
    return dict(mo_energy=_t(mo_energy, dev).contiguous(),
                t1T=t1.t().contiguous(),
                t2T=t2.permute(2, 3, 1, 0).contiguous(),
                vooo=ovoo.permute(1, 0, 3, 2).contiguous(),
                fvo=fock[nocc:, :nocc].contiguous(),
                vvop=vvop)


def _grads_to_pyscf(g: dict, nocc: int, nvir: int, packed: bool):
    """Un-transposes kernel-layout gradients (pyscfad/cc/ccsd_t.py:179-191)."""
    nmo = nocc + nvir
    t1_bar = g["t1T"].t()
    t2_bar = g["t2T"].permute(3, 2, 0, 1)
    fock_bar = g["t1T"].new_zeros((nmo, nmo))
    fock_bar[nocc:, :nocc] = g["fvo"]
    ovoo_bar = g["vooo"].permute(1, 0, 3, 2)
    ovov_bar = g["vvop"][:, :, :, :nocc].permute(2, 0, 3, 1)
    ovvv_bar = g["vvop"][:, :, :, nocc:].permute(2, 0, 3, 1)
    if packed:
        ovvv_bar = ovvv_bar + ovvv_bar.transpose(2, 3)
        ii = torch.arange(nvir, device=ovvv_bar.device)
        ovvv_bar[:, :, ii, ii] *= .5
        ovvv_bar = pack_tril(ovvv_bar)
    return t1_bar, t2_bar, fock_bar, g["mo_energy"], ovoo_bar, ovov_bar, ovvv_bar


class CCSDTKernel(torch.autograd.Function):
    """E(T)(t1, t2, mo_energy, fock, ovoo, ovov, ovvv) with the hand-written VJP
    (the torch counterpart of the reference's jax.custom_vjp, :36-79)."""

    @staticmethod
    def forward(ctx, t1, t2, mo_energy, fock, ovoo, ovov, ovvv, mode="fp64"):
        nocc, nvir = t1.shape
        packed = ovvv.dim() == 3
        from .eris import unpack_tril
        ovvv_full = unpack_tril(ovvv, nvir) if packed else ovvv
        L = kernel_layouts(t1, t2, mo_energy, fock, ovoo, ovov, ovvv_full, device=t1.device)
        ctx.L = L
        ctx.meta = (nocc, nvir, packed, mode)
        return triples.energy(L, mode)

    @staticmethod
    def backward(ctx, gE):
        nocc, nvir, packed, mode = ctx.meta
        _, g = triples.energy_vjp(ctx.L, 2.0 * float(gE), None, mode)
        ctx.L = None
        t1_bar, t2_bar, fock_bar, mo_bar, ovoo_bar, ovov_bar, ovvv_bar = _grads_to_pyscf(g, nocc, nvir, packed)
        return t1_bar, t2_bar, mo_bar, fock_bar, ovoo_bar, ovov_bar, ovvv_bar, None


def kernel(mycc, eris, t1=None, t2=None, verbose=None, mode="fp64"):
    """E(T) for a converged CCSD object (pyscfad/cc/ccsd_t.py:28-80).

    ``mycc`` needs ``t1``/``t2`` only when they are not passed.  With torch
    inputs the returned 0-d tensor carries the custom VJP; otherwise a float.
    """
    if t1 is None:
        t1 = mycc.t1
    if t2 is None:
        t2 = mycc.t2
    args = (t1, t2, eris.mo_energy, eris.fock, eris.ovoo, eris.ovov, eris.ovvv)
    if any(isinstance(a, torch.Tensor) for a in args):
        dev = next(a.device for a in args if isinstance(a, torch.Tensor))
        if dev.type != "cuda":
            dev = _dev()
        targs = [a if isinstance(a, torch.Tensor) else _t(a, dev) for a in args]
        targs = [a.to(device=dev, dtype=torch.float64) for a in targs]
        return CCSDTKernel.apply(*targs, mode)
    dev = _dev()
    nvir = np.shape(t1)[1]
    ovvv_full = eris.get_ovvv() if hasattr(eris, "get_ovvv") else eris.ovvv
    if np.ndim(ovvv_full) == 3:
        from .eris import unpack_tril
        ovvv_full = unpack_tril(ovvv_full, nvir)
    L = kernel_layouts(t1, t2, eris.mo_energy, eris.fock, eris.ovoo, eris.ovov, ovvv_full, dev)
    return float(triples.energy(L, mode))


def _ccsd_t_energy_vjp(eris, t1, t2, et_bar, max_memory=None, mode="fp64"):
    """Backward of the (T) energy (pyscfad/cc/ccsd_t.py:82-192), numpy in/out."""
    del max_memory
    nocc, nvir = np.shape(t1)
    et_bar = 2.0 * float(et_bar)  # pyscfad/cc/ccsd_t.py:86
    packed = np.ndim(eris.ovvv) == 3
    ovvv_full = eris.get_ovvv() if hasattr(eris, "get_ovvv") else eris.ovvv
    if np.ndim(ovvv_full) == 3:
        from .eris import unpack_tril
        ovvv_full = unpack_tril(ovvv_full, nvir)
    L = kernel_layouts(t1, t2, eris.mo_energy, eris.fock, eris.ovoo, eris.ovov, ovvv_full)
    _, g = triples.energy_vjp(L, et_bar, None, mode)
    out = _grads_to_pyscf(g, nocc, nvir, packed)
    return tuple(np.ascontiguousarray(x.cpu().numpy()) for x in out)
