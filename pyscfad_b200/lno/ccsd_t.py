"""Impurity (LNO) (T) correction on B200 — drop-in for pyscfad.lno.ccsd_t.

Mirrors pyscfad/lno/ccsd_t.py:
  * ``kernel(mycc, eris, ulo, t1, t2, verbose)`` (:34-58): mat = ulo^T ulo and
    E = _ccsd_t_energy(mat, t1T, t2T, mo_energy, fvo, ovoo, ovov, ovvv).
  * ``_ccsd_t_energy(mat, t1T, t2T, mo_energy, fvo, ovoo, ovov, ovvv,
    max_memory)`` (:70-113): the LNO-projected sum of lnoccsdt_contract over
    every LNO job, times 2/3; differentiable in every tensor argument, like the
    reference's custom_vjp (:115-237): the backward scales the cotangent by
    2/3, runs the hand-written VJP and returns (mat_bar, t1T_bar, t2T_bar,
    mo_energy_bar, fvo_bar, ovoo_bar, ovov_bar, ovvv_bar) with ovvv_bar
    symmetrised and packed lower-triangular when ovvv is packed (:224-235).

Both directions run on the float64 CUDA kernels of this package by default;
``mode="tf32"`` or ``"bf16x3"`` (an addition, nocc % 8 == 0) runs their
contractions on the tensor cores.  max_memory is accepted for signature
compatibility: vvop stays resident on the device.
"""
from __future__ import annotations

import numpy as np
import torch

from .. import triples
from ..cc.eris import pack_tril, unpack_tril

__all__ = ["kernel", "_ccsd_t_energy", "lno_layouts", "LNOTriples"]


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


def lno_layouts(t1T, t2T, mo_energy, fvo, ovoo, ovov, ovvv, device=None) -> dict:
    """Kernel-layout tensors as pyscfad/lno/ccsd_t.py:76-88 builds them: vooo =
    ovoo.transpose(1,0,3,2); vvop (v,v,o,nmo) with [:,:,:,:o] =
    ovov.transpose(1,3,0,2) and [:,:,:,o:] = ovvv.transpose(1,3,0,2), ovvv
    unpacked from (o, v, v(v+1)/2) when packed (get_ovvv, :60-67)."""
    dev = _dev(device)
    t1T, t2T = _t(t1T, dev), _t(t2T, dev)
    nvir, nocc = t1T.shape
    ovoo, ovov, ovvv = _t(ovoo, dev), _t(ovov, dev), _t(ovvv, dev)
    if ovvv.dim() == 3:
        ovvv = unpack_tril(ovvv, nvir)
    vvop = torch.empty((nvir, nvir, nocc, nocc + nvir), dtype=torch.float64, device=dev)
    vvop[:, :, :, :nocc] = ovov.permute(1, 3, 0, 2)
    vvop[:, :, :, nocc:] = ovvv.permute(1, 3, 0, 2)
    return dict(mo_energy=_t(mo_energy, dev).contiguous(), t1T=t1T.contiguous(), t2T=t2T.contiguous(),
                vooo=ovoo.permute(1, 0, 3, 2).contiguous(), fvo=_t(fvo, dev).contiguous(), vvop=vvop)


def lno_grads_to_pyscf(g: dict, nocc: int, nvir: int, packed: bool):
    """(ovoo_bar, ovov_bar, ovvv_bar) from kernel-layout gradients
    (pyscfad/lno/ccsd_t.py:224-235)."""
    ovoo_bar = g["vooo"].permute(1, 0, 3, 2)
    ovov_bar = g["vvop"][:, :, :, :nocc].permute(2, 0, 3, 1)
    ovvv_bar = g["vvop"][:, :, :, nocc:].permute(2, 0, 3, 1)
    if packed:
        ovvv_bar = ovvv_bar + ovvv_bar.transpose(2, 3)
        ii = torch.arange(nvir, device=ovvv_bar.device)
        ovvv_bar[:, :, ii, ii] *= .5
        ovvv_bar = pack_tril(ovvv_bar)
    return ovoo_bar, ovov_bar, ovvv_bar


class LNOTriples(torch.autograd.Function):
    """_ccsd_t_energy(mat, t1T, t2T, mo_energy, fvo, ovoo, ovov, ovvv) with the
    hand-written VJP (the torch counterpart of the reference's custom_vjp)."""

    @staticmethod
    def forward(ctx, mat, t1T, t2T, mo_energy, fvo, ovoo, ovov, ovvv, mode="fp64"):
        nvir, nocc = t1T.shape
        L = lno_layouts(t1T, t2T, mo_energy, fvo, ovoo, ovov, ovvv, device=t1T.device)
        m = mat.to(device=t1T.device, dtype=torch.float64).contiguous()
        ctx.L, ctx.mat, ctx.mode = L, m, mode
        ctx.meta = (nocc, nvir, ovvv.dim() == 3)
        return triples.lno_energy(L, m, mode=mode) * (2.0 / 3.0)   # pyscfad/lno/ccsd_t.py:111

    @staticmethod
    def backward(ctx, gE):
        nocc, nvir, packed = ctx.meta
        et_bar = float(gE) * (2.0 / 3.0)                  # pyscfad/lno/ccsd_t.py:127
        _, mat_bar, g = triples.lno_energy_vjp(ctx.L, ctx.mat, et_bar, mode=ctx.mode)
        ctx.L = ctx.mat = None
        ovoo_bar, ovov_bar, ovvv_bar = lno_grads_to_pyscf(g, nocc, nvir, packed)
        return mat_bar, g["t1T"], g["t2T"], g["mo_energy"], g["fvo"], ovoo_bar, ovov_bar, ovvv_bar, None


def _ccsd_t_energy(mat, t1T, t2T, mo_energy, fvo, ovoo, ovov, ovvv, max_memory=None, mode="fp64"):
    """The LNO (T) energy (pyscfad/lno/ccsd_t.py:70-113).  Torch inputs give a
    differentiable 0-d tensor; numpy inputs a float."""
    del max_memory
    args = (mat, t1T, t2T, mo_energy, fvo, ovoo, ovov, ovvv)
    if any(isinstance(a, torch.Tensor) for a in args):
        dev = next(a.device for a in args if isinstance(a, torch.Tensor))
        if dev.type != "cuda":
            dev = _dev()
        targs = [(a if isinstance(a, torch.Tensor) else _t(a, dev)).to(device=dev, dtype=torch.float64)
                 for a in args]
        return LNOTriples.apply(*targs, mode)
    dev = _dev()
    L = lno_layouts(t1T, t2T, mo_energy, fvo, ovoo, ovov, ovvv, dev)
    return float(triples.lno_energy(L, _t(mat, dev).contiguous(), mode=mode)) * 2.0 / 3.0


def kernel(mycc, eris, ulo, t1=None, t2=None, verbose=None, mode="fp64"):
    """LNO (T) correction (pyscfad/lno/ccsd_t.py:34-58): mat = ulo^T ulo, so a
    torch ``ulo`` that requires grad carries the gradient through mat."""
    if t1 is None:
        t1 = mycc.t1
    if t2 is None:
        t2 = mycc.t2
    torch_in = any(isinstance(a, torch.Tensor) for a in (ulo, t1, t2))
    if torch_in:
        dev = next(a.device for a in (ulo, t1, t2) if isinstance(a, torch.Tensor))
        if dev.type != "cuda":
            dev = _dev()
        ulo, t1, t2 = (_t(a, dev) for a in (ulo, t1, t2))
        mat = ulo.t() @ ulo
        t1T, t2T = t1.t(), t2.permute(2, 3, 1, 0)
    else:
        mat = np.dot(np.asarray(ulo).T, np.asarray(ulo))
        t1T, t2T = np.asarray(t1).T, np.asarray(t2).transpose(2, 3, 1, 0)
    nocc = t1T.shape[1]
    fvo = eris.fock[nocc:, :nocc]
    return _ccsd_t_energy(mat, t1T, t2T, eris.mo_energy, fvo, eris.ovoo, eris.ovov, eris.ovvv,
                          getattr(mycc, "max_memory", None), mode=mode)
