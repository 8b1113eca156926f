"""Density-fitted ERI producer for the (T) kernels, and its VJP, on the GPU.

pyscfad's DF-CCSD builds the (T) integrals from the three-index factors
(pyscfad/cc/dfccsd.py:73-88): with Lpq (naux, nmo, nmo),
Loo = Lpq[:, :o, :o], Lov = Lpq[:, :o, o:], Lvv = pack_tril(Lpq[:, o:, o:]),
ovoo = Lov^T Loo, ovov = Lov^T Lov, ovvv = Lov^T Lvv (packed); the (T) driver
then reshapes them into vooo and vvop (pyscfad/cc/ccsd_t.py:88-106).

``df_layouts`` forms the kernel layouts straight from the factors with the
library's float64 tensor-core kernels (C-ABI ``ct_df_layouts``):
    vvop[a, y, i, p] = sum_P Lov[P, i, a] R[P, p, y],  R = [Lov ; Lvv] over p,
    vooo[a, i, k, j] = sum_P Lov[P, i, a] Loo[P, j, k],
the transposes folded into the GEMMs' addressing, so neither the
(o, v, v, v) ovvv nor any host copy of vvop is formed.  ``df_factor_bar``
maps kernel-layout gradients of vvop and vooo back onto the factors by the
transposed contractions (``ct_df_factor_bar``), returning
(Loo_bar, Lov_bar, Lvv_bar) in the shapes of the inputs; a packed Lvv gets
the gradient of its packed entries (off-diagonal pairs summed, as the (T)
driver's ovvv gradient packing does at pyscfad/cc/ccsd_t.py:186-191).
torch only holds the device buffers and unpacks / splits the factors.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from .. import native

__all__ = ["df_layouts", "df_factor_bar"]


def _dev(device):
    if device is not None:
        dev = torch.device(device)
    elif torch.cuda.is_available():
        dev = torch.device("cuda", torch.cuda.current_device())
    else:
        raise native.CtError("pyscfad_b200.cc.df: no CUDA device available")
    if dev.type != "cuda":
        raise native.CtError("pyscfad_b200.cc.df runs on CUDA devices only")
    return dev


def _t(x, dev):
    if isinstance(x, torch.Tensor):
        return x.to(device=dev, dtype=torch.float64)
    return torch.as_tensor(np.asarray(x, dtype=np.float64), device=dev)


def _tril_idx(nvir, dev):
    idx, idy = np.tril_indices(nvir)
    return torch.as_tensor(idx, device=dev), torch.as_tensor(idy, device=dev)


def _factors(Loo, Lov, Lvv, nocc, nvir, dev):
    Loo = _t(Loo, dev)
    naux = Loo.shape[0]
    Loo = Loo.reshape(naux, nocc, nocc).contiguous()
    Lov = _t(Lov, dev).reshape(naux, nocc, nvir).contiguous()
    Lvv = _t(Lvv, dev)
    packed = Lvv.dim() == 2 and Lvv.shape[1] == nvir * (nvir + 1) // 2
    if packed:
        idx, idy = _tril_idx(nvir, dev)
        full = Lvv.new_zeros((naux, nvir, nvir))
        full[:, idx, idy] = Lvv
        full[:, idy, idx] = Lvv
        Lvv = full
    else:
        Lvv = Lvv.reshape(naux, nvir, nvir)
    return Loo, Lov, Lvv, packed


def _vp(t):
    return ctypes.c_void_p(t.data_ptr())


def _stream(dev):
    return ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)


def df_layouts(t1, t2, mo_energy, fock, Loo, Lov, Lvv, device=None) -> dict:
    """Kernel-layout tensors (mo_energy, t1T, t2T, vooo, fvo, vvop) from the DF
    factors on the device.  Loo (naux, o*o) or (naux, o, o); Lov (naux, o*v)
    or (naux, o, v); Lvv packed (naux, v(v+1)/2) or full (naux, v, v)."""
    dev = _dev(device)
    t1, t2 = _t(t1, dev), _t(t2, dev)
    nocc, nvir = t1.shape
    n = nocc + nvir
    Loo, Lov, Lvv, _ = _factors(Loo, Lov, Lvv, nocc, nvir, dev)
    naux = Loo.shape[0]
    R = torch.cat([Lov, Lvv], dim=1).contiguous()                      # [P, p, y]
    vvop = torch.empty((nvir, nvir, nocc, n), dtype=torch.float64, device=dev)
    vooo = torch.empty((nvir, nocc, nocc, nocc), dtype=torch.float64, device=dev)
    with torch.cuda.device(dev):
        native.check(native.lib().ct_df_layouts(nocc, nvir, naux, _vp(Loo), _vp(Lov), _vp(R), _vp(vooo), _vp(vvop),
                                                _stream(dev)), "ct_df_layouts")
    fock = _t(fock, dev)
    return dict(mo_energy=_t(mo_energy, dev).contiguous(), t1T=t1.t().contiguous(),
                t2T=t2.permute(2, 3, 1, 0).contiguous(), vooo=vooo, fvo=fock[nocc:, :nocc].contiguous(),
                vvop=vvop)


def df_factor_bar(g: dict, Loo, Lov, Lvv):
    """(Loo_bar, Lov_bar, Lvv_bar) from the kernel-layout gradients g["vvop"]
    and g["vooo"] (the chain rule through df_layouts), on g's device."""
    vvop_bar = g["vvop"].contiguous()
    vooo_bar = g["vooo"].contiguous()
    dev = _dev(vvop_bar.device)
    nvir, _, nocc, n = vvop_bar.shape
    Loo_in, Lov_in, Lvv_in = Loo, Lov, Lvv
    Loo, Lov, Lvv, packed = _factors(Loo, Lov, Lvv, nocc, nvir, dev)
    naux = Loo.shape[0]
    Rt = torch.cat([Lov, Lvv], dim=1).permute(0, 2, 1).contiguous()   # [P, y, p]
    dLoo = torch.zeros_like(Loo)
    dLov = torch.zeros_like(Lov)
    dRt = torch.zeros_like(Rt)
    with torch.cuda.device(dev):
        native.check(native.lib().ct_df_factor_bar(nocc, nvir, naux, _vp(Loo), _vp(Lov), _vp(Rt), _vp(vooo_bar),
                                                   _vp(vvop_bar), _vp(dLoo), _vp(dLov), _vp(dRt), _stream(dev)),
                     "ct_df_factor_bar")
    dR = dRt.permute(0, 2, 1)                                            # [P, p, y]
    dLov = dLov + dR[:, :nocc]
    dLvv = dR[:, nocc:].contiguous()
    if packed:
        idx, idy = _tril_idx(nvir, dev)
        sym = dLvv + dLvv.transpose(1, 2)
        ii = torch.arange(nvir, device=dev)
        sym[:, ii, ii] *= 0.5
        dLvv = sym[:, idx, idy]
    shape = lambda x: tuple(np.shape(x))  # noqa: E731
    return (dLoo.reshape(shape(Loo_in)), dLov.reshape(shape(Lov_in)), dLvv.reshape(shape(Lvv_in)))
