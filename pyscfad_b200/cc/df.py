"""Density-fitted ERI producer for the (T) kernels, and its VJP.

pyscfad's DF-CCSD builds the (T) integrals from the three-index factors
(pyscfad/cc/dfccsd.py:73-88): with Lpq (naux, nmo, nmo),
Loo = Lpq[:, :o, :o], Lov = Lpq[:, :o, o:], Lvv = pack_tril(Lpq[:, o:, o:]),
ovoo = Lov^T Loo, ovov = Lov^T Lov, ovvv = Lov^T Lvv (packed); the (T) driver
then reshapes them into vooo and vvop (pyscfad/cc/ccsd_t.py:88-106).

``df_layouts`` forms the kernel layouts straight from the factors on the
device, one slab of virtual indices at a time (float64 library GEMMs):
    vvop[a, y, i, p] = sum_P Lov[P, i, a] R[P, p, y],  R = [Lov ; Lvv] over p,
    vooo[a, i, k, j] = sum_P Lov[P, i, a] Loo[P, j, k],
so neither the (o, v, v, v) ovvv nor any host copy of vvop is formed.
``df_factor_bar`` maps kernel-layout gradients of vvop and vooo back onto the
factors by the transposed contractions (the same slabs), returning
(Loo_bar, Lov_bar, Lvv_bar) in the shapes of the inputs; a packed Lvv gets the
gradient of its packed entries (off-diagonal pairs summed, as the (T) driver's
ovvv gradient packing does at pyscfad/cc/ccsd_t.py:186-191).
"""
from __future__ import annotations

import numpy as np
import torch

__all__ = ["df_layouts", "df_factor_bar"]


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
    Loo = Loo.reshape(naux, nocc, nocc)
    Lov = _t(Lov, dev).reshape(naux, nocc, nvir)
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


def df_layouts(t1, t2, mo_energy, fock, Loo, Lov, Lvv, device=None, chunk: int = 32) -> dict:
    """Kernel-layout tensors (mo_energy, t1T, t2T, vooo, fvo, vvop) from the DF
    factors.  Loo (naux, o*o) or (naux, o, o); Lov (naux, o*v) or (naux, o, v);
    Lvv packed (naux, v(v+1)/2) or full (naux, v, v)."""
    dev = torch.device(device) if device is not None else (
        torch.device("cuda", torch.cuda.current_device()) if torch.cuda.is_available() else torch.device("cpu"))
    t1, t2 = _t(t1, dev), _t(t2, dev)
    nocc, nvir = t1.shape
    n = nocc + nvir
    Loo, Lov, Lvv, _ = _factors(Loo, Lov, Lvv, nocc, nvir, dev)
    naux = Loo.shape[0]
    R = torch.cat([Lov, Lvv], dim=1).reshape(naux, n * nvir)          # [P, (p, y)]
    vvop = torch.empty((nvir, nvir, nocc, n), dtype=torch.float64, device=dev)
    for a0 in range(0, nvir, chunk):
        a1 = min(nvir, a0 + chunk)
        M = Lov[:, :, a0:a1].reshape(naux, -1)                          # [P, (i, a)]
        G = (M.t() @ R).view(nocc, a1 - a0, n, nvir)                    # [i, a, p, y]
        vvop[a0:a1] = G.permute(1, 3, 0, 2)
        del G
    vooo = (Lov.reshape(naux, -1).t() @ Loo.reshape(naux, -1)).view(nocc, nvir, nocc, nocc)
    vooo = vooo.permute(1, 0, 3, 2).contiguous()                        # [a, i, k, j] = ovoo[i, a, j, k]
    fock = _t(fock, dev)
    return dict(mo_energy=_t(mo_energy, dev).contiguous(), t1T=t1.t().contiguous(),
                t2T=t2.permute(2, 3, 1, 0).contiguous(), vooo=vooo, fvo=fock[nocc:, :nocc].contiguous(),
                vvop=vvop)


def df_factor_bar(g: dict, Loo, Lov, Lvv, chunk: int = 32):
    """(Loo_bar, Lov_bar, Lvv_bar) from the kernel-layout gradients g["vvop"]
    and g["vooo"] (the chain rule through df_layouts), on g's device."""
    vvop_bar, vooo_bar = g["vvop"], g["vooo"]
    dev = vvop_bar.device
    nvir, _, nocc, n = vvop_bar.shape
    Loo_in, Lov_in, Lvv_in = Loo, Lov, Lvv
    Loo, Lov, Lvv, packed = _factors(Loo, Lov, Lvv, nocc, nvir, dev)
    naux = Loo.shape[0]
    R = torch.cat([Lov, Lvv], dim=1).reshape(naux, n * nvir)
    dLov = torch.zeros_like(Lov)                                         # [P, i, a]
    dR = torch.zeros((naux, n * nvir), dtype=torch.float64, device=dev)
    for a0 in range(0, nvir, chunk):
        a1 = min(nvir, a0 + chunk)
        Gb = vvop_bar[a0:a1].permute(2, 0, 3, 1).reshape(nocc * (a1 - a0), n * nvir)   # [(i, a), (p, y)]
        M = Lov[:, :, a0:a1].reshape(naux, -1)
        dLov[:, :, a0:a1] += (R @ Gb.t()).view(naux, nocc, a1 - a0)
        dR += M @ Gb
    dR = dR.view(naux, n, nvir)
    dLov += dR[:, :nocc]
    dLvv = dR[:, nocc:]
    # vooo[a, i, k, j] = sum_P Lov[P, i, a] Loo[P, j, k]
    Vb = vooo_bar.permute(1, 0, 3, 2).reshape(nocc * nvir, nocc * nocc)  # [(i, a), (j, k)]
    dLov += (Loo.reshape(naux, -1) @ Vb.t()).view(naux, nocc, nvir)
    dLoo = (Lov.reshape(naux, -1) @ Vb).view(naux, nocc, nocc)
    if packed:
        idx, idy = _tril_idx(nvir, dev)
        sym = dLvv + dLvv.transpose(1, 2)
        ii = torch.arange(nvir, device=dev)
        sym[:, ii, ii] *= 0.5
        dLvv = sym[:, idx, idy]
    shape = lambda x: tuple(np.shape(x))
    return (dLoo.reshape(shape(Loo_in)), dLov.reshape(shape(Lov_in)),
            dLvv.reshape(shape(Lvv_in)))
