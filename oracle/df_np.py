"""Oracle (test infrastructure): numpy restatement of the DF ERI producer of
the (T) inputs and its VJP.

Only tests use this module; the product never does.

Reference arithmetic: pyscfad's DF-CCSD forms, from Lpq (naux, nmo, nmo),
Loo = Lpq[:, :o, :o], Lov = Lpq[:, :o, o:], Lvv = Lpq[:, o:, o:] (stored
packed-tril), ovoo = Lov^T Loo, ovov = Lov^T Lov, ovvv = Lov^T Lvv
(pyscfad/cc/dfccsd.py:73-88); the (T) driver transposes them into
vooo = ovoo.transpose(1,0,3,2) and vvop = [ovov | ovvv].transpose(1,3,0,2)
(pyscfad/cc/ccsd_t.py:88-106).  The gradient of the factors is the chain
rule through those products; a packed Lvv receives the packed gradient with
off-diagonal pairs summed (as the driver packs the ovvv gradient,
pyscfad/cc/ccsd_t.py:186-191).
"""
from __future__ import annotations

import numpy as np


def unpack(Loo, Lov, Lvv, nocc, nvir):
    """(Loo (naux,o,o), Lov (naux,o,v), Lvv (naux,v,v), packed?)"""
    Loo = np.asarray(Loo, dtype=np.float64)
    naux = Loo.shape[0]
    Loo = Loo.reshape(naux, nocc, nocc)
    Lov = np.asarray(Lov, dtype=np.float64).reshape(naux, nocc, nvir)
    Lvv = np.asarray(Lvv, dtype=np.float64)
    packed = Lvv.ndim == 2 and Lvv.shape[1] == nvir * (nvir + 1) // 2
    if packed:
        idx, idy = np.tril_indices(nvir)
        full = np.zeros((naux, nvir, nvir))
        full[:, idx, idy] = Lvv
        full[:, idy, idx] = Lvv
        Lvv = full
    else:
        Lvv = Lvv.reshape(naux, nvir, nvir)
    return Loo, Lov, Lvv, packed


def vooo_vvop(Loo, Lov, Lvv, nocc, nvir):
    Loo, Lov, Lvv, _ = unpack(Loo, Lov, Lvv, nocc, nvir)
    ovoo = np.einsum("Pia,Pjk->iajk", Lov, Loo)
    ovov = np.einsum("Pia,Pjb->iajb", Lov, Lov)
    ovvv = np.einsum("Pia,Pbc->iabc", Lov, Lvv)
    vooo = np.ascontiguousarray(ovoo.transpose(1, 0, 3, 2))
    vvop = np.concatenate([ovov.transpose(1, 3, 0, 2), ovvv.transpose(1, 3, 0, 2)], axis=3)
    return vooo, np.ascontiguousarray(vvop)


def factor_bar(vooo_bar, vvop_bar, Loo, Lov, Lvv, nocc, nvir):
    """(Loo_bar, Lov_bar, Lvv_bar) in the shapes of the inputs."""
    shapes = [np.shape(x) for x in (Loo, Lov, Lvv)]
    Loo, Lov, Lvv, packed = unpack(Loo, Lov, Lvv, nocc, nvir)
    o = nocc
    ovoo_b = vooo_bar.transpose(1, 0, 3, 2)                       # [i, a, j, k]
    ovov_b = vvop_bar[:, :, :, :o].transpose(2, 0, 3, 1)           # [i, a, j, b]
    ovvv_b = vvop_bar[:, :, :, o:].transpose(2, 0, 3, 1)           # [i, a, b, c]
    dLov = (np.einsum("iajk,Pjk->Pia", ovoo_b, Loo)
            + np.einsum("iajb,Pjb->Pia", ovov_b, Lov) + np.einsum("iajb,Pia->Pjb", ovov_b, Lov)
            + np.einsum("iabc,Pbc->Pia", ovvv_b, Lvv))
    dLoo = np.einsum("iajk,Pia->Pjk", ovoo_b, Lov)
    dLvv = np.einsum("iabc,Pia->Pbc", ovvv_b, Lov)
    if packed:
        sym = dLvv + dLvv.transpose(0, 2, 1)
        ii = np.arange(nvir)
        sym[:, ii, ii] *= 0.5
        idx, idy = np.tril_indices(nvir)
        dLvv = sym[:, idx, idy]
    return dLoo.reshape(shapes[0]), dLov.reshape(shapes[1]), dLvv.reshape(shapes[2])
