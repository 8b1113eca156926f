"""Minimal ERI container with the attribute names pyscfad's (T) driver reads
(pyscfad/cc/ccsd.py:470-498, _ChemistsERIs): fock, mo_energy, ovoo, ovov and
ovvv, the latter either full (nocc, nvir, nvir, nvir) or packed lower-triangular
in its last two indices (nocc, nvir, nvir(nvir+1)/2) as the DF-CCSD path stores
it (pyscfad/cc/dfccsd.py:88).  Any object with these attributes works in its
place.
"""
from __future__ import annotations

import dataclasses
import numpy as np


def unpack_tril(tril, nvir: int):
    """(..., nvir(nvir+1)/2) -> (..., nvir, nvir), symmetric (numpy.tril_indices order)."""
    try:
        import torch
        if isinstance(tril, torch.Tensor):
            idx, idy = np.tril_indices(nvir)
            out = tril.new_zeros(tril.shape[:-1] + (nvir, nvir))
            out[..., idx, idy] = tril
            out[..., idy, idx] = tril
            return out
    except ImportError:  # pragma: no cover
        pass
    tril = np.asarray(tril)
    idx, idy = np.tril_indices(nvir)
    out = np.zeros(tril.shape[:-1] + (nvir, nvir), dtype=tril.dtype)
    out[..., idx, idy] = tril
    out[..., idy, idx] = tril
    return out


def pack_tril(mat):
    nvir = mat.shape[-1]
    idx, idy = np.tril_indices(nvir)
    return mat[..., idx, idy]


@dataclasses.dataclass
class ERIs:
    fock: object
    mo_energy: object
    ovoo: object
    ovov: object
    ovvv: object

    @property
    def nocc(self) -> int:
        return self.ovoo.shape[0]

    def ovvv_is_packed(self) -> bool:
        return len(self.ovvv.shape) == 3

    def get_ovvv(self):
        if self.ovvv_is_packed():
            return unpack_tril(self.ovvv, self.ovoo.shape[1])
        return self.ovvv

    @classmethod
    def from_system(cls, s, packed: bool = False):
        ovvv = pack_tril(s.ovvv) if packed else s.ovvv
        return cls(fock=s.fock, mo_energy=s.mo_energy, ovoo=s.ovoo, ovov=s.ovov, ovvv=ovvv)
