"""Seeded synthetic CCSD(T) inputs.

The systems follow one fixed recipe so that the CPU oracle, the GPU kernels and
the benchmark all see bit-identical inputs for a given seed:

* orbital energies: occupied sorted U[-2.0, -0.3] Eh, virtual sorted U[0.1, 3.0] Eh;
* MO ERIs (pq|rs) = sum_P B_pq^P B_rs^P with B = (X + X^T_pq)/2, X ~ N(0,1)/sqrt(naux);
  only the ovov / ovoo / ovvv slices that the (T) kernel reads are formed;
* t1 ~ N(0, (1e-4)^2), shape (nocc, nvir);
* t2 = (Y + Y.transpose(1,0,3,2))/2, Y ~ N(0, (1e-2)^2), so t2[i,j,a,b] = t2[j,i,b,a];
* fock = diag(mo_energy) (so fvo = 0) unless ``fvo_sigma`` > 0, in which case the
  virtual-occupied block gets N(0, fvo_sigma^2) entries so that the fvo path of
  the VJP is exercised.

Draw order from ``numpy.random.default_rng(seed)``: e_occ, e_vir, X, t1, Y, fvo.

The ERI slices are contracted on the GPU (torch float64 matmul) when one is
available and the system is large; the result is the same arithmetic either way
up to float64 rounding.
"""
from __future__ import annotations

import dataclasses
import numpy as np

__all__ = ["System", "make_system", "reference_layouts", "CONFIGS", "config_system"]


@dataclasses.dataclass
class System:
    nocc: int
    nvir: int
    mo_energy: np.ndarray      # (nmo,)
    fock: np.ndarray           # (nmo, nmo)
    t1: np.ndarray             # (nocc, nvir)
    t2: np.ndarray             # (nocc, nocc, nvir, nvir)
    ovov: np.ndarray           # (nocc, nvir, nocc, nvir)
    ovoo: np.ndarray           # (nocc, nvir, nocc, nocc)
    ovvv: np.ndarray           # (nocc, nvir, nvir, nvir), symmetric in the last two

    @property
    def nmo(self) -> int:
        return self.nocc + self.nvir


# benchmark workloads (nocc, nvir, naux, seed)
CONFIGS = {
    1: (8, 40, 120, 0),
    2: (16, 120, 400, 1),
    3: (32, 300, 900, 2),
    4: (48, 500, 1500, 3),
}


def _eri_slices(B: np.ndarray, nocc: int, device=None):
    """ovov, ovoo, ovvv from the symmetric DF factor B (naux, nmo, nmo)."""
    naux, nmo, _ = B.shape
    nvir = nmo - nocc
    if device is not None:
        import torch
        Bt = torch.from_numpy(B).to(device)
        Bov = Bt[:, :nocc, nocc:].reshape(naux, -1)
        Boo = Bt[:, :nocc, :nocc].reshape(naux, -1)
        Bvv = Bt[:, nocc:, nocc:].reshape(naux, -1)
        ovov = (Bov.T @ Bov).reshape(nocc, nvir, nocc, nvir).cpu().numpy()
        ovoo = (Bov.T @ Boo).reshape(nocc, nvir, nocc, nocc).cpu().numpy()
        ovvv = (Bov.T @ Bvv).reshape(nocc, nvir, nvir, nvir).cpu().numpy()
        del Bt, Bov, Boo, Bvv
        torch.cuda.empty_cache()
        return ovov, ovoo, ovvv
    Bov = np.ascontiguousarray(B[:, :nocc, nocc:]).reshape(naux, -1)
    Boo = np.ascontiguousarray(B[:, :nocc, :nocc]).reshape(naux, -1)
    Bvv = np.ascontiguousarray(B[:, nocc:, nocc:]).reshape(naux, -1)
    ovov = (Bov.T @ Bov).reshape(nocc, nvir, nocc, nvir)
    ovoo = (Bov.T @ Boo).reshape(nocc, nvir, nocc, nocc)
    ovvv = (Bov.T @ Bvv).reshape(nocc, nvir, nvir, nvir)
    return ovov, ovoo, ovvv


def make_system(nocc: int, nvir: int, naux: int, seed: int,
                fvo_sigma: float = 0.0, eri_scale: float = 1.0,
                device=None) -> System:
    """Build one seeded synthetic system (see module docstring for the recipe).

    ``eri_scale`` multiplies every ERI slice (E(T) scales as its square); it is
    1 for the benchmark workloads and only used for clearly labelled
    physical-scale variants.
    """
    rng = np.random.default_rng(seed)
    nmo = nocc + nvir
    e_occ = np.sort(rng.uniform(-2.0, -0.3, nocc))
    e_vir = np.sort(rng.uniform(0.1, 3.0, nvir))
    mo_energy = np.concatenate([e_occ, e_vir])
    X = rng.standard_normal((naux, nmo, nmo)) / np.sqrt(naux)
    B = (X + X.transpose(0, 2, 1)) * 0.5
    del X
    t1 = 1e-4 * rng.standard_normal((nocc, nvir))
    Y = 1e-2 * rng.standard_normal((nocc, nocc, nvir, nvir))
    t2 = (Y + Y.transpose(1, 0, 3, 2)) * 0.5
    del Y
    fock = np.diag(mo_energy)
    if fvo_sigma > 0:
        fvo = fvo_sigma * rng.standard_normal((nvir, nocc))
        fock = fock.copy()
        fock[nocc:, :nocc] = fvo
        fock[:nocc, nocc:] = fvo.T
    if device is None and nmo * nmo * naux > 4e7:
        try:
            import torch
            if torch.cuda.is_available():
                device = "cuda"
        except Exception:  # pragma: no cover - torch always present here
            device = None
    ovov, ovoo, ovvv = _eri_slices(B, nocc, device)
    if eri_scale != 1.0:
        ovov = ovov * eri_scale
        ovoo = ovoo * eri_scale
        ovvv = ovvv * eri_scale
    return System(nocc, nvir, mo_energy, fock, t1, t2, ovov, ovoo, ovvv)


def config_system(cfg: int, **kw) -> System:
    nocc, nvir, naux, seed = CONFIGS[cfg]
    return make_system(nocc, nvir, naux, seed, **kw)


# Physical-scale variants: every ERI slice multiplied by a power of two s so
# that |E(T)| of the whole system is about 1e-2 Eh (E(T) scales as s^2; the
# generator's own systems have |E(T)| ~ 1e2 - 1e7 Eh).  A power of two scales
# every intermediate of every precision mode exactly (no rounding changes), so
# a mode's energy at scale s is exactly s^2 times its energy at scale 1 and
# its error against float64 scales by s^2 as well.
PHYSICAL_ERI_SCALE = {3: 2.0 ** -14, 4: 2.0 ** -16}


def device_layouts(nocc: int, nvir: int, naux: int, seed: int, device="cuda",
                   fvo_sigma: float = 0.0, chunk: int = 32, eri_scale: float = 1.0) -> dict:
    """Kernel-layout tensors built directly on the device (same draws as
    ``make_system``; the ERI contractions run as float64 torch matmuls in
    virtual-index chunks so no host copy of vvop is ever formed).
    ``eri_scale`` multiplies vvop and vooo (see PHYSICAL_ERI_SCALE)."""
    import torch
    rng = np.random.default_rng(seed)
    o, v = nocc, nvir
    n = o + v
    e_occ = np.sort(rng.uniform(-2.0, -0.3, o))
    e_vir = np.sort(rng.uniform(0.1, 3.0, v))
    mo_energy = np.concatenate([e_occ, e_vir])
    X = rng.standard_normal((naux, n, n))
    Bt = torch.from_numpy(X).to(device)
    del X
    Bt = (Bt + Bt.transpose(1, 2)) * (0.5 / np.sqrt(naux))
    t1 = 1e-4 * rng.standard_normal((o, v))
    Y = rng.standard_normal((o, o, v, v))
    Yt = torch.from_numpy(Y).to(device)
    del Y
    t2 = (Yt + Yt.permute(1, 0, 3, 2)) * 0.5e-2
    del Yt
    t2T = t2.permute(2, 3, 1, 0).contiguous()
    del t2
    fock = np.diag(mo_energy)
    if fvo_sigma > 0:
        fvo = fvo_sigma * rng.standard_normal((v, o))
    else:
        fvo = np.zeros((v, o))
    Lia = Bt[:, :o, o:].contiguous()                  # (naux, o, v)
    R = Bt[:, :, o:].reshape(naux, n * v)             # (naux, n*v): [p, b]
    vvop = torch.empty((v, v, o, n), dtype=torch.float64, device=device)
    for a0 in range(0, v, chunk):
        a1 = min(v, a0 + chunk)
        L = Lia[:, :, a0:a1].reshape(naux, -1)        # (naux, o*da): [i, a]
        G = (L.t() @ R).view(o, a1 - a0, n, v)        # [i, a, p, b] = (ia|pb)
        vvop[a0:a1] = G.permute(1, 3, 0, 2)
        del G
    Boo = Bt[:, :o, :o].reshape(naux, o * o)
    vooo = (Lia.reshape(naux, o * v).t() @ Boo).view(o, v, o, o).permute(1, 0, 3, 2).contiguous()
    del Bt, Lia, R, Boo
    if eri_scale != 1.0:
        vvop.mul_(eri_scale)
        vooo.mul_(eri_scale)
    torch.cuda.empty_cache()
    f64 = dict(dtype=torch.float64, device=device)
    return dict(mo_energy=torch.tensor(mo_energy, **f64), t1T=torch.tensor(t1.T.copy(), **f64),
                t2T=t2T, vooo=vooo, fvo=torch.tensor(fvo, **f64), vvop=vvop)


def reference_layouts(s: System):
    """The kernel-facing tensors in the layouts pyscfad's (T) VJP driver builds.

    Mirrors pyscfad/cc/ccsd_t.py:88-106: t1T (v,o); t2T = t2.transpose(2,3,1,0)
    (v,v,o,o) indexed [a,b,j,i]; vooo = ovoo.transpose(1,0,3,2) (v,o,o,o);
    vvop (v,v,o,nmo) with [:,:,:,:o] = ovov.transpose(1,3,0,2) and
    [:,:,:,o:] = ovvv.transpose(1,3,0,2); fvo = fock[o:, :o].
    """
    o, v = s.nocc, s.nvir
    t1T = np.ascontiguousarray(s.t1.T)
    t2T = np.ascontiguousarray(s.t2.transpose(2, 3, 1, 0))
    vooo = np.ascontiguousarray(s.ovoo.transpose(1, 0, 3, 2))
    vvop = np.empty((v, v, o, o + v))
    vvop[:, :, :, :o] = s.ovov.transpose(1, 3, 0, 2)
    vvop[:, :, :, o:] = s.ovvv.transpose(1, 3, 0, 2)
    fvo = np.ascontiguousarray(s.fock[o:, :o])
    mo_energy = np.ascontiguousarray(s.mo_energy)
    return dict(mo_energy=mo_energy, t1T=t1T, t2T=t2T, vooo=vooo, fvo=fvo, vvop=vvop)
