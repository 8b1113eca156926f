"""GPU: the DF ERI producer kernels (ct_df_layouts, ct_df_factor_bar) against
the numpy oracle of pyscfad's DF formulas (oracle/df_np.py, checked on CPU
against pyscfad/cc/dfccsd.py:73-88 and the (T) driver's layouts), and the
whole chain: factors -> kernel layouts -> (T) energy and VJP -> factor
gradients, against central finite differences of E(T) in the factors.

Tolerances: float64 GEMMs vs float64 numpy, 1e-12 relative to each array's
norm; the chain's directional derivatives 1e-6 relative (h = 1e-4).
"""
import numpy as np
import pytest
import torch

from oracle import df_np
from pyscfad_b200 import triples
from pyscfad_b200.cc import df
from pyscfad_b200.cc.eris import pack_tril

pytestmark = pytest.mark.gpu


def _factors(o, v, naux, seed):
    g = np.random.default_rng(seed)
    n = o + v
    X = g.standard_normal((naux, n, n)) / np.sqrt(naux)
    Lpq = 0.5 * (X + X.transpose(0, 2, 1))
    t1 = 1e-2 * g.standard_normal((o, v))
    Y = 1e-2 * g.standard_normal((o, o, v, v))
    t2 = 0.5 * (Y + Y.transpose(1, 0, 3, 2))
    e = np.concatenate([np.sort(g.uniform(-2, -0.3, o)), np.sort(g.uniform(0.1, 3, v))])
    fock = np.diag(e)
    return (Lpq[:, :o, :o].reshape(naux, -1).copy(), Lpq[:, :o, o:].reshape(naux, -1).copy(),
            pack_tril(Lpq[:, o:, o:]), Lpq[:, o:, o:].copy(), t1, t2, e, fock)


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("shape", [(3, 7, 11), (8, 20, 40), (16, 37, 70)])
@pytest.mark.parametrize("packed", [True, False])
def test_df_kernels_match_oracle(shape, packed, cuda_dev):
    o, v, naux = shape
    Loo, Lov, Lvv_p, Lvv_f, t1, t2, e, fock = _factors(o, v, naux, sum(shape))
    Lvv = Lvv_p if packed else Lvv_f
    L = df.df_layouts(t1, t2, e, fock, Loo, Lov, Lvv, device=cuda_dev)
    vooo, vvop = df_np.vooo_vvop(Loo, Lov, Lvv, o, v)
    assert _rel(L["vooo"].cpu().numpy(), vooo) <= 1e-12
    assert _rel(L["vvop"].cpu().numpy(), vvop) <= 1e-12
    g = np.random.default_rng(3)
    Gvo, Gvv = g.standard_normal((v, o, o, o)), g.standard_normal((v, v, o, o + v))
    bars = df.df_factor_bar({"vooo": torch.from_numpy(Gvo).to(cuda_dev), "vvop": torch.from_numpy(Gvv).to(cuda_dev)},
                            Loo, Lov, Lvv)
    want = df_np.factor_bar(Gvo, Gvv, Loo, Lov, Lvv, o, v)
    for got, w in zip(bars, want):
        assert tuple(got.shape) == w.shape
        assert _rel(got.cpu().numpy(), w) <= 1e-12


def test_df_chain_through_the_triples_vjp(cuda_dev):
    """dE(T)/d(factors) from the kernels' VJP chained through ct_df_factor_bar,
    against central differences of E(T) computed from perturbed factors."""
    o, v, naux = 8, 24, 48
    Loo, Lov, Lvv, _, t1, t2, e, fock = _factors(o, v, naux, 11)

    def energy(Loo, Lov, Lvv):
        L = df.df_layouts(t1, t2, e, fock, Loo, Lov, Lvv, device=cuda_dev)
        return float(triples.energy(L, mode="fp64"))

    L = df.df_layouts(t1, t2, e, fock, Loo, Lov, Lvv, device=cuda_dev)
    _, grads = triples.energy_vjp(L, 2.0, mode="fp64")   # kernel et_bar = 2 x the cotangent of E(T)
    bars = df.df_factor_bar(grads, Loo, Lov, Lvv)
    g = np.random.default_rng(12)
    h = 1e-4
    for which, X in enumerate((Loo, Lov, Lvv)):
        d = g.standard_normal(X.shape)
        args_p, args_m = [Loo, Lov, Lvv], [Loo, Lov, Lvv]
        args_p[which] = X + h * d
        args_m[which] = X - h * d
        fd = (energy(*args_p) - energy(*args_m)) / (2 * h)
        an = float((bars[which].cpu().numpy() * d).sum())
        assert abs(fd - an) <= 1e-6 * max(abs(fd), 1e-12), (which, fd, an)
