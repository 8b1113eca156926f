"""CPU: the DF ERI producer's oracle (oracle/df_np.py) against the reference's
DF formulas (pyscfad/cc/dfccsd.py:73-88 + pyscfad/cc/ccsd_t.py:88-106, through
synth.reference_layouts), its VJP against central finite differences and
against the reference's own gradient chain; and that the product module
refuses to run without a CUDA device."""
import numpy as np
import pytest
import torch

import golden_io
from oracle import df_np
from pyscfad_b200 import native, synth
from pyscfad_b200.cc import df
from pyscfad_b200.cc.eris import pack_tril


def _factors(o, v, naux, seed):
    g = np.random.default_rng(seed)
    n = o + v
    X = g.standard_normal((naux, n, n)) / np.sqrt(naux)
    Lpq = 0.5 * (X + X.transpose(0, 2, 1))
    Loo = Lpq[:, :o, :o].reshape(naux, -1)
    Lov = Lpq[:, :o, o:].reshape(naux, -1)
    Lvv = pack_tril(Lpq[:, o:, o:])
    t1 = 1e-2 * g.standard_normal((o, v))
    Y = 1e-2 * g.standard_normal((o, o, v, v))
    t2 = 0.5 * (Y + Y.transpose(1, 0, 3, 2))
    e = np.concatenate([np.sort(g.uniform(-2, -0.3, o)), np.sort(g.uniform(0.1, 3, v))])
    fock = np.diag(e)
    fock[o:, :o] = 1e-3 * g.standard_normal((v, o))
    return Lpq, Loo, Lov, Lvv, t1, t2, e, fock


@pytest.mark.parametrize("packed", [True, False])
def test_oracle_layouts_match_reference_formulas(packed):
    o, v, naux = 3, 7, 11
    Lpq, Loo, Lov, Lvv, t1, t2, e, fock = _factors(o, v, naux, 3)
    LovT = Lov.T
    ovoo = (LovT @ Loo).reshape(o, v, o, o)
    ovov = (LovT @ Lov).reshape(o, v, o, v)
    ovvv = np.einsum("Pia,Pbc->iabc", Lpq[:, :o, o:], Lpq[:, o:, o:])
    s = synth.System(nocc=o, nvir=v, mo_energy=e, fock=fock, t1=t1, t2=t2, ovov=ovov, ovoo=ovoo, ovvv=ovvv)
    Lr = synth.reference_layouts(s)
    vooo, vvop = df_np.vooo_vvop(Loo, Lov, Lvv if packed else Lpq[:, o:, o:], o, v)
    np.testing.assert_allclose(vooo, Lr["vooo"], rtol=1e-13, atol=1e-15)
    np.testing.assert_allclose(vvop, Lr["vvop"], rtol=1e-13, atol=1e-15)


@pytest.mark.parametrize("packed", [True, False])
def test_oracle_factor_bar_matches_central_differences(packed):
    o, v, naux = 3, 4, 5
    Lpq, Loo, Lov, Lvv, *_ = _factors(o, v, naux, 4)
    Lvv_in = Lvv if packed else Lpq[:, o:, o:].copy()
    g = np.random.default_rng(5)
    Gvv = g.standard_normal((v, v, o, o + v))
    Gvo = g.standard_normal((v, o, o, o))
    bars = df_np.factor_bar(Gvo, Gvv, Loo, Lov, Lvv_in, o, v)

    def f(Loo, Lov, Lvv):
        vooo, vvop = df_np.vooo_vvop(Loo, Lov, Lvv, o, v)
        return (vvop * Gvv).sum() + (vooo * Gvo).sum()

    h = 1e-5
    for which, (X, bar) in enumerate(zip((Loo, Lov, Lvv_in), bars)):
        assert bar.shape == X.shape
        d = g.standard_normal(X.shape)
        args_p = [Loo, Lov, Lvv_in]
        args_m = [Loo, Lov, Lvv_in]
        args_p[which] = X + h * d
        args_m[which] = X - h * d
        fd = (f(*args_p) - f(*args_m)) / (2 * h)
        assert abs(fd - (bar * d).sum()) <= 1e-7 * max(1.0, abs(fd)), (which, fd, (bar * d).sum())


def test_oracle_factor_bar_matches_the_reference_chain():
    """The same gradient as pyscfad's own chain: the (T) driver's output
    transforms (ovoo_bar, ovov_bar, packed ovvv_bar; pyscfad/cc/ccsd_t.py:179-191)
    pulled back through ovoo = Lov^T Loo, ovov = Lov^T Lov, ovvv = Lov^T Lvv
    (pyscfad/cc/dfccsd.py:80-88)."""
    from oracle import ref
    o, v, naux = 3, 5, 8
    Lpq, Loo, Lov, Lvv, t1, t2, e, fock = _factors(o, v, naux, 6)
    g = np.random.default_rng(7)
    G = {"mo_energy": np.zeros(o + v), "t1T": np.zeros((v, o)), "t2T": np.zeros((v, v, o, o)),
         "fvo": np.zeros((v, o)), "vooo": g.standard_normal((v, o, o, o)),
         "vvop": g.standard_normal((v, v, o, o + v))}
    pg = ref.to_pyscf_grads(G, o, v)
    ovoo_b = pg["ovoo"].reshape(o * v, o * o)
    ovov_b = pg["ovov"].reshape(o * v, o * v)
    ovvv_b = pg["ovvv"].reshape(o * v, -1)
    Loo_b = Lov @ ovoo_b
    Lov_b = Lov @ (ovov_b + ovov_b.T) + Loo @ ovoo_b.T + Lvv @ ovvv_b.T
    Lvv_b = Lov @ ovvv_b
    bars = df_np.factor_bar(G["vooo"], G["vvop"], Loo, Lov, Lvv, o, v)
    for want, got in zip((Loo_b, Lov_b, Lvv_b), bars):
        np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-13)


def test_product_module_needs_a_cuda_device():
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    o, v, naux = 2, 3, 4
    Lpq, Loo, Lov, Lvv, t1, t2, e, fock = _factors(o, v, naux, 8)
    with pytest.raises(native.CtError):
        df.df_layouts(t1, t2, e, fock, Loo, Lov, Lvv)
    with pytest.raises(native.CtError):
        df.df_layouts(t1, t2, e, fock, Loo, Lov, Lvv, device="cpu")
