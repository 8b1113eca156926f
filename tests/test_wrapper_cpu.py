"""CPU: the host-side layout logic of the pyscfad-facing wrapper
(pyscfad_b200.cc.ccsd_t) on CPU tensors, against the numpy restatement of the
reference driver's transforms (pyscfad/cc/ccsd_t.py:88-106 and :179-191)."""
import numpy as np
import torch

import golden_io
from oracle import ref
from pyscfad_b200 import synth
from pyscfad_b200.cc import ccsd_t as cct
from pyscfad_b200.cc.eris import pack_tril, unpack_tril


def test_kernel_layouts_match_reference_driver():
    meta, _ = golden_io.load("small_o4v10_fvo")
    s = golden_io.system(meta)
    L = cct.kernel_layouts(s.t1, s.t2, s.mo_energy, s.fock, s.ovoo, s.ovov, s.ovvv, device="cpu")
    Lr = synth.reference_layouts(s)
    for k in golden_io.KEYS:
        assert L[k].is_contiguous(), k
        np.testing.assert_array_equal(L[k].numpy(), Lr[k], err_msg=k)


def test_gradient_untranspose_and_packed_ovvv():
    o, v = 3, 5
    g = np.random.default_rng(3)
    shapes = dict(mo_energy=(o + v,), t1T=(v, o), t2T=(v, v, o, o), vooo=(v, o, o, o), fvo=(v, o),
                  vvop=(v, v, o, o + v))
    G = {k: g.standard_normal(sh) for k, sh in shapes.items()}
    out = cct._grads_to_pyscf({k: torch.from_numpy(x) for k, x in G.items()}, o, v, packed=True)
    exp = ref.to_pyscf_grads(G, o, v)
    names = ("t1", "t2", "fock", "mo_energy", "ovoo", "ovov", "ovvv")
    for name, x in zip(names, out):
        np.testing.assert_allclose(x.numpy(), exp[name], rtol=0, atol=1e-15, err_msg=name)


def test_tril_pack_roundtrip():
    v = 6
    x = np.random.default_rng(4).standard_normal((2, 3, v, v))
    sym = x + x.transpose(0, 1, 3, 2)
    np.testing.assert_array_equal(unpack_tril(pack_tril(sym), v), sym)
    t = torch.from_numpy(sym)
    np.testing.assert_array_equal(unpack_tril(pack_tril(t), v).numpy(), sym)


def test_lno_layouts_match_reference_driver():
    """pyscfad_b200.lno.ccsd_t builds the kernel layouts of
    pyscfad/lno/ccsd_t.py:76-88 from (t1T, t2T, ..., packed ovvv)."""
    from pyscfad_b200.lno import ccsd_t as lno
    meta, _ = golden_io.load("small_o4v10_fvo")
    s = golden_io.system(meta)
    o = s.nocc
    L = lno.lno_layouts(s.t1.T, s.t2.transpose(2, 3, 1, 0), s.mo_energy, s.fock[o:, :o], s.ovoo, s.ovov,
                        pack_tril(s.ovvv), device="cpu")
    Lr = synth.reference_layouts(s)
    for k in golden_io.KEYS:
        assert L[k].is_contiguous(), k
        np.testing.assert_allclose(L[k].numpy(), Lr[k], rtol=0, atol=0, err_msg=k)


def test_lno_gradient_transforms():
    from pyscfad_b200.lno import ccsd_t as lno
    o, v = 3, 5
    g = np.random.default_rng(6)
    G = {"vooo": g.standard_normal((v, o, o, o)), "vvop": g.standard_normal((v, v, o, o + v))}
    ovoo, ovov, ovvv = lno.lno_grads_to_pyscf({k: torch.from_numpy(x) for k, x in G.items()}, o, v, packed=True)
    full = {"t1T": np.zeros((v, o)), "t2T": np.zeros((v, v, o, o)), "fvo": np.zeros((v, o)),
            "mo_energy": np.zeros(o + v), **G}
    exp = ref.to_pyscf_grads(full, o, v)
    np.testing.assert_allclose(ovoo.numpy(), exp["ovoo"], rtol=0, atol=1e-15)
    np.testing.assert_allclose(ovov.numpy(), exp["ovov"], rtol=0, atol=1e-15)
    np.testing.assert_allclose(ovvv.numpy(), exp["ovvv"], rtol=0, atol=1e-15)
