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
