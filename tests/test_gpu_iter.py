"""GPU: the iterative (T) solver on 6-D amplitudes (pyscfad/cc/ccsd_t_slow.py:
128-293; pyscfad_b200/cc/ccsd_t_iter.py) against the numpy restatement
(oracle/ccsd_t_iter_np.py, pinned on CPU to the compiled reference's E(T)).

Tolerances (float64 throughout): the seed arrays within 1e-12 of their largest
element; energies within 1e-11 relative; converged amplitudes within 1e-9 of
their largest element (the solvers stop at |t3_new - t3| < 1e-11).
"""
from types import SimpleNamespace

import numpy as np
import pytest
import torch

import golden_io
from oracle import ccsd_t_iter_np as it
from pyscfad_b200 import synth, triples
from pyscfad_b200.cc import ccsd_t_iter
from test_oracle import _perturbed_fock

pytestmark = pytest.mark.gpu


def _layouts(s, dev):
    return {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in synth.reference_layouts(s).items()}


@pytest.mark.parametrize("name", ["tiny_o3v7", "small_o4v10_fvo", "mid_o6v17_fvo"])
def test_t3_seed_matches_oracle(name, cuda_dev):
    """ct_t3_init: P6(w + v) / d3 and r3_6d(P6(w)) / 3 at every (i,j,k,a,b,c)."""
    meta, _ = golden_io.load(name)
    s = golden_io.system(meta)
    t3c, t3x = ccsd_t_iter.t3_seed(_layouts(s, cuda_dev))
    w6 = it.P6(it.get_w_6d(s.ovvv, s.ovoo, s.t2))
    v6 = it.P6(it.get_v_6d(s.ovov, s.t1, s.t2, s.fock))
    d3 = it._d3(s.mo_energy, s.nocc)
    want_c = ((w6 + v6) / d3).transpose(3, 4, 5, 0, 1, 2)
    want_x = (it.r3_6d(w6) / 3.0).transpose(3, 4, 5, 0, 1, 2)
    got_c, got_x = t3c.cpu().numpy(), t3x.cpu().numpy()
    assert np.abs(got_c - want_c).max() <= 1e-12 * np.abs(want_c).max()
    assert np.abs(got_x - want_x).max() <= 1e-12 * np.abs(want_x).max()


@pytest.mark.parametrize("name", ["small_o4v10_fvo", "cfg1_o8v40_fvo"])
def test_iterative_canonical_is_e_t(name, cuda_dev):
    """Canonical orbitals: converged after one cycle at E(T) of ct_energy."""
    meta, _ = golden_io.load(name)
    s = golden_io.system(meta)
    e_t = triples.energy(_layouts(s, cuda_dev)).item()
    conv, e, t3 = ccsd_t_iter.iterative_kernel(SimpleNamespace(t1=s.t1, t2=s.t2), s)
    assert conv
    assert abs(e - e_t) <= 1e-11 * abs(e_t), (e, e_t)
    assert t3.shape == (s.nocc,) * 3 + (s.nvir,) * 3


@pytest.mark.parametrize("name,scale", [("small_o4v10_fvo", 0.05), ("mid_o6v17_fvo", 0.03)])
def test_iterative_noncanonical_matches_oracle(name, scale, cuda_dev):
    """Off-diagonal Fock blocks: the same cycle count, energy and amplitudes as
    the numpy solver."""
    meta, _ = golden_io.load(name)
    s = _perturbed_fock(golden_io.system(meta), scale, 7)
    conv_r, e_r, t3_r, hist = it.iterative_kernel(s.t1, s.t2, s.mo_energy, s.fock, s.ovov, s.ovoo, s.ovvv,
                                                  tol=1e-12, tolnormt=1e-11)
    conv, e, t3 = ccsd_t_iter.iterative_kernel(SimpleNamespace(t1=s.t1, t2=s.t2), s, tol=1e-12, tolnormt=1e-11)
    assert conv and conv_r and len(hist) > 3
    assert abs(e - e_r) <= 1e-11 * abs(e_r), (e, e_r)
    assert np.abs(t3.cpu().numpy() - t3_r).max() <= 1e-9 * np.abs(t3_r).max()
