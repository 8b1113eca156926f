"""GPU parity of the FP64 path against the reference's own kernels (golden
fixtures from oracle/_ref), the numpy oracle, and central finite differences.

Tolerances: energies |dE| <= max(1e-10 Eh, 1e-12 |E|) (the FP64 gate);
gradients 1e-8 relative to each gradient's norm against the reference VJP;
finite differences (h = 1e-5, 32 random joint directions) 1e-6 relative, the
truncation/rounding floor of a central difference at |E| ~ 3e4 Eh.
"""
import ctypes

import numpy as np
import pytest
import torch

import golden_io
from oracle import ccsd_t_np as onp
from oracle import ref
from pyscfad_b200 import native, synth, triples
from pyscfad_b200.cc import ERIs
from pyscfad_b200.cc import ccsd_t as cct

pytestmark = pytest.mark.gpu


def dev_layouts(L, dev):
    return {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in L.items()}


def e_tol(e):
    return max(1e-10, 1e-12 * abs(e))


@pytest.mark.parametrize("name", golden_io.names())
def test_fp64_energy_matches_reference(name, cuda_dev):
    meta, _ = golden_io.load(name)
    L = synth.reference_layouts(golden_io.system(meta))
    np.testing.assert_allclose(golden_io.checksum(L), meta["checksum"], rtol=1e-12, atol=1e-12)
    e = triples.energy(dev_layouts(L, cuda_dev)).item()
    assert abs(e - meta["e_t"]) <= e_tol(meta["e_t"]), (e, meta["e_t"])


@pytest.mark.parametrize("name", golden_io.names())
def test_fp64_vjp_matches_reference(name, cuda_dev):
    meta, arr = golden_io.load(name)
    L = synth.reference_layouts(golden_io.system(meta))
    e, g = triples.energy_vjp(dev_layouts(L, cuda_dev), 2.0)  # kernel et_bar = 2 x cotangent 1
    assert abs(e.item() - meta["e_t"]) <= e_tol(meta["e_t"])
    for k in golden_io.KEYS:
        gk = g[k].cpu().numpy()
        nrm = float(arr[f"norm_{k}"])
        if f"grad_{k}" in arr:
            assert np.abs(gk - arr[f"grad_{k}"]).max() <= 1e-8 * max(nrm, 1e-300) + 1e-15, k
        proj = np.array([np.vdot(gk, golden_io.direction(k, gk.shape, meta["seed"], i))
                         for i in range(meta["ndir"])])
        scale = nrm * np.sqrt(gk.size)
        assert np.abs(proj - arr[f"proj_{k}"]).max() <= 1e-8 * max(scale, 1e-300) + 1e-15, k
        assert abs(np.linalg.norm(gk) - nrm) <= 1e-8 * max(nrm, 1e-300) + 1e-15, k


def test_fp64_vjp_central_differences(cuda_dev):
    """cfg2 (o16 v120 naux400 seed1): 32 random joint directions, h = 1e-5."""
    meta, _ = golden_io.load("cfg2_o16v120")
    L = dev_layouts(synth.reference_layouts(golden_io.system(meta)), cuda_dev)
    _, g = triples.energy_vjp(L, 2.0)
    gen = torch.Generator(device="cpu").manual_seed(2024)
    scales = {k: max(float(L[k].std()), 1e-3) if L[k].numel() > 1 else 1.0 for k in golden_io.KEYS}
    h = 1e-5
    rel = []
    for _ in range(32):
        u = {k: (torch.randn(L[k].shape, generator=gen, dtype=torch.float64) * scales[k]).to(cuda_dev)
             for k in golden_io.KEYS}
        lp = {k: (L[k] + h * u[k]).contiguous() for k in golden_io.KEYS}
        lm = {k: (L[k] - h * u[k]).contiguous() for k in golden_io.KEYS}
        fd = (triples.energy(lp).item() - triples.energy(lm).item()) / (2 * h)
        an = sum(float((g[k] * u[k]).sum()) for k in golden_io.KEYS)
        rel.append(abs(fd - an) / max(abs(an), 1e-12))
    assert max(rel) < 1e-6, max(rel)


def test_job_energies_match_oracle(cuda_dev):
    meta, _ = golden_io.load("small_o4v10_fvo")
    L = synth.reference_layouts(golden_io.system(meta))
    v = meta["nvir"]
    je = torch.zeros(v * (v + 1) * (v + 2) // 6, dtype=torch.float64, device=cuda_dev)
    e = triples.energy(dev_layouts(L, cuda_dev), job_e=je).item()
    ref_je = onp.job_energies(L, onp.sorted_jobs(v))
    np.testing.assert_allclose(je.cpu().numpy(), ref_je, rtol=1e-11, atol=1e-16)
    assert abs(je.sum().item() - e) < 1e-13


def test_energy_bitwise_repeatable(cuda_dev):
    meta, _ = golden_io.load("cfg1_o8v40")
    L = dev_layouts(synth.reference_layouts(golden_io.system(meta)), cuda_dev)
    e1 = triples.energy(L).item()
    e2 = triples.energy(L).item()
    assert e1 == e2


def _lib_call(*args):
    conv = []
    for i, a in enumerate(args):
        if isinstance(a, np.ndarray):
            assert a.dtype == np.float64 and a.flags.c_contiguous
            conv.append(a.ctypes.data_as(ctypes.c_void_p))
        elif i == 5:
            conv.append(ctypes.c_double(a))
        else:
            conv.append(ctypes.c_int(a))
    native.check(native.lib().ctb_ccsd_t_energy_vjp(*conv), "ctb_ccsd_t_energy_vjp")


@pytest.mark.parametrize("na,nb", [(1, 1), (3, 2), (4, 3)])
def test_host_entry_through_reference_driver_loop(na, nb, cuda_dev):
    """The host-pointer drop-in, driven by the reference's slab loop
    (pyscfad/cc/ccsd_t.py:145-177), reproduces the reference VJP."""
    meta, arr = golden_io.load("small_o4v10_fvo")
    L = synth.reference_layouts(golden_io.system(meta))
    g = ref.blocked_vjp(_lib_call, L, 2.0, na, nb)
    for k in golden_io.KEYS:
        nrm = float(arr[f"norm_{k}"])
        assert np.abs(g[k] - arr[f"grad_{k}"]).max() <= 1e-9 * nrm + 1e-15, k


@pytest.mark.parametrize("na,nb", [(3, 2), (4, 3)])
def test_host_entry_in_many_stages(na, nb, cuda_dev, monkeypatch):
    """The host-pointer entry runs a block in stages of the jobs' smallest
    index (one wave each, its copies in and gradients out overlapping the
    neighbouring stages); with waves of 3 jobs every smallest index is a stage
    of its own, and the reference's slab loop still reproduces the reference
    VJP."""
    meta, arr = golden_io.load("small_o4v10_fvo")
    L = synth.reference_layouts(golden_io.system(meta))
    native.lib().ct_release_workspace()
    monkeypatch.setenv("CTB_MAX_WAVE", "3")
    try:
        g = ref.blocked_vjp(_lib_call, L, 2.0, na, nb)
    finally:
        monkeypatch.delenv("CTB_MAX_WAVE")
        native.lib().ct_release_workspace()
    for k in golden_io.KEYS:
        nrm = float(arr[f"norm_{k}"])
        assert np.abs(g[k] - arr[f"grad_{k}"]).max() <= 1e-9 * nrm + 1e-15, k


def test_host_energy_entry_slabs(cuda_dev):
    meta, _ = golden_io.load("mid_o6v17_fvo")
    L = synth.reference_layouts(golden_io.system(meta))
    args = [np.ascontiguousarray(L[k]) for k in ("mo_energy", "t1T", "t2T", "vooo", "fvo")]
    vvop = np.ascontiguousarray(L["vvop"])
    tot = np.zeros(1)
    for a0, a1 in [(0, 5), (5, 11), (11, 17)]:
        st = native.lib().ctb_ccsd_t_energy(tot.ctypes.data_as(ctypes.c_void_p),
                                            *[x.ctypes.data_as(ctypes.c_void_p) for x in args],
                                            meta["nocc"], meta["nvir"], a0, a1,
                                            vvop.ctypes.data_as(ctypes.c_void_p), 0)
        native.check(st)
    assert abs(tot[0] - meta["e_t"]) <= e_tol(meta["e_t"])


@pytest.mark.parametrize("packed", [True, False])
def test_pyscf_layout_autograd(packed, cuda_dev):
    """cc.ccsd_t.kernel with torch inputs: forward E and the custom backward
    equal the reference driver's (T) energy and _ccsd_t_energy_vjp outputs."""
    meta, arr = golden_io.load("small_o4v10_fvo")
    s = golden_io.system(meta)
    eris = ERIs.from_system(s, packed=packed)
    tt = lambda x: torch.from_numpy(np.ascontiguousarray(x)).to(cuda_dev).requires_grad_(True)  # noqa: E731
    t1, t2 = tt(s.t1), tt(s.t2)
    teris = ERIs(fock=tt(eris.fock), mo_energy=tt(eris.mo_energy), ovoo=tt(eris.ovoo),
                 ovov=tt(eris.ovov), ovvv=tt(eris.ovvv))
    e = cct.kernel(None, teris, t1, t2)
    assert abs(e.item() - meta["e_t"]) <= e_tol(meta["e_t"])
    e.backward()
    g = {k: arr[f"grad_{k}"] for k in golden_io.KEYS}
    want = ref.to_pyscf_grads(g, meta["nocc"], meta["nvir"])
    np.testing.assert_allclose(t1.grad.cpu().numpy(), want["t1"], rtol=1e-9, atol=1e-14)
    np.testing.assert_allclose(t2.grad.cpu().numpy(), want["t2"], rtol=1e-9, atol=1e-14)
    np.testing.assert_allclose(teris.fock.grad.cpu().numpy(), want["fock"], rtol=1e-9, atol=1e-14)
    np.testing.assert_allclose(teris.mo_energy.grad.cpu().numpy(), want["mo_energy"], rtol=1e-9, atol=1e-14)
    np.testing.assert_allclose(teris.ovoo.grad.cpu().numpy(), want["ovoo"], rtol=1e-9, atol=1e-14)
    np.testing.assert_allclose(teris.ovov.grad.cpu().numpy(), want["ovov"], rtol=1e-9, atol=1e-14)
    if packed:
        np.testing.assert_allclose(teris.ovvv.grad.cpu().numpy(), want["ovvv"], rtol=1e-9, atol=1e-14)
    else:
        raw = g["vvop"][:, :, :, meta["nocc"]:].transpose(2, 0, 3, 1)
        np.testing.assert_allclose(teris.ovvv.grad.cpu().numpy(), raw, rtol=1e-9, atol=1e-14)


def test_numpy_driver_entry(cuda_dev):
    """_ccsd_t_energy_vjp(eris, t1, t2, et_bar, max_memory) returns the
    reference driver's 7-tuple (pyscfad/cc/ccsd_t.py:179-192)."""
    meta, arr = golden_io.load("tiny_o3v7")
    s = golden_io.system(meta)
    eris = ERIs.from_system(s, packed=True)
    out = cct._ccsd_t_energy_vjp(eris, s.t1, s.t2, 0.7, 2000)
    g = {k: 0.7 * arr[f"grad_{k}"] for k in golden_io.KEYS}
    want = ref.to_pyscf_grads(g, meta["nocc"], meta["nvir"])
    for got, key in zip(out, ("t1", "t2", "fock", "mo_energy", "ovoo", "ovov", "ovvv")):
        np.testing.assert_allclose(got, want[key], rtol=1e-9, atol=1e-15)
    assert abs(cct.kernel(None, eris, s.t1, s.t2) - meta["e_t"]) <= e_tol(meta["e_t"])


def test_bad_inputs_raise(cuda_dev):
    meta, _ = golden_io.load("tiny_o3v7")
    L = dev_layouts(synth.reference_layouts(golden_io.system(meta)), cuda_dev)
    bad = dict(L)
    bad["t2T"] = L["t2T"].float()
    with pytest.raises(native.CtError):
        triples.energy(bad)
    bad = dict(L)
    bad["vvop"] = L["vvop"][:, :, :, :-1].contiguous()
    with pytest.raises(native.CtError):
        triples.energy(bad)
    with pytest.raises(native.CtError):
        triples.energy(L, mode="fp8")


def test_small_waves_match_single_wave(cuda_dev, monkeypatch):
    """Forcing many tiny waves (scratch budget of 1-3 jobs) changes nothing."""
    meta, arr = golden_io.load("mid_o6v17_fvo")
    L = dev_layouts(synth.reference_layouts(golden_io.system(meta)), cuda_dev)
    e0, g0 = triples.energy_vjp(L, 2.0)
    native.lib().ct_release_workspace()
    monkeypatch.setenv("CTB_MAX_WAVE", "3")
    try:
        e1, g1 = triples.energy_vjp(L, 2.0)
    finally:
        monkeypatch.delenv("CTB_MAX_WAVE")
        native.lib().ct_release_workspace()
    assert abs(e0.item() - e1.item()) < 1e-12
    for k in golden_io.KEYS:
        torch.testing.assert_close(g0[k], g1[k], rtol=1e-11, atol=1e-15)


def test_device_block_entries_sum_to_full(cuda_dev):
    """ct_energy_vjp_block over the reference driver's blocks, and
    ct_energy_block over a-slabs, reproduce the full energy and VJP."""
    meta, arr = golden_io.load("mid_o6v17_fvo")
    L = dev_layouts(synth.reference_layouts(golden_io.system(meta)), cuda_dev)
    o, v = meta["nocc"], meta["nvir"]
    G = {k: torch.zeros_like(L[k]) for k in golden_io.KEYS}
    prob = native.CtProblem(o, v, *[ctypes.c_void_p(L[k].data_ptr()) for k in golden_io.KEYS])
    gr = native.CtGrads(*[ctypes.c_void_p(G[k].data_ptr()) for k in golden_io.KEYS])
    e = torch.zeros((), dtype=torch.float64, device=cuda_dev)
    etot = 0.0
    for a0, a1 in reversed(ref.slabs(0, v, 3)):
        blocks = [(a0, a1, a0, a1)] + [(a0, a1, b0, b1) for b0, b1 in ref.slabs(0, a0, 2)]
        for blk in blocks:
            native.check(native.lib().ct_energy_vjp_block(ctypes.byref(prob), 0, 2.0, ctypes.byref(gr), *blk,
                                                          ctypes.c_void_p(e.data_ptr()), None))
            torch.cuda.synchronize()
            etot += e.item()
    assert abs(etot - meta["e_t"]) <= e_tol(meta["e_t"])
    for k in golden_io.KEYS:
        gk = G[k].cpu().numpy()
        proj = np.array([np.vdot(gk, golden_io.direction(k, gk.shape, meta["seed"], i))
                         for i in range(meta["ndir"])])
        scale = float(arr[f"norm_{k}"]) * np.sqrt(gk.size)
        assert np.abs(proj - arr[f"proj_{k}"]).max() <= 1e-8 * scale + 1e-15, k
    es = 0.0
    for a0, a1 in [(0, 6), (6, 13), (13, 17)]:
        native.check(native.lib().ct_energy_block(ctypes.byref(prob), 0, a0, a1, ctypes.c_void_p(e.data_ptr()),
                                                  None, None))
        torch.cuda.synchronize()
        es += e.item()
    assert abs(es - meta["e_t"]) <= e_tol(meta["e_t"])
    with pytest.raises(native.CtError):
        native.check(native.lib().ct_energy_vjp_block(ctypes.byref(prob), 0, 2.0, ctypes.byref(gr), 3, 9, 2, 8,
                                                      None, None))


def test_peak_probes(cuda_dev):
    for kind in (0, 1):
        t = ctypes.c_double(0)
        native.check(native.lib().ct_peak_probe(kind, ctypes.byref(t)))
        assert 5.0 < t.value < 200.0
