"""GPU: the LNO-projected (T) energy (lnoccsdt_contract with a general
projector) on the float64 path against the compiled reference kernel.

Tolerances: 1e-10 relative to the reference's sum (float64 throughout; the
reference adds per-thread partials in OpenMP order); mat = I against 3/2 of
the canonical energy of the same kernel path, 1e-12 relative.

The TF32 / BF16x3 LNO energies are checked against the float64 LNO energy
with the canonical mixed path's energy tolerances (TF32 5e-5, BF16x3 1e-5
relative; the tests print the observed errors), and with mat = I against 3/2
of the same mode's canonical energy to 1e-6 relative (the mixed projection
reads the W and z/D cubes rounded to float).  The mixed LNO VJP: energy with
those tolerances, mat_bar and every gradient within the canonical mixed
path's gradient tolerances (TF32 2e-3, BF16x3 2e-4 of each norm) against the
float64 LNO VJP.
"""
import ctypes

import numpy as np
import pytest
import torch

import golden_io
from oracle import ccsd_t_np as onp
from oracle import ref
from pyscfad_b200 import native, synth, triples

pytestmark = pytest.mark.gpu


def dev_layouts(L, dev):
    return {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in L.items()}


def _expected(Lh, mat, a0, a1):
    """The compiled reference when oracle/_ref is built, else the numpy
    restatement (pinned to it by the CPU tests)."""
    if ref.available():
        return ref.lno_contract(mat, **Lh, a0=a0, a1=a1)
    return onp.lno_energy(Lh, mat, a0, a1)


def _vjp_expected(Lh, mat, eb, block=None):
    """(mat_bar, grads) of lnoccsdt_energy_vjp over every LNO job or one slab
    block: compiled reference, else the numpy restatement."""
    if ref.available():
        if block is None:
            return ref.lno_energy_vjp(mat, **Lh, et_bar=eb)
        b0, b1, c0, c1 = block
        return ref.lno_energy_vjp_block(mat, **Lh, et_bar=eb, b0=b0, b1=b1, c0=c0, c1=c1)
    _, mb, g = onp.lno_energy_vjp(Lh, mat, eb, block=block)
    return mb, g


@pytest.mark.parametrize("name", ["tiny_o3v7", "edge_o2v3", "small_o4v10_fvo", "mid_o6v17_fvo", "cfg1_o8v40"])
def test_lno_energy_vs_reference(name, cuda_dev):
    meta, _ = golden_io.load(name)
    Lh = synth.reference_layouts(golden_io.system(meta))
    L = dev_layouts(Lh, cuda_dev)
    o, v = meta["nocc"], meta["nvir"]
    mat = np.random.default_rng(11).standard_normal((o, o))
    md = torch.from_numpy(mat).to(cuda_dev)
    for a0, a1 in [(0, v), (0, 1), (v // 3, v // 2 + 1), (v - 1, v)]:
        e = triples.lno_energy(L, md, a0, a1).item()
        er = _expected(Lh, mat, a0, a1)
        assert abs(e - er) <= 1e-10 * abs(er), (a0, a1, e, er)


def test_lno_identity_is_three_halves_of_canonical(cuda_dev):
    meta, _ = golden_io.load("cfg1_o8v40_fvo")
    L = dev_layouts(synth.reference_layouts(golden_io.system(meta)), cuda_dev)
    o = meta["nocc"]
    e_lno = triples.lno_energy(L, torch.eye(o, dtype=torch.float64, device=cuda_dev)).item()
    e_can = triples.energy(L).item()
    assert abs(e_lno - 1.5 * e_can) <= 1e-12 * abs(e_can)


def test_lno_slab_block_larger_system(cuda_dev):
    """nocc=16 / nvir=120, a projector of rank 8 (a local-orbital-like
    ulo^T ulo), one a-slab, job energies summing to the slab energy, and two
    calls bitwise equal."""
    meta, _ = golden_io.load("cfg2_o16v120")
    Lh = synth.reference_layouts(golden_io.system(meta))
    L = dev_layouts(Lh, cuda_dev)
    o, v = meta["nocc"], meta["nvir"]
    u = np.linalg.qr(np.random.default_rng(12).standard_normal((o, o)))[0][:8]
    mat = u.T @ u
    md = torch.from_numpy(mat).to(cuda_dev)
    a0, a1 = 110, 112
    je = torch.zeros(v * (v + 1) * (v + 2) // 6, dtype=torch.float64, device=cuda_dev)
    e = triples.lno_energy(L, md, a0, a1, job_e=je).item()
    er = _expected(Lh, mat, a0, a1)
    assert abs(e - er) <= 1e-10 * abs(er), (e, er)
    assert abs(float(je.sum()) - e) <= 1e-12 * abs(e)
    assert triples.lno_energy(L, md, a0, a1).item() == e


def test_lno_host_pointer_entry_accumulates(cuda_dev):
    meta, _ = golden_io.load("small_o4v10_fvo")
    Lh = synth.reference_layouts(golden_io.system(meta))
    o, v = meta["nocc"], meta["nvir"]
    mat = np.random.default_rng(13).standard_normal((o, o))
    arrs = {k: np.ascontiguousarray(x, dtype=np.float64) for k, x in Lh.items()}
    e = np.array([0.25])
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    native.check(native.lib().ctb_lnoccsdt_contract(
        p(e), p(mat), p(arrs["mo_energy"]), p(arrs["t1T"]), p(arrs["t2T"]), p(arrs["vooo"]), p(arrs["fvo"]),
        o, v, 2, 7, p(arrs["vvop"])))
    er = _expected(Lh, mat, 2, 7)
    assert abs(e[0] - 0.25 - er) <= 1e-10 * abs(er)


def test_lno_rejects_bad_arguments(cuda_dev):
    meta, _ = golden_io.load("small_o4v10_fvo")
    L = dev_layouts(synth.reference_layouts(golden_io.system(meta)), cuda_dev)
    o, v = meta["nocc"], meta["nvir"]
    md = torch.eye(o, dtype=torch.float64, device=cuda_dev)
    with pytest.raises(native.CtError):
        triples.lno_energy(L, md, 3, 3)
    with pytest.raises(native.CtError):
        triples.lno_energy(L, md, 0, v + 1)
    prob = native.CtProblem(o, v, *[ctypes.c_void_p(L[k].data_ptr()) for k in golden_io.KEYS])
    out = torch.zeros((), dtype=torch.float64, device=cuda_dev)
    st = native.lib().ct_lno_energy(ctypes.byref(prob), None, 0, v, ctypes.c_void_p(out.data_ptr()), None, None)
    assert st != 0


@pytest.mark.parametrize("name", ["tiny_o3v7", "edge_o2v3", "small_o4v10_fvo", "mid_o6v17_fvo", "cfg1_o8v40_fvo"])
def test_lno_vjp_vs_reference(name, cuda_dev):
    """ct_lno_energy_vjp against the compiled lnoccsdt_energy_vjp over every
    LNO job: mat_bar and every gradient within 1e-10 of each norm."""
    meta, _ = golden_io.load(name)
    Lh = synth.reference_layouts(golden_io.system(meta))
    L = dev_layouts(Lh, cuda_dev)
    o = meta["nocc"]
    mat = np.random.default_rng(17).standard_normal((o, o))
    eb = 0.7
    e, mb, g = triples.lno_energy_vjp(L, torch.from_numpy(mat).to(cuda_dev), eb)
    torch.cuda.synchronize()
    mb_r, g_r = _vjp_expected(Lh, mat, eb)
    er = _expected(Lh, mat, 0, meta["nvir"])
    assert abs(e.item() - er) <= 1e-10 * abs(er)
    assert np.linalg.norm(mb.cpu().numpy() - mb_r) <= 1e-10 * np.linalg.norm(mb_r)
    for k in golden_io.KEYS:
        nrm = np.linalg.norm(g_r[k])
        assert np.linalg.norm(g[k].cpu().numpy() - g_r[k]) <= 1e-10 * nrm + 1e-300, (k, nrm)


def test_lno_vjp_identity_is_three_halves_of_canonical(cuda_dev):
    """mat = I: the LNO sum is 3/2 E(T), so its gradients are 3/2 of the
    canonical VJP's (whose et_bar is twice the cotangent).  Repeated calls give
    a bitwise-equal mat_bar (fixed-order sums); the other gradients take float64
    atomics on this path, so they agree to round-off."""
    meta, _ = golden_io.load("mid_o6v17_fvo")
    L = dev_layouts(synth.reference_layouts(golden_io.system(meta)), cuda_dev)
    o = meta["nocc"]
    eye = torch.eye(o, dtype=torch.float64, device=cuda_dev)
    _, mb1, g1 = triples.lno_energy_vjp(L, eye, 0.4)
    _, g0 = triples.energy_vjp(L, 2 * 0.4)
    for k in golden_io.KEYS:
        nrm = float(torch.linalg.norm(g0[k]))
        assert float(torch.linalg.norm(g1[k] - 1.5 * g0[k])) <= 1e-12 * nrm + 1e-300, k
    _, mb2, g2 = triples.lno_energy_vjp(L, eye, 0.4)
    assert torch.equal(mb1, mb2)
    for k in golden_io.KEYS:
        assert float(torch.linalg.norm(g1[k] - g2[k])) <= 1e-14 * float(torch.linalg.norm(g1[k])) + 1e-300, k


@pytest.mark.parametrize("blk", [(7, 10, 7, 10), (7, 10, 0, 7), (3, 6, 0, 2), (2, 5, 2, 5)])
def test_lno_vjp_block_vs_reference(blk, cuda_dev):
    """One block of the LNO backward's slab loop on device data against the
    compiled kernel run on the driver's caches."""
    meta, _ = golden_io.load("small_o4v10_fvo")
    Lh = synth.reference_layouts(golden_io.system(meta))
    L = dev_layouts(Lh, cuda_dev)
    o = meta["nocc"]
    mat = np.random.default_rng(19).standard_normal((o, o))
    _, mb, g = triples.lno_energy_vjp(L, torch.from_numpy(mat).to(cuda_dev), 0.3, block=blk)
    mb_r, g_r = _vjp_expected(Lh, mat, 0.3, blk)
    assert np.linalg.norm(mb.cpu().numpy() - mb_r) <= 1e-10 * np.linalg.norm(mb_r)
    for k in golden_io.KEYS:
        nrm = np.linalg.norm(g_r[k])
        assert np.linalg.norm(g[k].cpu().numpy() - g_r[k]) <= 1e-10 * nrm + 1e-300, k


def _prange(start, stop, step):
    return [(i, min(i + step, stop)) for i in range(start, stop, step)]


def test_lno_vjp_host_dropin_in_the_reference_slab_loop(cuda_dev):
    """The LNO backward's slab loop (pyscfad/lno/ccsd_t.py:193-220) with
    ctb_lnoccsdt_energy_vjp in place of lnoccsdt_energy_vjp, small slabs so
    diagonal and off-diagonal blocks both occur, against the compiled kernel
    over every LNO job."""
    meta, _ = golden_io.load("mid_o6v17_fvo")
    Lh = synth.reference_layouts(golden_io.system(meta))
    o, v = meta["nocc"], meta["nvir"]
    mat = np.random.default_rng(23).standard_normal((o, o))
    eb = 0.45
    arr = {k: np.ascontiguousarray(x, dtype=np.float64) for k, x in Lh.items()}
    vvop = arr["vvop"]
    bars = {k: np.zeros_like(arr[k]) for k in ("mo_energy", "t1T", "t2T", "vooo", "fvo")}
    mat_bar = np.zeros_like(mat)
    vvop_bar = np.zeros_like(vvop)
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)

    def contract(b0, b1, c0, c1, cache, cache_bar):
        native.check(native.lib().ctb_lnoccsdt_energy_vjp(
            p(mat), p(arr["mo_energy"]), p(arr["t1T"]), p(arr["t2T"]), p(arr["vooo"]), p(arr["fvo"]), eb,
            o, v, b0, b1, c0, c1, *[p(c) for c in cache], p(mat_bar), p(bars["mo_energy"]), p(bars["t1T"]),
            p(bars["t2T"]), p(bars["vooo"]), p(bars["fvo"]), *[p(c) for c in cache_bar]))

    bufsize = 8
    for a0, a1 in reversed(_prange(0, v, bufsize)):
        row_a = np.ascontiguousarray(vvop[a0:a1, :])
        row_a_bar = np.zeros_like(row_a)
        if (a0, a1) == (0, v):
            col_a, col_a_bar = row_a, row_a_bar
        else:
            col_a = np.ascontiguousarray(vvop[:, a0:a1])
            col_a_bar = np.zeros_like(col_a)
        contract(a0, a1, a0, a1, (row_a, col_a, row_a, col_a), (row_a_bar, col_a_bar, row_a_bar, col_a_bar))
        for b0, b1 in _prange(0, a0, bufsize // 4):
            row_b = np.ascontiguousarray(vvop[b0:b1, :])
            row_b_bar = np.zeros_like(row_b)
            col_b = np.ascontiguousarray(vvop[:, b0:b1])
            col_b_bar = np.zeros_like(col_b)
            contract(a0, a1, b0, b1, (row_a, col_a, row_b, col_b), (row_a_bar, col_a_bar, row_b_bar, col_b_bar))
            vvop_bar[b0:b1, :] += row_b_bar
            vvop_bar[:, b0:b1] += col_b_bar
        vvop_bar[a0:a1, :] += row_a_bar
        if (a0, a1) != (0, v):
            vvop_bar[:, a0:a1] += col_a_bar
    mb_r, g_r = _vjp_expected(Lh, mat, eb)
    assert np.linalg.norm(mat_bar - mb_r) <= 1e-10 * np.linalg.norm(mb_r)
    bars["vvop"] = vvop_bar
    for k in golden_io.KEYS:
        nrm = np.linalg.norm(g_r[k])
        assert np.linalg.norm(bars[k] - g_r[k]) <= 1e-10 * nrm + 1e-300, k


def test_lno_wrapper_energy_and_custom_vjp(cuda_dev):
    """pyscfad_b200.lno.ccsd_t: _ccsd_t_energy (x 2/3) on numpy and torch
    inputs with packed ovvv, its backward against the compiled kernel with the
    driver's 2/3 on the cotangent and its output transforms, and kernel()
    with a differentiable ulo (mat = ulo^T ulo)."""
    from pyscfad_b200.cc.eris import pack_tril
    from pyscfad_b200.lno import ccsd_t as lno
    meta, _ = golden_io.load("small_o4v10_fvo")
    s = golden_io.system(meta)
    Lh = synth.reference_layouts(s)
    o, v = s.nocc, s.nvir
    ulo = np.random.default_rng(29).standard_normal((3, o))
    mat = ulo.T @ ulo
    args = [mat, s.t1.T.copy(), s.t2.transpose(2, 3, 1, 0).copy(), s.mo_energy, s.fock[o:, :o].copy(), s.ovoo,
            s.ovov, pack_tril(s.ovvv)]
    e_ref = _expected(Lh, mat, 0, v) * 2.0 / 3.0
    assert abs(lno._ccsd_t_energy(*args) - e_ref) <= 1e-10 * abs(e_ref)
    targs = [torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device=cuda_dev, requires_grad=True)
             for a in args]
    e = lno._ccsd_t_energy(*targs)
    assert abs(e.item() - e_ref) <= 1e-10 * abs(e_ref)
    e.backward()
    mb_r, g_r = _vjp_expected(Lh, mat, 2.0 / 3.0)
    full = dict(g_r)
    exp = ref.to_pyscf_grads(full, o, v)
    want = [mb_r, g_r["t1T"], g_r["t2T"], g_r["mo_energy"], g_r["fvo"], exp["ovoo"], exp["ovov"], exp["ovvv"]]
    for t, w in zip(targs, want):
        assert np.linalg.norm(t.grad.cpu().numpy() - w) <= 1e-10 * np.linalg.norm(w) + 1e-300
    # kernel(): gradient through mat = ulo^T ulo
    from types import SimpleNamespace
    from pyscfad_b200.cc import ERIs
    u = torch.tensor(ulo, dtype=torch.float64, device=cuda_dev, requires_grad=True)
    eris = ERIs.from_system(s, packed=True)
    ek = lno.kernel(SimpleNamespace(t1=torch.from_numpy(s.t1).to(cuda_dev), t2=torch.from_numpy(s.t2).to(cuda_dev),
                                    max_memory=4000), eris, u)
    assert abs(ek.item() - e_ref) <= 1e-10 * abs(e_ref)
    ek.backward()
    gu = ulo @ (mb_r + mb_r.T)
    assert np.linalg.norm(u.grad.cpu().numpy() - gu) <= 1e-10 * np.linalg.norm(gu)


MIXED_TOL = {"tf32": 5e-5, "bf16x3": 1e-5}


def _projector(o, rank, seed):
    u = np.linalg.qr(np.random.default_rng(seed).standard_normal((o, o)))[0][:rank]
    return u.T @ u


def _mixed_system(name):
    """golden systems by name; "o40v24" a synthetic nocc=40 one (the 8-tile
    projection build, nocc > 32)"""
    if name == "o40v24":
        return synth.reference_layouts(synth.make_system(40, 24, 96, 41, fvo_sigma=1e-2))
    meta, _ = golden_io.load(name)
    return synth.reference_layouts(golden_io.system(meta))


@pytest.mark.parametrize("mode", ["tf32", "bf16x3"])
@pytest.mark.parametrize("name", ["cfg1_o8v40_fvo", "cfg2_o16v120", "o40v24"])
def test_lno_energy_mixed_vs_fp64(mode, name, cuda_dev):
    """ct_lno_energy_mode: the mixed-precision LNO energy against the float64
    LNO energy for a rank-nocc/2 projector, full range and one a-slab, job
    energies summing to the slab energy, and two calls bitwise equal."""
    L = dev_layouts(_mixed_system(name), cuda_dev)
    o, v = L["t1T"].shape[1], L["t1T"].shape[0]
    md = torch.from_numpy(_projector(o, o // 2, 17)).to(cuda_dev)
    for a0, a1 in [(0, v), (v // 3, v // 2 + 1)]:
        e64 = triples.lno_energy(L, md, a0, a1).item()
        je = torch.zeros(v * (v + 1) * (v + 2) // 6, dtype=torch.float64, device=cuda_dev)
        em = triples.lno_energy(L, md, a0, a1, job_e=je, mode=mode).item()
        rel = abs(em - e64) / abs(e64)
        print(f"\n{name} {mode} slab ({a0}, {a1}): LNO energy rel {rel:.2e}")
        assert rel < MIXED_TOL[mode], (a0, a1, em, e64)
        assert abs(float(je.sum()) - em) <= 1e-12 * abs(em)
        assert triples.lno_energy(L, md, a0, a1, mode=mode).item() == em


@pytest.mark.parametrize("mode", ["tf32", "bf16x3"])
def test_lno_mixed_identity_is_three_halves_of_canonical(mode, cuda_dev):
    L = dev_layouts(_mixed_system("cfg2_o16v120"), cuda_dev)
    o = L["t1T"].shape[1]
    e_lno = triples.lno_energy(L, torch.eye(o, dtype=torch.float64, device=cuda_dev), mode=mode).item()
    e_can = triples.energy(L, mode=mode).item()
    assert abs(e_lno - 1.5 * e_can) <= 1e-6 * abs(e_can), (e_lno, 1.5 * e_can)


def test_lno_mixed_rejects_unaligned_nocc(cuda_dev):
    """The mixed modes need nocc % 8 == 0 (the qr-tiled slots); nocc = 4 is refused."""
    meta, _ = golden_io.load("small_o4v10_fvo")
    L = dev_layouts(synth.reference_layouts(golden_io.system(meta)), cuda_dev)
    md = torch.eye(meta["nocc"], dtype=torch.float64, device=cuda_dev)
    with pytest.raises(native.CtError):
        triples.lno_energy(L, md, mode="tf32")


MIXED_GRAD_TOL = {"tf32": 2e-3, "bf16x3": 2e-4}


@pytest.mark.parametrize("mode", ["tf32", "bf16x3"])
@pytest.mark.parametrize("name,blk", [("cfg1_o8v40_fvo", None), ("cfg2_o16v120", None), ("o40v24", None),
                                      ("cfg2_o16v120", (60, 90, 0, 40)), ("cfg2_o16v120", (60, 90, 60, 90))])
def test_lno_vjp_mixed_vs_fp64(mode, name, blk, cuda_dev):
    """ct_lno_energy_vjp_mode against the float64 LNO VJP (every LNO job, or
    one slab block): energy, mat_bar and the six gradients."""
    L = dev_layouts(_mixed_system(name), cuda_dev)
    o = L["t1T"].shape[1]
    md = torch.from_numpy(_projector(o, o // 2, 23)).to(cuda_dev)
    e64, mb64, g64 = triples.lno_energy_vjp(L, md, 0.6, block=blk)
    em, mbm, gm = triples.lno_energy_vjp(L, md, 0.6, block=blk, mode=mode)
    torch.cuda.synchronize()
    rel_e = abs(em.item() - e64.item()) / abs(e64.item())
    rel = {k: float(torch.linalg.norm(gm[k] - g64[k])) / max(float(torch.linalg.norm(g64[k])), 1e-300)
           for k in golden_io.KEYS}
    rel["mat_bar"] = float(torch.linalg.norm(mbm - mb64)) / float(torch.linalg.norm(mb64))
    print(f"\n{name} {blk} {mode}: LNO VJP energy rel {rel_e:.2e}; " + " ".join(f"{k}={x:.1e}" for k, x in rel.items()))
    assert rel_e < MIXED_TOL[mode], (em.item(), e64.item())
    for k, x in rel.items():
        assert x <= MIXED_GRAD_TOL[mode], (k, x)


@pytest.mark.parametrize("mode", ["tf32", "bf16x3"])
def test_lno_vjp_mixed_identity_is_three_halves_of_canonical(mode, cuda_dev):
    """mat = I in the same mixed mode: 3/2 of the canonical mixed VJP's
    gradients (whose et_bar is twice the cotangent).  The two paths round
    different intermediates to float (the canonical one forms W-bar in float
    arithmetic, the LNO one from float A, B and z/D cubes in float64) before
    the same tensor-core bar GEMMs, so they agree to 1e-4 of each norm; mat_bar
    is bitwise repeatable."""
    L = dev_layouts(_mixed_system("cfg2_o16v120"), cuda_dev)
    o = L["t1T"].shape[1]
    eye = torch.eye(o, dtype=torch.float64, device=cuda_dev)
    _, mb1, g1 = triples.lno_energy_vjp(L, eye, 0.4, mode=mode)
    _, g0 = triples.energy_vjp(L, 2 * 0.4, mode=mode)
    errs = {k: float(torch.linalg.norm(g1[k] - 1.5 * g0[k])) / float(torch.linalg.norm(g0[k]))
            for k in golden_io.KEYS}
    print(f"\n{mode} LNO(mat=I) vs 3/2 canonical: " + " ".join(f"{k}={x:.1e}" for k, x in errs.items()))
    for k, x in errs.items():
        assert x <= 1e-4, (k, x)
    _, mb2, _ = triples.lno_energy_vjp(L, eye, 0.4, mode=mode)
    assert torch.equal(mb1, mb2)


def test_lno_wrapper_mixed_mode(cuda_dev):
    """pyscfad_b200.lno.ccsd_t._ccsd_t_energy(..., mode="tf32") with packed
    ovvv: energy and all eight gradients (backward through the mixed LNO VJP)
    against the float64 wrapper, within the mixed tolerances."""
    from pyscfad_b200.cc.eris import pack_tril
    from pyscfad_b200.lno import ccsd_t as lno
    meta, _ = golden_io.load("cfg2_o16v120")
    s = golden_io.system(meta)
    o = s.nocc
    args = [_projector(o, 8, 31), s.t1.T.copy(), s.t2.transpose(2, 3, 1, 0).copy(), s.mo_energy,
            s.fock[o:, :o].copy(), s.ovoo, s.ovov, pack_tril(s.ovvv)]
    res = {}
    for mode in ("fp64", "tf32"):
        targs = [torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device=cuda_dev, requires_grad=True)
                 for a in args]
        e = lno._ccsd_t_energy(*targs, mode=mode)
        e.backward()
        res[mode] = (e.item(), [t.grad.detach().clone() for t in targs])
    (e64, g64), (em, gm) = res["fp64"], res["tf32"]
    assert abs(em - e64) <= MIXED_TOL["tf32"] * abs(e64), (em, e64)
    for i, (a, b) in enumerate(zip(gm, g64)):
        assert float(torch.linalg.norm(a - b)) <= MIXED_GRAD_TOL["tf32"] * float(torch.linalg.norm(b)) + 1e-300, i
