"""GPU: the mixed-precision (tcgen05) path against the FP64 path and the
reference's golden values.

Tolerances, stated per precision (energies relative to |E|, gradients relative
to each gradient's norm): TF32 (10-bit mantissa products, float32 accumulate)
5e-5 energy / 2e-3 gradient; BF16x3 (hi/lo bf16 split products, about 16
mantissa bits, float32 accumulate) 1e-5 energy / 2e-4 gradient.  They sit 3-10x
above the largest errors observed on these systems (TF32: energy 5.4e-6,
gradients 2.5e-4; BF16x3: energy 7.3e-7, gradients 6.3e-5); the tests print
the observed values.  The absolute 1e-6 Eh mixed gate is reported, not
asserted, at these generator scales (|E| >> 1 Eh).
"""
import ctypes

import numpy as np
import pytest
import torch

import golden_io
from pyscfad_b200 import native, synth, triples

pytestmark = pytest.mark.gpu

TOL = {"tf32": (5e-5, 2e-3), "bf16x3": (1e-5, 2e-4)}
MODES = ["tf32", "bf16x3"]


def dev_layouts(L, dev):
    return {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in L.items()}


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("name", ["cfg1_o8v40", "cfg1_o8v40_fvo", "cfg2_o16v120"])
def test_mixed_energy_vs_reference(mode, name, cuda_dev):
    meta, _ = golden_io.load(name)
    L = dev_layouts(synth.reference_layouts(golden_io.system(meta)), cuda_dev)
    e = triples.energy(L, mode=mode).item()
    rel = abs(e - meta["e_t"]) / abs(meta["e_t"])
    print(f"\n{name} {mode}: energy rel {rel:.2e}")
    assert rel < TOL[mode][0], (e, meta["e_t"], rel)


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("name", ["cfg1_o8v40_fvo", "cfg2_o16v120"])
def test_mixed_vjp_vs_fp64(mode, name, cuda_dev):
    meta, arr = golden_io.load(name)
    L = dev_layouts(synth.reference_layouts(golden_io.system(meta)), cuda_dev)
    e64, g64 = triples.energy_vjp(L, 2.0, mode="fp64")
    em, gm = triples.energy_vjp(L, 2.0, mode=mode)
    rel_e = abs(em.item() - e64.item()) / abs(e64.item())
    rel_g = {k: float(torch.linalg.norm(gm[k] - g64[k])) / max(float(torch.linalg.norm(g64[k])), 1e-300)
             for k in golden_io.KEYS}
    print(f"\n{name} {mode}: energy rel {rel_e:.2e}; gradients " + " ".join(f"{k}={x:.1e}" for k, x in rel_g.items()))
    assert rel_e < TOL[mode][0]
    for k in golden_io.KEYS:
        nrm = float(torch.linalg.norm(g64[k]))
        err = float(torch.linalg.norm(gm[k] - g64[k]))
        assert err <= TOL[mode][1] * nrm + 1e-14, (k, err / max(nrm, 1e-300))


@pytest.mark.parametrize("mode", MODES)
def test_mixed_o32_block(mode, cuda_dev):
    """nocc=32 through the block entry (the shapes of the larger workloads)."""
    Ld = synth.device_layouts(32, 48, 144, 5, device=cuda_dev)
    e64 = torch.zeros((), dtype=torch.float64, device=cuda_dev)
    em = torch.zeros((), dtype=torch.float64, device=cuda_dev)
    prob = native.CtProblem(32, 48, *[ctypes.c_void_p(Ld[k].data_ptr()) for k in golden_io.KEYS])
    g64 = {k: torch.zeros_like(Ld[k]) for k in golden_io.KEYS}
    gm = {k: torch.zeros_like(Ld[k]) for k in golden_io.KEYS}
    for G, m, out in ((g64, 0, e64), (gm, native.mode_id(mode), em)):
        gr = native.CtGrads(*[ctypes.c_void_p(G[k].data_ptr()) for k in golden_io.KEYS])
        native.check(native.lib().ct_energy_vjp_block(ctypes.byref(prob), m, 2.0, ctypes.byref(gr), 40, 48, 40, 48,
                                                      ctypes.c_void_p(out.data_ptr()), None))
    torch.cuda.synchronize()
    rel_e = abs(em.item() - e64.item()) / abs(e64.item())
    rel_g = {k: float(torch.linalg.norm(gm[k] - g64[k])) / max(float(torch.linalg.norm(g64[k])), 1e-300)
             for k in golden_io.KEYS}
    print(f"o32 block {mode}: energy rel {rel_e:.2e}; gradients "
          + " ".join(f"{k}={v:.1e}" for k, v in rel_g.items()))
    assert rel_e < TOL[mode][0]
    for k in golden_io.KEYS:
        nrm = float(torch.linalg.norm(g64[k]))
        assert float(torch.linalg.norm(gm[k] - g64[k])) <= TOL[mode][1] * nrm + 1e-14, k


@pytest.mark.parametrize("mode", MODES)
def test_mixed_rejects_unaligned_nocc(mode, cuda_dev):
    meta, _ = golden_io.load("small_o4v10_fvo")
    L = dev_layouts(synth.reference_layouts(golden_io.system(meta)), cuda_dev)
    with pytest.raises(native.CtError):
        triples.energy(L, mode=mode)


def test_bf16x3_more_accurate_than_tf32(cuda_dev):
    """The split-product mode is the more accurate one on the same inputs."""
    meta, _ = golden_io.load("cfg2_o16v120")
    L = dev_layouts(synth.reference_layouts(golden_io.system(meta)), cuda_dev)
    e64, g64 = triples.energy_vjp(L, 2.0, mode="fp64")
    errs = {}
    for mode in MODES:
        em, gm = triples.energy_vjp(L, 2.0, mode=mode)
        errs[mode] = float(torch.linalg.norm(gm["t2T"] - g64["t2T"]) / torch.linalg.norm(g64["t2T"]))
    assert errs["bf16x3"] < 0.25 * errs["tf32"], errs


_PAIR_SCRIPT = r"""
import ctypes, json, sys, torch
sys.path.insert(0, sys.argv[1]); sys.path.insert(0, sys.argv[1] + "/tests")
import golden_io
from pyscfad_b200 import native, synth
dev = torch.device("cuda", 0)
out = {}
for nocc, nvir, blk in ((16, 40, (32, 40, 32, 40)), (32, 48, (40, 48, 40, 48))):
    Ld = synth.device_layouts(nocc, nvir, 3 * nvir, 7, device=dev)
    prob = native.CtProblem(nocc, nvir, *[ctypes.c_void_p(Ld[k].data_ptr()) for k in golden_io.KEYS])
    res = {}
    for mode in ("fp64", "tf32", "bf16x3"):
        e = torch.zeros((), dtype=torch.float64, device=dev)
        G = {k: torch.zeros_like(Ld[k]) for k in golden_io.KEYS}
        gr = native.CtGrads(*[ctypes.c_void_p(G[k].data_ptr()) for k in golden_io.KEYS])
        native.check(native.lib().ct_energy_vjp_block(ctypes.byref(prob), native.mode_id(mode), 2.0, ctypes.byref(gr),
                                                      *blk, ctypes.c_void_p(e.data_ptr()), None))
        torch.cuda.synchronize()
        res[mode] = (e.item(), G)
    e64, g64 = res["fp64"]
    for mode in ("tf32", "bf16x3"):
        em, gm = res[mode]
        out[f"o{nocc}_{mode}"] = [abs(em - e64) / abs(e64)] + [
            float(torch.linalg.norm(gm[k] - g64[k]) / torch.linalg.norm(g64[k])) for k in golden_io.KEYS]
print(json.dumps(out))
"""


def test_f1_cta_pairs_match_fp64():
    """F1 on CTA pairs (tcgen05 cta_group::2, CTB_CTA_PAIRS=1; nocc % 16 == 0)
    against the FP64 path, in a child process that selects the pairs at load."""
    import json
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, CTB_CTA_PAIRS="1")
    r = subprocess.run([sys.executable, "-c", _PAIR_SCRIPT, root], env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    print("CTA-pair F1 errors (energy, then gradients):", out)
    for key, errs in out.items():
        mode = key.split("_")[1]
        assert errs[0] < TOL[mode][0], (key, errs)
        assert max(errs[1:]) < TOL[mode][1], (key, errs)


def _host_call(mode):
    """ctb_ccsd_t_energy_vjp_mode with the reference's 25 arguments and a mode"""
    mid = native.mode_id(mode)

    def call(*args):
        conv = []
        for i, a in enumerate(args):
            if isinstance(a, np.ndarray):
                assert a.dtype == np.float64 and a.flags.c_contiguous
                conv.append(a.ctypes.data_as(ctypes.c_void_p))
            elif i == 5:
                conv.append(ctypes.c_double(a))
            else:
                conv.append(ctypes.c_int(a))
        native.check(native.lib().ctb_ccsd_t_energy_vjp_mode(*conv, mid), "ctb_ccsd_t_energy_vjp_mode")
    return call


@pytest.mark.parametrize("mode", MODES)
def test_mixed_host_entry_in_stages_matches_fp64(mode, cuda_dev, monkeypatch):
    """ctb_ccsd_t_energy_vjp_mode through the reference's slab loop (3 x 2
    slabs), each block run in stages of its jobs' smallest index (many of
    them with 40-job waves: the operand conversion then runs stage by stage),
    against the float64 host entry, within the gradient tolerance."""
    from oracle import ref
    meta, _ = golden_io.load("cfg1_o8v40_fvo")
    L = synth.reference_layouts(golden_io.system(meta))
    g64 = ref.blocked_vjp(_host_call("fp64"), L, 2.0, 3, 2)
    native.lib().ct_release_workspace()
    monkeypatch.setenv("CTB_MAX_WAVE", "40")
    try:
        gm = ref.blocked_vjp(_host_call(mode), L, 2.0, 3, 2)
    finally:
        monkeypatch.delenv("CTB_MAX_WAVE")
        native.lib().ct_release_workspace()
    rel = {k: float(np.linalg.norm(gm[k] - g64[k]) / np.linalg.norm(g64[k])) for k in golden_io.KEYS}
    print(f"\nhost entry in stages, {mode}: " + " ".join(f"{k}={x:.1e}" for k, x in rel.items()))
    for k, x in rel.items():
        assert x <= TOL[mode][1], (k, x)
