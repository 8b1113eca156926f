"""GPU: the tcgen05 modes against the FP64 path at the sizes of the larger
workloads (nocc=32/nvir=300 and the nocc=48/nvir=500 benchmark system), and
additivity of a-slab energies on the benchmark system.

The systems are generated on the device; the comparison runs the last a-slab
of each (all jobs with a0 <= a < a1, through the off-diagonal and diagonal
blocks the reference's driver issues), about 250k jobs at nvir=500.  Gradient buffers accumulate, so one buffer set holds the FP64 VJP
(cotangent +2) and then the mixed VJP with cotangent -2 is added to it: what
is left is g64 - gm, and no second gradient set of vvop's size is needed.

Tolerances, relative to |E| and to each gradient's norm: energy 2e-5 in both
modes, gradients 2e-3 (TF32) and 1e-3 (BF16x3); the largest errors observed on
these systems are TF32 2.0e-6 / 5.7e-4 and BF16x3 2.8e-6 / 4.3e-4 (the t2T and
vooo gradients, summed over many terms in float32, are where the two modes
meet).  Slab
additivity: |E[a0,a2) - E[a0,a1) - E[a1,a2)| <= 1e-12 |E[a0,a2)|.

Physical-scale gate on the benchmark system: with the ERIs scaled by
s = synth.PHYSICAL_ERI_SCALE[4] (|E(T)| of the whole system about 1e-2 Eh),
each mode's slab error is s^2 times the one measured here (a power-of-two
scale changes no rounding; tests/test_gpu_physical.py checks that identity),
and it must stay within 1e-6 Eh.
"""
import ctypes

import pytest
import torch

import golden_io
from pyscfad_b200 import native, synth

pytestmark = pytest.mark.gpu

TOL = {"tf32": (2e-5, 2e-3), "bf16x3": (2e-5, 1e-3)}


def _vp(t):
    return ctypes.c_void_p(t.data_ptr())


def _problem(L, o, v):
    return native.CtProblem(o, v, *[_vp(L[k]) for k in golden_io.KEYS])


def _vjp(prob, mode, et_bar, G, a0, a1):
    """The a-slab [a0, a1) as the reference's driver splits it: the off-diagonal
    block (b < a0) and the diagonal block; returns the slab's energy."""
    gr = native.CtGrads(*[_vp(G[k]) for k in golden_io.KEYS])
    out = torch.zeros(2, dtype=torch.float64, device=G["vvop"].device)
    for i, (b0, b1) in enumerate(((0, a0), (a0, a1))):
        native.check(native.lib().ct_energy_vjp_block(ctypes.byref(prob), native.mode_id(mode), et_bar,
                                                      ctypes.byref(gr), a0, a1, b0, b1, _vp(out[i:i + 1]), None))
    torch.cuda.synchronize()
    return out.sum().item()


def _compare(nocc, nvir, naux, seed, a0, a1, dev, slab_check=False, phys_scale=None):
    torch.cuda.empty_cache()
    L = synth.device_layouts(nocc, nvir, naux, seed, device=dev, fvo_sigma=1e-3)
    prob = _problem(L, nocc, nvir)
    G = {k: torch.zeros_like(L[k]) for k in golden_io.KEYS}
    f64 = dict(dtype=torch.float64, device=dev)
    ref = _vjp(prob, "fp64", 2.0, G, a0, a1)
    norms = {k: float(torch.linalg.norm(G[k])) for k in golden_io.KEYS}
    report = {}
    try:
        for mode in ("tf32", "bf16x3"):
            em = _vjp(prob, mode, -2.0, G, a0, a1)      # G = g64 - gm
            rel_e = abs(em - ref) / abs(ref)
            rel_g = {k: float(torch.linalg.norm(G[k])) / max(norms[k], 1e-300) for k in golden_io.KEYS}
            report[mode] = (rel_e, rel_g)
            assert rel_e < TOL[mode][0], (mode, em, ref, rel_e)
            if phys_scale is not None:
                d_phys = phys_scale ** 2 * abs(em - ref)
                report[mode + "_phys"] = d_phys
                assert d_phys <= 1e-6, (mode, d_phys)
            for k in golden_io.KEYS:
                assert rel_g[k] <= TOL[mode][1] + 1e-14 / max(norms[k], 1e-300), (mode, k, rel_g[k])
            _vjp(prob, mode, 2.0, G, a0, a1)            # back to g64 for the next mode
        if slab_check:
            whole = torch.zeros((), **f64)
            parts = torch.zeros(2, **f64)
            mid = (a0 + a1) // 2
            lib = native.lib()
            native.check(lib.ct_energy_block(ctypes.byref(prob), native.mode_id("tf32"), a0, a1, _vp(whole),
                                             None, None))
            native.check(lib.ct_energy_block(ctypes.byref(prob), native.mode_id("tf32"), a0, mid, _vp(parts[0:1]),
                                             None, None))
            native.check(lib.ct_energy_block(ctypes.byref(prob), native.mode_id("tf32"), mid, a1, _vp(parts[1:2]),
                                             None, None))
            torch.cuda.synchronize()
            w, p = whole.item(), parts.sum().item()
            report["slabs"] = (w, p)
            assert abs(w - p) <= 1e-12 * abs(w), (w, p)
            assert abs(w - ref) / abs(ref) < TOL["tf32"][0]
    finally:
        del G, L
        native.check(native.lib().ct_release_workspace())
        torch.cuda.empty_cache()
    print(f"\nnocc={nocc} nvir={nvir} a=[{a0},{a1}) E64={ref:.12e}")
    for mode in ("tf32", "bf16x3"):
        if mode in report:
            rel_e, rel_g = report[mode]
            print(f"  {mode}: energy rel {rel_e:.2e}; gradient rel max {max(rel_g.values()):.2e} "
                  + " ".join(f"{k}={x:.1e}" for k, x in rel_g.items()))
            if mode + "_phys" in report:
                print(f"  {mode}: physical-scale |dE| of the slab {report[mode + '_phys']:.2e} Eh")
    if "slabs" in report:
        print(f"  tf32 slabs: whole {report['slabs'][0]:.15e} parts {report['slabs'][1]:.15e}")


def test_modes_vs_fp64_nocc32_nvir300(cuda_dev):
    _compare(32, 300, 900, 2, 292, 300, cuda_dev)


def test_modes_vs_fp64_and_additivity_benchmark_system(cuda_dev):
    """nocc=48/nvir=500: inputs 57 GB, one gradient set 57 GB, the mixed
    path's cached operand copies 31 GB and the wave scratch; the test asks
    for the headroom before it allocates so a short device fails with a
    message instead of an allocation error half-way."""
    torch.cuda.empty_cache()
    free, _ = torch.cuda.mem_get_info(cuda_dev)
    assert free >= 165e9, f"needs ~160 GB free on the device, has {free / 1e9:.1f} GB"
    _compare(48, 500, 1500, 3, 498, 500, cuda_dev, slab_check=True, phys_scale=synth.PHYSICAL_ERI_SCALE[4])
