"""GPU: the mixed-precision gate |dE(T)| <= 1e-6 Eh on physical-scale variants.

At the generator's own scale |E(T)| is 1e2 - 1e7 Eh, so an absolute 1e-6 Eh
gate would mean 1e-13 relative, below float64 summation noise.  The
physical-scale variant multiplies every ERI slice by a power of two s
(synth.PHYSICAL_ERI_SCALE) so that |E(T)| of the whole system is about
1e-2 Eh, where the gate is meaningful.

Checked on the nocc=32/nvir=300/naux=900 (seed 2) system, whole:
  * scale invariance: each mode's energy at scale s equals s^2 times its
    energy at scale 1 to 1e-14 relative (a power of two changes no rounding),
    so errors measured at one scale hold at the other;
  * the gate: |E_mode(s) - E_fp64(s)| <= 1e-6 Eh for TF32 and BF16x3.
The nocc=48/nvir=500 system's gate is checked in test_gpu_large.py on the
slab it already computes, through the same scaling.
"""
import ctypes

import pytest
import torch

import golden_io
from pyscfad_b200 import native, synth

pytestmark = pytest.mark.gpu

GATE_EH = 1e-6


def _energy(L, o, v, mode):
    prob = native.CtProblem(o, v, *[ctypes.c_void_p(L[k].data_ptr()) for k in golden_io.KEYS])
    out = torch.zeros((), dtype=torch.float64, device=L["vvop"].device)
    native.check(native.lib().ct_energy(ctypes.byref(prob), native.mode_id(mode), ctypes.c_void_p(out.data_ptr()),
                                        None, None), "ct_energy")
    torch.cuda.synchronize()
    return out.item()


def test_physical_scale_gate_nocc32_nvir300(cuda_dev):
    o, v, naux, seed = 32, 300, 900, 2
    s = synth.PHYSICAL_ERI_SCALE[3]
    torch.cuda.empty_cache()
    L = synth.device_layouts(o, v, naux, seed, device=cuda_dev)
    e1 = {m: _energy(L, o, v, m) for m in ("fp64", "tf32", "bf16x3")}
    L["vvop"].mul_(s)
    L["vooo"].mul_(s)
    es = {m: _energy(L, o, v, m) for m in ("tf32", "bf16x3")}
    es["fp64"] = s * s * e1["fp64"]
    del L
    native.check(native.lib().ct_release_workspace())
    torch.cuda.empty_cache()
    print(f"\nphysical scale s=2^{int(round(__import__('math').log2(s)))}: E_fp64 = {es['fp64']:.6e} Eh "
          f"(generator scale {e1['fp64']:.6e} Eh)")
    for m in ("tf32", "bf16x3"):
        inv = abs(es[m] - s * s * e1[m]) / abs(s * s * e1[m])
        d = abs(es[m] - es["fp64"])
        print(f"  {m}: |dE| = {d:.3e} Eh (rel {d / abs(es['fp64']):.2e}); scale invariance {inv:.1e}")
        assert inv <= 1e-14, (m, inv)
        assert d <= GATE_EH, (m, d)
    assert 1e-3 <= abs(es["fp64"]) <= 1e-1, es["fp64"]
