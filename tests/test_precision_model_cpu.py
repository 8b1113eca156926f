"""CPU: where the mixed modes' energy error comes from (a numpy model of each
rounding, on the nocc=8/nvir=40 golden system).

* TF32 operands (10-bit mantissa, round to nearest) alone put the energy off by
  a few 1e-6 relative, which is what the TF32 path shows on this system;
* BF16x3 operands (x = hi + lo, two bf16 planes) alone: about 1e-8;
* float32 storage of the W blocks and float32 orbit arithmetic (W, V, r3),
  with float64 denominators and sums as the kernels keep them: about 1e-10.
So a BF16x3 energy error far above 1e-8 cannot come from its operands or from
the float32 epilogue; it is the tensor pipe's float32 accumulation.
"""
import numpy as np

import golden_io
from oracle import ccsd_t_np as onp
from pyscfad_b200 import synth


def tf32(x):
    b = x.astype(np.float32).view(np.uint32).astype(np.uint64)
    b = (b + (1 << 12)) & ~np.uint64((1 << 13) - 1)
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def bf16(x):
    b = x.astype(np.float32).view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & ~np.uint64(0xFFFF)
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def bf16x3(x):
    hi = bf16(x)
    return hi + bf16(x - hi)


def rounded(L, f, o):
    Lr = dict(L)
    vv = L["vvop"].copy()
    vv[..., o:] = f(vv[..., o:])
    Lr["vvop"] = vv
    Lr["t2T"], Lr["vooo"] = f(L["t2T"]), f(L["vooo"])
    return Lr


def energy_f32_epilogue(L, jobs):
    """W blocks rounded to float32, W/V/r3 in float32, products and sums in float64."""
    o = L["t1T"].shape[1]
    t2T, vvop, vooo = L["t2T"], L["vvop"], L["vooo"]
    t1h = (0.5 * L["t1T"]).astype(np.float32)
    total = 0.0
    for s0 in range(0, len(jobs), 512):
        J = jobs[s0:s0 + 512]
        w = np.zeros((len(J), o, o, o), np.float32)
        v = np.zeros((len(J), o, o, o), np.float32)
        for s, (x, y, z) in enumerate(onp._orderings(J)):
            P = np.einsum("jpf,jfqr->jpqr", vvop[x, y, :, o:], t2T[z], optimize=True)
            P -= np.einsum("jpql,jlr->jpqr", vooo[x], t2T[z, y], optimize=True)
            V = np.einsum("jpq,jr->jpqr", vvop[x, y, :, :o].astype(np.float32), t1h[z])
            w += P.astype(np.float32).transpose(onp._b(onp.SCATTER_T[s]))
            v += V.transpose(onp._b(onp.SCATTER_T[s]))
        zz = onp.r3(w + v).astype(np.float32)
        d3, _ = onp._d3(L, J)
        total += 2.0 * float((w.astype(np.float64) * zz.astype(np.float64) * d3).sum())
    return total


def test_rounding_model_of_the_mixed_modes():
    meta, _ = golden_io.load("cfg1_o8v40")
    s = golden_io.system(meta)
    L = synth.reference_layouts(s)
    o, v = s.nocc, s.nvir
    e64 = meta["e_t"]
    rel = lambda e: abs(e - e64) / abs(e64)  # noqa: E731
    r_tf32 = rel(onp.energy(rounded(L, tf32, o)))
    r_bf = rel(onp.energy(rounded(L, bf16x3, o)))
    r_epi = rel(energy_f32_epilogue(L, onp.sorted_jobs(v)))
    print(f"\noperands tf32 {r_tf32:.1e}, operands bf16x3 {r_bf:.1e}, float32 W storage + epilogue {r_epi:.1e}")
    assert 1e-6 < r_tf32 < 2e-5
    assert r_bf < 5e-8
    assert r_epi < 1e-9
