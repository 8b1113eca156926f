"""Device time of the LNO-projected (T) paths beside the canonical ones on
one synthetic system generated in HBM:

    python -m pyscfad_b200.lno.timing [--nocc 32] [--nvir 120] [--reps 3] [--mode fp64]

Prints one JSON line: ms per call (CUDA events on the current stream, after
one warm-up call) of the canonical energy, the LNO energy (rank-half
projector), the canonical energy+VJP and the LNO energy+VJP over every job,
in the precision ``--mode`` names.
"""
from __future__ import annotations

import argparse
import ctypes
import json

import torch

from .. import native, synth, triples


def _time(fn, reps):
    fn()
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record()
    for _ in range(reps):
        fn()
    t1.record()
    torch.cuda.synchronize()
    return t0.elapsed_time(t1) / reps


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--nocc", type=int, default=32)
    ap.add_argument("--nvir", type=int, default=120)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--mode", default="fp64", choices=sorted(native.MODES))
    a = ap.parse_args(argv)
    dev = torch.device("cuda", 0)
    L = synth.device_layouts(a.nocc, a.nvir, 3 * a.nvir, 7, device=dev)
    g = torch.Generator(device="cpu").manual_seed(7)
    u = torch.linalg.qr(torch.randn(a.nocc, a.nocc, generator=g, dtype=torch.float64))[0][: a.nocc // 2]
    mat = (u.t() @ u).to(dev)
    grads = {k: torch.zeros_like(x) for k, x in L.items()}
    mb = torch.zeros_like(mat)
    res = {
        "energy_ms": _time(lambda: triples.energy(L, mode=a.mode), a.reps),
        "lno_energy_ms": _time(lambda: triples.lno_energy(L, mat, mode=a.mode), a.reps),
        "energy_vjp_ms": _time(lambda: triples.energy_vjp(L, 2.0, grads, mode=a.mode), a.reps),
        "lno_energy_vjp_ms": _time(lambda: triples.lno_energy_vjp(L, mat, 1.0, grads, mb, mode=a.mode), a.reps),
    }
    # per-kernel device time of one LNO energy call and one LNO VJP call
    L_ = native.lib()
    kinds = {0: "F1", 1: "F2", 2: "orbit epilogue", 3: "V-term / LNO energy projection", 4: "VB", 5: "TB",
             6: "OB1", 7: "OB2", 8: "reductions / LNO VJP projection", 9: "operand preparation",
             10: "F1 (tcgen05)", 11: "VB (tcgen05)", 12: "TB (tcgen05)", 13: "F2 (tcgen05)", 14: "OB1 (tcgen05)",
             15: "OB2 (tcgen05)"}
    runs = [("lno_energy", lambda: triples.lno_energy(L, mat, mode=a.mode)),
            ("lno_energy_vjp", lambda: triples.lno_energy_vjp(L, mat, 1.0, grads, mb, mode=a.mode))]
    for name, fn in runs:
        native.check(L_.ct_profile_enable(1))
        fn()
        torch.cuda.synchronize()
        prof = {}
        for k, kn in kinds.items():
            tot, n = ctypes.c_double(0), ctypes.c_int(0)
            native.check(L_.ct_profile_read(k, ctypes.byref(tot), ctypes.byref(n)))
            if n.value:
                prof[kn] = round(tot.value, 1)
        native.check(L_.ct_profile_enable(0))
        res[name + "_kernel_ms"] = prof
    res["lno_energy_over_energy"] = res["lno_energy_ms"] / res["energy_ms"]
    res["lno_vjp_over_vjp"] = res["lno_energy_vjp_ms"] / res["energy_vjp_ms"]
    dtype = {"fp64": "f64", "tf32": "tf32", "bf16x3": "bf16x3"}[a.mode]
    print(json.dumps({"nocc": a.nocc, "nvir": a.nvir, "reps": a.reps, "dtype": dtype,
                      **{k: (round(v, 3) if isinstance(v, float) else v) for k, v in res.items()}}))


if __name__ == "__main__":
    main()
