"""Regenerate the golden fixtures from the reference's own compiled CPU kernels.

    make -C oracle && python tests/golden/make_golden.py

Inputs are not stored: they are rebuilt from ``pyscfad_b200.synth.make_system``
with the recorded (nocc, nvir, naux, seed, fvo_sigma); an input checksum is
stored to detect generator drift.  Outputs come from oracle/_ref/libref_cc.so
(the reference's lnoccsdt_contract and ccsd_t_energy_vjp).  Small cases keep
every gradient element; larger cases keep projections of each gradient on
seeded random directions (``direction(key, shape, case_seed)`` below) plus its
Frobenius norm.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

CASES = [
    # name, nocc, nvir, naux, seed, fvo_sigma, full (store whole gradients)
    ("tiny_o3v7", 3, 7, 20, 5, 0.0, True),
    ("small_o4v10_fvo", 4, 10, 30, 7, 1e-2, True),
    ("edge_o2v3", 2, 3, 8, 11, 1e-2, True),
    ("edge_o1v4", 1, 4, 6, 13, 1e-2, True),
    ("mid_o6v17_fvo", 6, 17, 40, 21, 1e-2, False),
    ("cfg1_o8v40", 8, 40, 120, 0, 0.0, False),
    ("cfg1_o8v40_fvo", 8, 40, 120, 0, 1e-2, False),
    ("cfg2_o16v120", 16, 120, 400, 1, 0.0, False),
]
NDIR = 8
KEYS = ("mo_energy", "t1T", "t2T", "vooo", "fvo", "vvop")


def direction(key: str, shape, case_seed: int, k: int) -> np.ndarray:
    rng = np.random.default_rng([case_seed, KEYS.index(key), k, 4242])
    return rng.standard_normal(shape)


def input_checksum(L) -> list:
    return [float(np.sum(L[k])) for k in KEYS] + [float(np.sum(L[k] ** 2)) for k in KEYS]


def main(only=None):
    from pyscfad_b200 import synth
    from oracle import ref
    for name, o, v, naux, seed, fs, full in CASES:
        if only and name not in only:
            continue
        s = synth.make_system(o, v, naux, seed, fvo_sigma=fs)
        L = synth.reference_layouts(s)
        e = ref.energy(**L)
        g = ref.energy_vjp_layouts(**L, et_bar=1.0)
        meta = dict(name=name, nocc=o, nvir=v, naux=naux, seed=seed, fvo_sigma=fs,
                    e_t=e, checksum=input_checksum(L), ndir=NDIR,
                    source="oracle/_ref/libref_cc.so (lnoccsdt_contract x2/3, ccsd_t_energy_vjp et_bar=1)")
        arrays = {}
        for k in KEYS:
            arrays[f"norm_{k}"] = np.array(np.linalg.norm(g[k]))
            arrays[f"proj_{k}"] = np.array([np.vdot(g[k], direction(k, g[k].shape, seed, i))
                                            for i in range(NDIR)])
            if full:
                arrays[f"grad_{k}"] = g[k]
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), meta=json.dumps(meta), **arrays)
        print(name, repr(e))


if __name__ == "__main__":
    main(sys.argv[1:] or None)
