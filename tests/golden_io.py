"""Loads the golden fixtures written by tests/golden/make_golden.py."""
import json
import os

import numpy as np

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
KEYS = ("mo_energy", "t1T", "t2T", "vooo", "fvo", "vvop")


def names():
    return sorted(f[:-4] for f in os.listdir(HERE) if f.endswith(".npz"))


def load(name):
    z = np.load(os.path.join(HERE, name + ".npz"))
    meta = json.loads(str(z["meta"]))
    arrays = {k: z[k] for k in z.files if k != "meta"}
    return meta, arrays


def direction(key, shape, case_seed, k):
    rng = np.random.default_rng([case_seed, KEYS.index(key), k, 4242])
    return rng.standard_normal(shape)


def system(meta):
    from pyscfad_b200 import synth
    return synth.make_system(meta["nocc"], meta["nvir"], meta["naux"], meta["seed"],
                             fvo_sigma=meta["fvo_sigma"])


def checksum(L):
    return [float(np.sum(L[k])) for k in KEYS] + [float(np.sum(L[k] ** 2)) for k in KEYS]
