"""GPU: the allocation-free energy entry point (ct_energy_noalloc).

It serves callers that must not have the library allocate device memory (a
framework that owns all device memory, such as an XLA FFI handler, or callers
avoiding cudaMalloc's device synchronization).  Its scratch is a fixed 32 MiB
file-scope device array shared by every call, so this test calls it twice in a
row through the C-ABI and checks both results against ct_energy within the
float64 tolerance used by the other parity tests.  The file is named to be
collected last.
"""
import ctypes

import numpy as np
import pytest
import torch

import golden_io
from pyscfad_b200 import native, synth

pytestmark = pytest.mark.gpu


def _problem(L, o, v):
    return native.CtProblem(o, v, *[ctypes.c_void_p(L[k].data_ptr()) for k in golden_io.KEYS])


@pytest.mark.parametrize("name", ["cfg1_o8v40_fvo", "mid_o6v17_fvo"])
def test_noalloc_energy_matches_ct_energy_twice(name, cuda_dev):
    meta, _ = golden_io.load(name)
    L = {k: torch.from_numpy(np.ascontiguousarray(x)).to(cuda_dev)
         for k, x in synth.reference_layouts(golden_io.system(meta)).items()}
    prob = _problem(L, meta["nocc"], meta["nvir"])
    lib = native.lib()
    ref = torch.zeros((), dtype=torch.float64, device=cuda_dev)
    native.check(lib.ct_energy(ctypes.byref(prob), 0, ctypes.c_void_p(ref.data_ptr()), None, None), "ct_energy")
    tol = max(1e-10, 1e-12 * abs(meta["e_t"]))
    for _ in range(2):
        out = torch.full((), float("nan"), dtype=torch.float64, device=cuda_dev)
        native.check(lib.ct_energy_noalloc(ctypes.byref(prob), ctypes.c_void_p(out.data_ptr()), None),
                     "ct_energy_noalloc")
        torch.cuda.synchronize()
        assert abs(out.item() - ref.item()) <= tol, (out.item(), ref.item())
        assert abs(out.item() - meta["e_t"]) <= tol


def test_noalloc_rejects_oversize(cuda_dev):
    # nvir = 400 needs 400*401*402/6 > 4 Mi doubles for the job energies alone
    o, v = 8, 400
    dummy = torch.zeros(16, dtype=torch.float64, device=cuda_dev)
    prob = native.CtProblem(o, v, *[ctypes.c_void_p(dummy.data_ptr())] * 6)
    out = torch.zeros((), dtype=torch.float64, device=cuda_dev)
    st = native.lib().ct_energy_noalloc(ctypes.byref(prob), ctypes.c_void_p(out.data_ptr()), None)
    assert st == -9
