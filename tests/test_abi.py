"""CPU: the C-ABI library loads and exports every function include/*.h declares;
argument validation answers without touching a device."""
import ctypes
import glob
import os
import re

import pytest

from pyscfad_b200 import native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_ ]*?[\s\*]+([A-Za-z_][A-Za-z0-9_]*)\s*\(",
                             src, flags=re.M):
            if m.group(1) not in ("if", "while", "for", "return"):
                names.append(m.group(1))
    return sorted(set(names))


def test_header_declares_expected():
    d = declared_functions()
    for name in native.EXPORTS:
        assert name in d, name


def test_library_exports_every_declared_symbol():
    L = native.lib()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing


def test_status_strings_and_version():
    L = native.lib()
    assert L.ct_version() >= 1
    assert L.ct_status_string(0) == b"ok"
    assert b"mode" in L.ct_status_string(-4)


def test_validation_without_device():
    L = native.lib()
    # null problem -> CT_ERR_NULL before any device work
    e = ctypes.c_double(0)
    assert L.ct_energy(None, 0, ctypes.c_void_p(ctypes.addressof(e)), None, None) == -5
    prob = native.CtProblem(0, 10, *([None] * 6))
    assert L.ct_energy(ctypes.byref(prob), 0, ctypes.c_void_p(1), None, None) == -1
    prob = native.CtProblem(4, 10, *([ctypes.c_void_p(8)] * 6))
    assert L.ct_energy(ctypes.byref(prob), 7, ctypes.c_void_p(1), None, None) == -4
    assert L.ctb_ccsd_t_energy(None, *([None] * 5), 4, 10, 0, 10, None, 0) == -5


def test_workspace_bytes_query():
    L = native.lib()
    b64 = L.ct_workspace_bytes(16, 120, 0, 1)
    assert b64 > 7 * 16 ** 3 * 8
    assert L.ct_workspace_bytes(0, 10, 0, 1) < 0


def test_mode_ids():
    assert native.mode_id("fp64") == 0 and native.mode_id("TF32") == 1 and native.mode_id("bf16x3") == 2
    with pytest.raises(native.CtError):
        native.mode_id("fp8")


def test_lno_validation_without_device():
    L = native.lib()
    d = ctypes.c_void_p(8)
    prob = native.CtProblem(4, 10, *([d] * 6))
    gr = native.CtGrads(*([d] * 6))
    # null problem / projector -> CT_ERR_NULL; empty or out-of-range slab -> CT_ERR_SHAPE
    assert L.ct_lno_energy(None, d, 0, 10, d, None, None) == -5
    assert L.ct_lno_energy(ctypes.byref(prob), None, 0, 10, d, None, None) == -5
    assert L.ct_lno_energy(ctypes.byref(prob), d, 3, 3, d, None, None) == -1
    assert L.ct_lno_energy(ctypes.byref(prob), d, 0, 11, d, None, None) == -1
    assert L.ct_lno_energy_vjp(None, d, 1.0, ctypes.byref(gr), d, None, None) == -5
    assert L.ct_lno_energy_vjp(ctypes.byref(prob), d, 1.0, ctypes.byref(gr), None, None, None) == -5
    # a slab block must be diagonal or lie below: (b0,b1,c0,c1) = (2,5,3,6) is neither
    assert L.ct_lno_energy_vjp_block(ctypes.byref(prob), d, 1.0, 2, 5, 3, 6, ctypes.byref(gr), d, None, None) == -1
    big = native.CtProblem(65, 10, *([d] * 6))
    assert L.ct_lno_energy(ctypes.byref(big), d, 0, 10, d, None, None) == -1
    assert L.ctb_lnoccsdt_contract(None, *([None] * 6), 4, 10, 0, 10, None) == -5
    assert L.ctb_lnoccsdt_energy_vjp(*([None] * 6), 1.0, 4, 10, 0, 10, 0, 10, *([None] * 14)) == -5


def test_noalloc_capacity_rule_without_device():
    """ct_energy_noalloc answers CT_ERR_SIZE exactly when
    nvir(nvir+1)(nvir+2)/6 + 7 nocc^3 + 65 exceeds CT_NOALLOC_SCRATCH_DOUBLES
    (the size check comes before any device call).  No integer shape lands on
    the bound itself, so the shapes closest to it on either side are used."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("fake pointers: only meaningful where the call cannot reach a device")
    L = native.lib()
    cap = 4 * 1024 * 1024
    d = ctypes.c_void_p(256)
    for o, v in [(7, 292), (6, 292), (58, 256), (29, 288), (5, 292), (8, 291), (8, 292), (64, 1), (65, 1)]:
        prob = native.CtProblem(o, v, *([d] * 6))
        st = L.ct_energy_noalloc(ctypes.byref(prob), d, None)
        need = v * (v + 1) * (v + 2) // 6 + 7 * o ** 3 + 65
        if o > 64:
            assert st == -1, (o, v, st)
        elif need > cap:
            assert st == -9, (o, v, need, st)
        else:
            assert st == -6, (o, v, need, st)   # fits; CT_ERR_NO_DEVICE on a machine without a GPU


def test_xla_ffi_source_is_header_guarded():
    """The XLA FFI handlers compile to an empty unit where jaxlib's headers are
    absent (this image), so the tree builds everywhere."""
    import shutil
    import subprocess
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no host C++ compiler")
    src = os.path.join(ROOT, "pyscfad_b200", "ffi", "ct_xla_ffi.cc")
    r = subprocess.run([gxx, "-std=c++17", "-fsyntax-only", "-I", os.path.join(ROOT, "include"), src],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_mode_and_iterative_entries_validate_without_device():
    """ct_lno_energy_mode, ct_lno_energy_vjp_mode, ct_t3_init and ct_t3_update
    reject bad arguments before any device work."""
    L = native.lib()
    d = ctypes.c_void_p(8)
    prob = native.CtProblem(4, 10, *([d] * 6))
    gr = native.CtGrads(*([d] * 6))
    assert L.ct_lno_energy_mode(ctypes.byref(prob), 7, d, 0, 10, d, None, None) == -4
    assert L.ct_lno_energy_mode(ctypes.byref(prob), 1, None, 0, 10, d, None, None) == -5
    assert L.ct_lno_energy_mode(ctypes.byref(prob), 1, d, 4, 4, d, None, None) == -1
    assert L.ct_lno_energy_vjp_mode(ctypes.byref(prob), 7, d, 1.0, 0, 10, 0, 10, ctypes.byref(gr), d, None,
                                    None) == -4
    assert L.ct_lno_energy_vjp_mode(ctypes.byref(prob), 1, d, 1.0, 2, 5, 3, 6, ctypes.byref(gr), d, None,
                                    None) == -1
    assert L.ct_t3_init(None, d, d, None) == -5
    assert L.ct_t3_init(ctypes.byref(prob), None, d, None) == -5
    e = [ctypes.c_void_p(8 * (i + 1)) for i in range(8)]
    assert L.ct_t3_update(0, 10, *e, None, None) == -1
    assert L.ct_t3_update(4, 10, e[0], e[1], e[2], e[3], None, e[5], e[6], e[7], e[0], None) == -5
    # t3_new may not alias an input (P3 reads other elements of the products)
    assert L.ct_t3_update(4, 10, e[0], e[1], e[2], e[3], e[4], e[5], e[4], e[7], e[0], None) == -1
