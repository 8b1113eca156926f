"""ctypes binding of the C-ABI in include/pyscfad_b200.h.

The shared library is built in-tree (``python -m pyscfad_b200._build``) and is
the only compute path: nothing here falls back to a CPU implementation, and any
call made without the library, without a GPU, or with a failing status raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libpyscfad_b200.so")

CT_OK = 0
MODES = {"fp64": 0, "tf32": 1, "bf16x3": 2}

EXPORTS = (
    "ct_version", "ct_status_string", "ct_energy", "ct_energy_vjp",
    "ctb_ccsd_t_energy_vjp", "ctb_ccsd_t_energy_vjp_mode", "ctb_ccsd_t_energy",
    "ct_release_workspace", "ct_workspace_bytes", "ct_energy_vjp_block", "ct_energy_block",
    "ct_profile_enable", "ct_profile_read", "ct_profile_reset", "ct_peak_probe",
    "ct_energy_noalloc", "ct_energy_jobs", "ct_lno_energy", "ct_lno_energy_mode", "ctb_lnoccsdt_contract",
    "ct_lno_energy_vjp",
    "ct_lno_energy_vjp_block", "ct_lno_energy_vjp_mode", "ctb_lnoccsdt_energy_vjp", "ct_t3_init", "ct_t3_update",
    "ct_mlp_forward", "ct_mlp_mse", "ct_mlp_work_floats", "ct_mlp_backward", "ct_mlp_adam",
    "ct_mlp_to_bf16", "ct_mlp_infer_bf16", "ct_surrogate_features", "ct_df_layouts", "ct_df_factor_bar",
)

# surrogate MLP shapes (include/pyscfad_b200.h)
MLP_IN = 12
MLP_HIDDEN = 128
MLP_NPARAM = MLP_HIDDEN * MLP_IN + MLP_HIDDEN + MLP_HIDDEN * MLP_HIDDEN + MLP_HIDDEN + MLP_HIDDEN + 1


class CtProblem(ctypes.Structure):
    _fields_ = [("nocc", ctypes.c_int), ("nvir", ctypes.c_int),
                ("mo_energy", ctypes.c_void_p), ("t1T", ctypes.c_void_p),
                ("t2T", ctypes.c_void_p), ("vooo", ctypes.c_void_p),
                ("fvo", ctypes.c_void_p), ("vvop", ctypes.c_void_p)]


class CtGrads(ctypes.Structure):
    _fields_ = [("mo_energy", ctypes.c_void_p), ("t1T", ctypes.c_void_p),
                ("t2T", ctypes.c_void_p), ("vooo", ctypes.c_void_p),
                ("fvo", ctypes.c_void_p), ("vvop", ctypes.c_void_p)]


class CtError(RuntimeError):
    pass


_lib = None


def lib():
    """Load the library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise CtError(f"pyscfad_b200 CUDA library not built: {LIB_PATH} "
                      "(run python -m pyscfad_b200._build)")
    L = ctypes.CDLL(LIB_PATH)
    dp, vp, ci, cd = ctypes.POINTER(ctypes.c_double), ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    L.ct_version.restype = ci
    L.ct_status_string.restype = ctypes.c_char_p
    L.ct_status_string.argtypes = [ci]
    L.ct_energy.restype = ci
    L.ct_energy.argtypes = [ctypes.POINTER(CtProblem), ci, vp, vp, vp]
    L.ct_energy_vjp.restype = ci
    L.ct_energy_vjp.argtypes = [ctypes.POINTER(CtProblem), ci, cd, ctypes.POINTER(CtGrads), vp, vp]
    blk = [vp, vp, vp, vp, vp, cd, ci, ci, ci, ci, ci, ci, vp, vp, vp, vp,
           vp, vp, vp, vp, vp, vp, vp, vp, vp]
    L.ctb_ccsd_t_energy_vjp.restype = ci
    L.ctb_ccsd_t_energy_vjp.argtypes = blk
    L.ctb_ccsd_t_energy_vjp_mode.restype = ci
    L.ctb_ccsd_t_energy_vjp_mode.argtypes = blk + [ci]
    L.ctb_ccsd_t_energy.restype = ci
    L.ctb_ccsd_t_energy.argtypes = [vp, vp, vp, vp, vp, vp, ci, ci, ci, ci, vp, ci]
    L.ct_energy_vjp_block.restype = ci
    L.ct_energy_vjp_block.argtypes = [ctypes.POINTER(CtProblem), ci, cd, ctypes.POINTER(CtGrads),
                                      ci, ci, ci, ci, vp, vp]
    L.ct_energy_block.restype = ci
    L.ct_energy_block.argtypes = [ctypes.POINTER(CtProblem), ci, ci, ci, vp, vp, vp]
    L.ct_lno_energy.restype = ci
    L.ct_lno_energy.argtypes = [ctypes.POINTER(CtProblem), vp, ci, ci, vp, vp, vp]
    L.ct_lno_energy_mode.restype = ci
    L.ct_lno_energy_mode.argtypes = [ctypes.POINTER(CtProblem), ci, vp, ci, ci, vp, vp, vp]
    L.ct_lno_energy_vjp.restype = ci
    L.ct_lno_energy_vjp.argtypes = [ctypes.POINTER(CtProblem), vp, cd, ctypes.POINTER(CtGrads), vp, vp, vp]
    L.ct_lno_energy_vjp_block.restype = ci
    L.ct_lno_energy_vjp_block.argtypes = [ctypes.POINTER(CtProblem), vp, cd, ci, ci, ci, ci,
                                          ctypes.POINTER(CtGrads), vp, vp, vp]
    L.ct_t3_init.restype = ci
    L.ct_t3_init.argtypes = [ctypes.POINTER(CtProblem), vp, vp, vp]
    L.ct_t3_update.restype = ci
    L.ct_t3_update.argtypes = [ci, ci, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]
    L.ct_lno_energy_vjp_mode.restype = ci
    L.ct_lno_energy_vjp_mode.argtypes = [ctypes.POINTER(CtProblem), ci, vp, cd, ci, ci, ci, ci,
                                         ctypes.POINTER(CtGrads), vp, vp, vp]
    L.ctb_lnoccsdt_energy_vjp.restype = ci
    L.ctb_lnoccsdt_energy_vjp.argtypes = [vp, vp, vp, vp, vp, vp, cd, ci, ci, ci, ci, ci, ci,
                                          vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]
    L.ctb_lnoccsdt_contract.restype = ci
    L.ctb_lnoccsdt_contract.argtypes = [vp, vp, vp, vp, vp, vp, vp, ci, ci, ci, ci, vp]
    L.ct_profile_enable.restype = ci
    L.ct_profile_enable.argtypes = [ci]
    L.ct_profile_read.restype = ci
    L.ct_profile_read.argtypes = [ci, dp, ctypes.POINTER(ci)]
    L.ct_profile_reset.restype = ci
    L.ct_peak_probe.restype = ci
    L.ct_peak_probe.argtypes = [ci, dp]
    L.ct_df_layouts.restype = ci
    L.ct_df_layouts.argtypes = [ci, ci, ci, vp, vp, vp, vp, vp, vp]
    L.ct_df_factor_bar.restype = ci
    L.ct_df_factor_bar.argtypes = [ci, ci, ci, vp, vp, vp, vp, vp, vp, vp, vp, vp]
    L.ct_energy_noalloc.restype = ci
    L.ct_energy_noalloc.argtypes = [ctypes.POINTER(CtProblem), vp, vp]
    L.ct_energy_jobs.restype = ci
    L.ct_energy_jobs.argtypes = [ctypes.POINTER(CtProblem), ci, vp, ci, vp, vp, vp]
    fp = vp
    L.ct_mlp_forward.restype = ci
    L.ct_mlp_forward.argtypes = [fp, fp, ci, fp, fp, fp, vp]
    L.ct_mlp_mse.restype = ci
    L.ct_mlp_mse.argtypes = [fp, fp, ci, fp, vp, vp]
    L.ct_mlp_work_floats.restype = ctypes.c_longlong
    L.ct_mlp_work_floats.argtypes = [ci]
    L.ct_mlp_backward.restype = ci
    L.ct_mlp_backward.argtypes = [fp, fp, fp, fp, fp, ci, fp, fp, vp]
    L.ct_mlp_adam.restype = ci
    L.ct_mlp_adam.argtypes = [fp, fp, fp, fp, ci, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                              ctypes.c_float, ctypes.c_float, vp]
    L.ct_mlp_to_bf16.restype = ci
    L.ct_mlp_to_bf16.argtypes = [fp, vp, vp]
    L.ct_mlp_infer_bf16.restype = ci
    L.ct_mlp_infer_bf16.argtypes = [vp, fp, ci, fp, vp]
    L.ct_surrogate_features.restype = ci
    L.ct_surrogate_features.argtypes = [ctypes.POINTER(CtProblem), vp, ctypes.c_longlong, fp, fp, vp]
    L.ct_release_workspace.restype = ci
    L.ct_workspace_bytes.restype = ctypes.c_longlong
    L.ct_workspace_bytes.argtypes = [ci, ci, ci, ci]
    _lib = L
    return L


def check(status: int, what: str = "call"):
    if status != CT_OK:
        msg = lib().ct_status_string(status).decode()
        raise CtError(f"pyscfad_b200 {what} failed: status {status} ({msg})")


def mode_id(mode) -> int:
    if isinstance(mode, int):
        return mode
    try:
        return MODES[mode.lower()]
    except KeyError:
        raise CtError(f"unknown precision mode {mode!r}; expected one of {sorted(MODES)}") from None
