"""Iterative (T) on the full 6-D triples amplitudes — mirror of the solver in
pyscfad/cc/ccsd_t_slow.py:128-293 (``iterative_kernel``, ``update_amps``,
``energy``) on the device.

The reference forms t3[i,j,k,a,b,c] with JAX einsums.  Here:
  * the seed t3_c = P6(w + v) / d3 (update_amps' initial guess, :188-208) and
    the energy weight t3_x = r3_6d(P6(w)) / 3 (energy, :210-220: r3_6d and d3
    commute, so energy(t2, t3) = sum t3 * t3_x) come from the F1/F2 GEMMs and
    the orbit epilogue of the float64 (T) path, which write every element at
    all simultaneous permutations of (a, b, c) and (i, j, k) (``ct_t3_init``);
  * a step is t3 <- t3_c + (P3(fvv' t3) - P3(foo' t3)) / d3 with fvv', foo'
    the Fock blocks without their diagonals: the two products are one plain
    GEMM each (cuBLAS): fvv' on the first virtual index of the
    [a][b][c][i][j][k] array, foo' on the first occupied index of an
    occupied-major copy [i][a][b][c][j][k]; the P3 sums, the division, the next
    step's occupied-major copy and the fixed-order sums of |t3_new - t3|^2 and
    of the energy are one kernel (``ct_t3_update``).
``t3`` is returned as the reference's [i,j,k,a,b,c] view.  DIIS (the
reference's optional ``run_diis``) and the implicit-differentiation backward
of ``make_implicit_diff`` are not built.  Memory: eight (v^3 o^3) float64
arrays on the device.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from .. import native, triples
from .ccsd_t import _dev, kernel_layouts


def _ovvv_full(eris, nvir):
    ovvv = eris.get_ovvv() if hasattr(eris, "get_ovvv") else eris.ovvv
    if np.ndim(ovvv) == 3:
        from .eris import unpack_tril
        ovvv = unpack_tril(ovvv, nvir)
    return ovvv


def t3_seed(L: dict):
    """(t3_c, t3_x): P6(w + v) / d3 and r3_6d(P6(w)) / 3 as (v,v,v,o,o,o) device arrays."""
    nvir, nocc = L["t1T"].shape
    dev = L["t1T"].device
    shape = (nvir, nvir, nvir, nocc, nocc, nocc)
    t3c = torch.empty(shape, dtype=torch.float64, device=dev)
    t3x = torch.empty(shape, dtype=torch.float64, device=dev)
    prob = triples._problem(L, nocc, nvir)
    with torch.cuda.device(dev):
        st = native.lib().ct_t3_init(ctypes.byref(prob), ctypes.c_void_p(t3c.data_ptr()),
                                     ctypes.c_void_p(t3x.data_ptr()), triples._stream(dev))
    native.check(st, "ct_t3_init")
    return t3c, t3x


def _offdiag(f):
    f = f.clone()
    f.diagonal().zero_()
    return f


def iterative_kernel(mycc, eris=None, t1=None, t2=None, t3=None, max_cycle=50, tol=1e-8, tolnormt=1e-6,
                     verbose=None, stats: dict | None = None):
    """(conv, E, t3) of the iterative (T) solver (pyscfad/cc/ccsd_t_slow.py:262-293).

    ``eris`` needs mo_energy, fock, ovov, ovoo and ovvv (packed or full);
    ``t3`` (optional, [i,j,k,a,b,c]) replaces the initial guess.  Converged
    when |dE| < tol and |t3_new - t3| < tolnormt (the reference's _iter,
    :233-260).  ``stats`` (optional dict) receives the number of cycles and
    their mean device time (CUDA events) as "cycles" and "cycle_ms"."""
    del verbose
    if eris is None:
        eris = mycc.ao2mo(mycc.mo_coeff)
    if t1 is None:
        t1 = mycc.t1
    if t2 is None:
        t2 = mycc.t2
    dev = _dev()
    nocc, nvir = np.shape(t1)
    L = kernel_layouts(t1, t2, eris.mo_energy, eris.fock, eris.ovoo, eris.ovov, _ovvv_full(eris, nvir), dev)
    fock = torch.as_tensor(np.asarray(eris.fock) if not isinstance(eris.fock, torch.Tensor) else eris.fock,
                           dtype=torch.float64).to(dev)
    foo, fvv = _offdiag(fock[:nocc, :nocc]), _offdiag(fock[nocc:, nocc:])
    t3c, t3x = t3_seed(L)
    if t3 is None:
        cur = t3c.clone()
    else:
        cur = torch.as_tensor(t3, dtype=torch.float64).to(dev).permute(3, 4, 5, 0, 1, 2).contiguous()
    et = float(torch.sum(cur * t3x))
    cur_m = cur.permute(3, 0, 1, 2, 4, 5).contiguous()     # [i][a][b][c][j][k]
    tvv, too_m = torch.empty_like(t3c), torch.empty_like(t3c)
    new, new_m = torch.empty_like(t3c), torch.empty_like(t3c)
    sums = torch.zeros(2, dtype=torch.float64, device=dev)
    conv = False
    ncyc = 0
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)] if stats is not None else None
    with torch.cuda.device(dev):
        if ev:
            ev[0].record()
        for _ in range(max_cycle):
            ncyc += 1
            # fvv' t3 on the first virtual index; foo' t3 on the first occupied
            # index of the occupied-major copy
            torch.mm(fvv, cur.view(nvir, -1), out=tvv.view(nvir, -1))
            torch.mm(foo, cur_m.view(nocc, -1), out=too_m.view(nocc, -1))
            p = [ctypes.c_void_p(x.data_ptr()) for x in (L["mo_energy"], t3c, tvv, too_m, cur, t3x, new, new_m, sums)]
            st = native.lib().ct_t3_update(nocc, nvir, *p, triples._stream(dev))
            native.check(st, "ct_t3_update")
            normt2, e_new = sums.tolist()
            cur, new = new, cur
            cur_m, new_m = new_m, cur_m
            eold, et = et, e_new
            if abs(et - eold) < tol and normt2 ** 0.5 < tolnormt:
                conv = True
                break
        if ev:
            ev[1].record()
            torch.cuda.synchronize(dev)
            stats["cycles"] = ncyc
            stats["cycle_ms"] = ev[0].elapsed_time(ev[1]) / max(1, ncyc)
    return conv, et, cur.permute(3, 4, 5, 0, 1, 2)


def energy(t3_x: torch.Tensor, t3: torch.Tensor) -> float:
    """energy(t2, t3, eris) of :210-220 from the seed's weight t3_x (both [a][b][c][i][j][k])."""
    return float(torch.sum(t3 * t3_x))


def _timing(argv=None):
    """python -m pyscfad_b200.cc.ccsd_t_iter [--nocc 16] [--nvir 60]: device time
    of the seed and of the cycles on a synthetic system whose occupied and
    virtual Fock blocks carry small off-diagonal parts; one JSON line."""
    import argparse
    import dataclasses
    import json
    import time

    from .. import synth
    ap = argparse.ArgumentParser()
    ap.add_argument("--nocc", type=int, default=16)
    ap.add_argument("--nvir", type=int, default=60)
    ap.add_argument("--scale", type=float, default=0.02)
    a = ap.parse_args(argv)
    s = synth.make_system(a.nocc, a.nvir, 3 * a.nvir, 11)
    rng = np.random.default_rng(11)
    f = np.array(s.fock, copy=True)
    for lo, hi in ((0, a.nocc), (a.nocc, a.nocc + a.nvir)):
        x = rng.standard_normal((hi - lo, hi - lo)) * a.scale
        x = 0.5 * (x + x.T)
        np.fill_diagonal(x, 0.0)
        f[lo:hi, lo:hi] += x
    s = dataclasses.replace(s, fock=f)
    mycc = type("CC", (), {"t1": s.t1, "t2": s.t2})()
    dev = _dev()
    L = kernel_layouts(s.t1, s.t2, s.mo_energy, s.fock, s.ovoo, s.ovov, s.ovvv, dev)
    t3_seed(L)   # warm-up (plan, workspace)
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ev[0].record()
    t3c, t3x = t3_seed(L)
    ev[1].record()
    torch.cuda.synchronize()
    seed_ms = ev[0].elapsed_time(ev[1])
    del t3c, t3x, L
    t0 = time.perf_counter()
    st: dict = {}
    conv, e, _ = iterative_kernel(mycc, s, tol=1e-10, tolnormt=1e-9, stats=st)
    torch.cuda.synchronize()
    wall = (time.perf_counter() - t0) * 1e3
    n = a.nvir ** 3 * a.nocc ** 3
    print(json.dumps({"nocc": a.nocc, "nvir": a.nvir, "t3_elements": n, "t3_gb": n * 8 / 1e9,
                      "seed_ms": round(seed_ms, 2), "cycles": st["cycles"], "cycle_ms": round(st["cycle_ms"], 2),
                      "solver_wall_ms": round(wall, 1), "converged": conv, "energy": e}))


if __name__ == "__main__":
    _timing()
