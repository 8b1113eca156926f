"""Oracle (test infrastructure): ctypes driver for the reference's own CPU
(T) kernels, compiled from the reference sources into oracle/_ref/libref_cc.so
by oracle/Makefile.

Only tests, the smoke check and the benchmark's CPU-baseline leg use this
module; the product never does.

Entry points used (pyscfadlib/pyscfadlib/vjp/cc):
  * ``lnoccsdt_contract`` (lno_ccsd_t.c:96-138) with mat = I gives 3/2 of the
    canonical (T) energy; pyscfad/lno/ccsd_t.py:111 applies the 2/3.  With a
    general projector it is the LNO-projected energy (``lno_contract``).
  * ``ccsd_t_energy_vjp`` (ccsd_t_vjp.c:332-497), driven over the single slab
    block (a0,a1,b0,b1) = (0,nvir,0,nvir), which enumerates every a>=b>=c job
    (ccsd_t.c:43-69) with vvop itself as the row/col caches.
The layout transforms and the packed-tril ovvv gradient restate the Python
driver pyscfad/cc/ccsd_t.py:82-192.
"""
from __future__ import annotations

import ctypes
import os
import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libref_cc.so")
_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError(f"oracle library missing: {LIB_PATH} (run make -C oracle)")
        _lib = ctypes.CDLL(LIB_PATH)
        _lib.lnoccsdt_contract.restype = None
        _lib.ccsd_t_energy_vjp.restype = None
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.c_void_p)


def energy(mo_energy, t1T, t2T, vooo, fvo, vvop, a0: int = 0, a1: int | None = None) -> float:
    """Canonical E(T) from the reference kernel (reference layouts).

    With (a0, a1) a sub-range of the outer virtual index, returns that slab's
    share (still x2/3), which is how bounded CPU samples are timed.
    """
    nvir, nocc = t1T.shape
    if a1 is None:
        a1 = nvir
    mat = np.eye(nocc)
    e = np.zeros(1)
    args = [np.ascontiguousarray(x, dtype=np.float64) for x in (mo_energy, t1T, t2T, vooo, fvo, vvop)]
    lib().lnoccsdt_contract(_p(e), _p(mat), *[_p(x) for x in args[:5]],
                            ctypes.c_int(nocc), ctypes.c_int(nvir),
                            ctypes.c_int(a0), ctypes.c_int(a1), _p(args[5]))
    return float(e[0]) * 2.0 / 3.0


def lno_contract(mat, mo_energy, t1T, t2T, vooo, fvo, vvop, a0: int = 0, a1: int | None = None) -> float:
    """Raw ``lnoccsdt_contract`` (lno_ccsd_t.c:96-138) with a general
    projector ``mat`` (nocc, nocc): the sum over LNO jobs (a, b>=c) with
    a0 <= a < a1 of fac * (w projected on its first occupied index) . z / D,
    without the driver's 2/3."""
    nvir, nocc = t1T.shape
    if a1 is None:
        a1 = nvir
    e = np.zeros(1)
    m = np.ascontiguousarray(mat, dtype=np.float64)
    args = [np.ascontiguousarray(x, dtype=np.float64) for x in (mo_energy, t1T, t2T, vooo, fvo, vvop)]
    lib().lnoccsdt_contract(_p(e), _p(m), *[_p(x) for x in args[:5]],
                            ctypes.c_int(nocc), ctypes.c_int(nvir),
                            ctypes.c_int(a0), ctypes.c_int(a1), _p(args[5]))
    return float(e[0])


def lno_energy_vjp_block(mat, mo_energy, t1T, t2T, vooo, fvo, vvop, et_bar: float, b0: int, b1: int,
                         c0: int, c1: int):
    """One block of the LNO backward's slab loop (pyscfad/lno/ccsd_t.py:154-220):
    ``lnoccsdt_energy_vjp`` on (b0,b1,c0,c1) with the caches the driver cuts
    (rows vvop[s0:s1, :], columns vvop[:, s0:s1]), and the cache gradients
    added back into a full vvop_bar as the driver does.  Returns (mat_bar,
    gradients in the kernel layouts)."""
    nvir, nocc = t1T.shape
    lib().lnoccsdt_energy_vjp.restype = None
    m = np.ascontiguousarray(mat, dtype=np.float64)
    args = [np.ascontiguousarray(x, dtype=np.float64) for x in (mo_energy, t1T, t2T, vooo, fvo)]
    vvop = np.ascontiguousarray(vvop, dtype=np.float64)

    def caches(s0, s1):
        row = np.ascontiguousarray(vvop[s0:s1, :])
        col = row if (s0, s1) == (0, nvir) else np.ascontiguousarray(vvop[:, s0:s1])
        return row, col, np.zeros_like(row), (None if col is row else np.zeros_like(col))

    ra, ca, rab, cab = caches(b0, b1)
    cab = rab if cab is None else cab
    if (c0, c1) == (b0, b1):
        rb, cb, rbb, cbb = ra, ca, rab, cab
    else:
        rb, cb, rbb, cbb = caches(c0, c1)
        cbb = rbb if cbb is None else cbb
    mat_bar = np.zeros_like(m)
    bars = [np.zeros_like(x) for x in args]
    lib().lnoccsdt_energy_vjp(_p(m), *[_p(x) for x in args], ctypes.c_double(et_bar),
                              ctypes.c_int(nocc), ctypes.c_int(nvir),
                              ctypes.c_int(b0), ctypes.c_int(b1), ctypes.c_int(c0), ctypes.c_int(c1),
                              _p(ra), _p(ca), _p(rb), _p(cb),
                              _p(mat_bar), *[_p(x) for x in bars],
                              _p(rab), _p(cab), _p(rbb), _p(cbb))
    vvop_bar = np.zeros_like(vvop)

    def add(s0, s1, rowbar, colbar):
        vvop_bar[s0:s1, :] += rowbar
        if (s0, s1) != (0, nvir):
            vvop_bar[:, s0:s1] += colbar

    add(b0, b1, rab, cab)
    if (c0, c1) != (b0, b1):
        add(c0, c1, rbb, cbb)
    out = dict(zip(("mo_energy", "t1T", "t2T", "vooo", "fvo"), bars))
    out["vvop"] = vvop_bar
    return mat_bar, out


def lno_energy_vjp(mat, mo_energy, t1T, t2T, vooo, fvo, vvop, et_bar: float = 1.0):
    """``lnoccsdt_energy_vjp`` (lno_ccsd_t_vjp.c:400-566) over the full block
    (b0,b1,c0,c1) = (0,nvir,0,nvir), i.e. every LNO job (a, b>=c), with vvop
    itself as the four caches.  ``et_bar`` is passed as it is (the driver's
    2/3, pyscfad/lno/ccsd_t.py:127, is the caller's).  Returns (mat_bar,
    gradients in the kernel layouts)."""
    nvir, nocc = t1T.shape
    lib().lnoccsdt_energy_vjp.restype = None
    m = np.ascontiguousarray(mat, dtype=np.float64)
    args = [np.ascontiguousarray(x, dtype=np.float64) for x in (mo_energy, t1T, t2T, vooo, fvo)]
    vvop = np.ascontiguousarray(vvop, dtype=np.float64)
    mat_bar = np.zeros_like(m)
    bars = [np.zeros_like(x) for x in args]
    vvop_bar = np.zeros_like(vvop)
    lib().lnoccsdt_energy_vjp(_p(m), *[_p(x) for x in args], ctypes.c_double(et_bar),
                              ctypes.c_int(nocc), ctypes.c_int(nvir),
                              ctypes.c_int(0), ctypes.c_int(nvir), ctypes.c_int(0), ctypes.c_int(nvir),
                              _p(vvop), _p(vvop), _p(vvop), _p(vvop),
                              _p(mat_bar), *[_p(x) for x in bars],
                              _p(vvop_bar), _p(vvop_bar), _p(vvop_bar), _p(vvop_bar))
    out = dict(zip(("mo_energy", "t1T", "t2T", "vooo", "fvo"), bars))
    out["vvop"] = vvop_bar
    return mat_bar, out


def energy_vjp_layouts(mo_energy, t1T, t2T, vooo, fvo, vvop, et_bar: float = 1.0,
                       a0: int = 0, a1: int | None = None, b0: int = 0, b1: int | None = None):
    """Gradients in the kernel layouts (mo_energy, t1T, t2T, vooo, fvo, vvop).

    ``et_bar`` is the cotangent of E(T); the driver's factor 2
    (pyscfad/cc/ccsd_t.py:86) is applied here.  The default block covers all
    jobs; a diagonal slab (a0,a1,a0,a1) restricts to a>=b>=c with a0<=c<=b<=a<a1
    plus c<a0, as ccsd_t.c:43-69 enumerates.
    """
    nvir, nocc = t1T.shape
    if a1 is None:
        a1 = nvir
    if b1 is None:
        b0, b1 = a0, a1
    assert (a0, a1) == (b0, b1), "only diagonal slabs are driven from here"
    args = [np.ascontiguousarray(x, dtype=np.float64) for x in (mo_energy, t1T, t2T, vooo, fvo)]
    vvop = np.ascontiguousarray(vvop, dtype=np.float64)
    bars = [np.zeros_like(x) for x in args]
    cache_row = np.ascontiguousarray(vvop[a0:a1, :a1])
    cache_row_bar = np.zeros_like(cache_row)
    if a0 == 0:
        cache_col, cache_col_bar = cache_row, cache_row_bar
    else:
        cache_col = np.ascontiguousarray(vvop[:a0, a0:a1])
        cache_col_bar = np.zeros_like(cache_col)
    lib().ccsd_t_energy_vjp(*[_p(x) for x in args], ctypes.c_double(2.0 * et_bar),
                            ctypes.c_int(nocc), ctypes.c_int(nvir),
                            ctypes.c_int(a0), ctypes.c_int(a1), ctypes.c_int(a0), ctypes.c_int(a1),
                            _p(cache_row), _p(cache_col), _p(cache_row), _p(cache_col),
                            *[_p(x) for x in bars],
                            _p(cache_row_bar), _p(cache_col_bar), _p(cache_row_bar), _p(cache_col_bar))
    vvop_bar = np.zeros_like(vvop)
    vvop_bar[a0:a1, :a1] += cache_row_bar
    if a0 != 0:
        vvop_bar[:a0, a0:a1] += cache_col_bar
    names = ("mo_energy", "t1T", "t2T", "vooo", "fvo")
    out = {n: b for n, b in zip(names, bars)}
    out["vvop"] = vvop_bar
    return out


def slabs(start: int, stop: int, nslab: int):
    """Partition [start, stop) into <= nslab contiguous slabs of balanced
    lower-triangular cost (the role of pyscf.lib.prange_tril in
    pyscfad/cc/ccsd_t.py:145,158; the exact split does not change the result)."""
    if stop <= start:
        return []
    cost = lambda p: p * (p + 1) // 2  # noqa: E731
    total = cost(stop) - cost(start)
    out, p0 = [], start
    for s in range(1, nslab + 1):
        target = cost(start) + total * s / nslab
        p1 = p0 + 1
        while p1 < stop and cost(p1) < target:
            p1 += 1
        out.append((p0, p1))
        p0 = p1
        if p0 >= stop:
            break
    if out[-1][1] < stop:
        out[-1] = (out[-1][0], stop)
    return out


def blocked_vjp(call, L: dict, et_bar_kernel: float, na: int = 3, nb: int = 2):
    """The reference driver's slab loop (pyscfad/cc/ccsd_t.py:145-177) around a
    ccsd_t_energy_vjp-compatible ``call`` (the 25-argument C signature, numpy
    arrays); returns kernel-layout gradients."""
    vvop = L["vvop"]
    nvir, nocc = L["t1T"].shape
    ins = [np.ascontiguousarray(L[k]) for k in ("mo_energy", "t1T", "t2T", "vooo", "fvo")]
    bars = [np.zeros_like(x) for x in ins]
    vvop_bar = np.zeros_like(vvop)

    def contract(a0, a1, b0, b1, cache, cache_bar):
        call(*ins, et_bar_kernel, nocc, nvir, a0, a1, b0, b1, *cache, *bars, *cache_bar)

    for a0, a1 in reversed(slabs(0, nvir, na)):
        row_a = np.ascontiguousarray(vvop[a0:a1, :a1])
        row_a_bar = np.zeros_like(row_a)
        if a0 == 0:
            col_a, col_a_bar = row_a, row_a_bar
        else:
            col_a = np.ascontiguousarray(vvop[:a0, a0:a1])
            col_a_bar = np.zeros_like(col_a)
        contract(a0, a1, a0, a1, (row_a, col_a, row_a, col_a), (row_a_bar, col_a_bar, row_a_bar, col_a_bar))
        for b0, b1 in slabs(0, a0, nb):
            row_b = np.ascontiguousarray(vvop[b0:b1, :b1])
            row_b_bar = np.zeros_like(row_b)
            if b0 == 0:
                col_b, col_b_bar = row_b, row_b_bar
            else:
                col_b = np.ascontiguousarray(vvop[:b0, b0:b1])
                col_b_bar = np.zeros_like(col_b)
            contract(a0, a1, b0, b1, (row_a, col_a, row_b, col_b),
                     (row_a_bar, col_a_bar, row_b_bar, col_b_bar))
            vvop_bar[b0:b1, :b1] += row_b_bar
            if b0 != 0:
                vvop_bar[:b0, b0:b1] += col_b_bar
        vvop_bar[a0:a1, :a1] += row_a_bar
        if a0 != 0:
            vvop_bar[:a0, a0:a1] += col_a_bar
    out = dict(zip(("mo_energy", "t1T", "t2T", "vooo", "fvo"), bars))
    out["vvop"] = vvop_bar
    return out


def ref_call(*args):
    """ccsd_t_energy_vjp of the compiled reference with numpy/scalar arguments."""
    conv = []
    for i, a in enumerate(args):
        if isinstance(a, np.ndarray):
            conv.append(_p(a))
        elif i == 5:
            conv.append(ctypes.c_double(a))
        else:
            conv.append(ctypes.c_int(a))
    lib().ccsd_t_energy_vjp(*conv)


def to_pyscf_grads(g: dict, nocc: int, nvir: int):
    """Un-transpose kernel-layout gradients as pyscfad/cc/ccsd_t.py:179-191 does."""
    nmo = nocc + nvir
    t1_bar = np.asarray(g["t1T"].T)
    t2_bar = np.asarray(g["t2T"].transpose(3, 2, 0, 1))
    fock_bar = np.zeros((nmo, nmo))
    fock_bar[nocc:, :nocc] = g["fvo"]
    ovoo_bar = np.asarray(g["vooo"].transpose(1, 0, 3, 2))
    vvop_bar = g["vvop"]
    ovov_bar = np.asarray(vvop_bar[:, :, :, :nocc].transpose(2, 0, 3, 1))
    ovvv_bar = vvop_bar[:, :, :, nocc:].transpose(2, 0, 3, 1).copy()
    ovvv_bar += ovvv_bar.transpose(0, 1, 3, 2)
    idx, idy = np.diag_indices(nvir)
    ovvv_bar[:, :, idx, idy] *= .5
    idx, idy = np.tril_indices(nvir)
    ovvv_tril_bar = np.asarray(ovvv_bar[:, :, idx, idy])
    return dict(t1=t1_bar, t2=t2_bar, fock=fock_bar, mo_energy=g["mo_energy"],
                ovoo=ovoo_bar, ovov=ovov_bar, ovvv=ovvv_tril_bar)
