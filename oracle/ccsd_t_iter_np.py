"""Oracle (test infrastructure): numpy restatement of pyscfad's iterative (T)
solver on the full 6-D triples amplitudes, pyscfad/cc/ccsd_t_slow.py:128-293,
in its own layouts (pyscf's ovov/ovoo/ovvv, t1 (o,v), t2 (o,o,v,v); t3 and the
intermediates as [i,j,k,a,b,c]).  Only tests use this module.

Followed line by line:
  * get_w_6d (:139-146): w = einsum('abif,cfkj->ijkabc', vvov, t2T)
                           - einsum('aijm,bcmk->ijkabc', vooo, t2T);
  * get_v_6d (:149-158): v = (vvoo[ab,ij] t1T[c,k] + t2T[ab,ij] fvo[c,k]) / 2;
  * r3_6d (:161-164), get_d3 (:167-171), P3 (:174-176), P6 (:179-186);
  * update_amps (:188-208): t3 = (P6(w + v) + P3(fvv' t3) - P3(foo' t3)) / d3
    with fvv', foo' the Fock blocks with their diagonals zeroed (initial guess:
    no Fock terms);
  * energy (:210-220): sum t3 * r3_6d(P6(w) / d3) * d3 / 3;
  * the loop of _iter (:233-260) without DIIS (the reference only runs DIIS
    when the CC object carries one): converged when |dE| < tol and
    |t3_new - t3| < tolnormt.
For canonical orbitals (foo, fvv diagonal) the first update is the fixed
point and the energy is E(T) (tests/test_oracle.py checks it against the
compiled reference's energy); small systems only (o^3 v^3 doubles).
"""
from __future__ import annotations

import numpy as np


def get_w_6d(ovvv, ovoo, t2):
    vvov = ovvv.transpose(1, 3, 0, 2)
    vooo = ovoo.transpose(1, 0, 3, 2)
    t2T = t2.transpose(2, 3, 0, 1)
    w = np.einsum("abif,cfkj->ijkabc", vvov, t2T, optimize=True)
    w -= np.einsum("aijm,bcmk->ijkabc", vooo, t2T, optimize=True)
    return w


def get_v_6d(ovov, t1, t2, fock):
    nocc = t1.shape[0]
    vvoo = ovov.transpose(1, 3, 0, 2)
    fvo = fock[nocc:, :nocc]
    t1T = t1.T
    t2T = t2.transpose(2, 3, 0, 1)
    v = np.einsum("abij,ck->ijkabc", vvoo, t1T)
    v += np.einsum("abij,ck->ijkabc", t2T, fvo)
    return 0.5 * v


def r3_6d(w):
    return (4 * w + w.transpose(2, 0, 1, 3, 4, 5) + w.transpose(1, 2, 0, 3, 4, 5)
            - 2 * w.transpose(2, 1, 0, 3, 4, 5) - 2 * w.transpose(0, 2, 1, 3, 4, 5)
            - 2 * w.transpose(1, 0, 2, 3, 4, 5))


def get_d3(eia):
    return (eia[:, None, None, :, None, None] + eia[None, :, None, None, :, None]
            + eia[None, None, :, None, None, :])


def P3(w):
    return w + w.transpose(1, 0, 2, 4, 3, 5) + w.transpose(2, 1, 0, 5, 4, 3)


def P6(w):
    return (w + w.transpose(1, 0, 2, 4, 3, 5) + w.transpose(2, 1, 0, 5, 4, 3)
            + w.transpose(0, 2, 1, 3, 5, 4) + w.transpose(1, 2, 0, 4, 5, 3)
            + w.transpose(2, 0, 1, 5, 3, 4))


def _d3(mo_energy, nocc):
    eia = mo_energy[:nocc, None] - mo_energy[None, nocc:]
    return get_d3(eia)


def update_amps(t1, t2, t3, mo_energy, fock, ovov, ovoo, ovvv, initial_guess=False):
    nocc, nvir = t1.shape
    t3new = P6(get_w_6d(ovvv, ovoo, t2) + get_v_6d(ovov, t1, t2, fock))
    if not initial_guess:
        fvv = np.array(fock[nocc:, nocc:], copy=True)
        fvv[np.diag_indices(nvir)] = 0.0
        t3new += P3(np.einsum("ae,ijkebc->ijkabc", fvv, t3, optimize=True))
        foo = np.array(fock[:nocc, :nocc], copy=True)
        foo[np.diag_indices(nocc)] = 0.0
        t3new -= P3(np.einsum("im,mjkabc->ijkabc", foo, t3, optimize=True))
    return t3new / _d3(mo_energy, nocc)


def energy(t2, t3, mo_energy, ovoo, ovvv):
    nocc = t3.shape[0]
    d3 = _d3(mo_energy, nocc)
    w = P6(get_w_6d(ovvv, ovoo, t2)) / d3
    return float(np.einsum("ijkabc,ijkabc", t3, r3_6d(w) * d3) / 3.0)


def iterative_kernel(t1, t2, mo_energy, fock, ovov, ovoo, ovvv, max_cycle=50, tol=1e-8, tolnormt=1e-6):
    """(converged, E, t3, energies per cycle) of the iterative (T) solver."""
    t3 = update_amps(t1, t2, None, mo_energy, fock, ovov, ovoo, ovvv, initial_guess=True)
    et = energy(t2, t3, mo_energy, ovoo, ovvv)
    hist = [et]
    conv = False
    for _ in range(max_cycle):
        t3new = update_amps(t1, t2, t3, mo_energy, fock, ovov, ovoo, ovvv)
        normt = float(np.linalg.norm((t3new - t3).ravel()))
        t3 = t3new
        eold, et = et, energy(t2, t3, mo_energy, ovoo, ovvv)
        hist.append(et)
        if abs(et - eold) < tol and normt < tolnormt:
            conv = True
            break
    return conv, et, t3, hist
