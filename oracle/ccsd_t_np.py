"""Oracle (test infrastructure): numpy restatement of pyscfad's CCSD(T)
energy and hand-written VJP, in the kernel layouts of the C driver.

Only tests, the smoke check and the benchmark's CPU-baseline leg use this
module; the product never does.

Layouts (pyscfad/cc/ccsd_t.py:88-106): t1T (v,o); t2T (v,v,o,o) = t2[i,j,a,b]
stored at [a,b,j,i]; vooo (v,o,o,o) = ovoo.transpose(1,0,3,2); vvop (v,v,o,nmo)
= [ovov | ovvv] transposed (1,3,0,2); fvo (v,o); mo_energy (nmo).

Arithmetic followed, per sorted job a>=b>=c (ccsd_t.c:6-72 job list):
  * P_xyz[p,q,r] = sum_f vvop[x,y,p,o+f] t2T[z,f,q,r] - sum_l vooo[x,p,q,l] t2T[z,y,l,r]
    and V_xyz[p,q,r] = vvop[x,y,p,q] t1T[z,r]/2 + t2T[y,x,p,q] fvo[z,r]/2
    (get_wv, ccsd_t.c:121-152);
  * w, v = sum over the six (x,y,z) orderings scattered through the permutation
    maps idx0..idx5 (get_wz, ccsd_t_vjp.c:9-40; _make_permute_indices ccsd_t.c:74-96);
  * z = r3(w + v) with weights (4,1,1,-2,-2,-2) (add_and_permute, ccsd_t.c:98-119);
  * d3 = fac/(e_i+e_j+e_k-e_a-e_b-e_c), fac 1/6, 1/2, 1 (get_d3, ccsd_t_vjp.c:42-53);
  * E(T) = 2 sum_jobs sum_ijk w z d3 (equals pyscfad/cc/ccsd_t_slow.py:68-125);
  * backward: ccsd_t_vjp.c:55-329 (z_bar, d3_bar, w_bar, v_bar, mo_energy_bar and the
    eris/amplitude bars of get_eris_amps_bar), with et_bar doubled as
    pyscfad/cc/ccsd_t.py:86 does.
"""
from __future__ import annotations

import numpy as np

# scatter transposes for w (w[idx_s(pqr)] += P_s[pqr]) and gather transposes
# for w_bar (Wbar_s[pqr] = w_bar[idx_s(pqr)]), without the leading job axis
SCATTER_T = [(0, 1, 2), (0, 2, 1), (1, 0, 2), (2, 0, 1), (1, 2, 0), (2, 1, 0)]
GATHER_T = [(0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)]


def sorted_jobs(nvir: int, a0: int = 0, a1: int | None = None):
    """All (a,b,c) with a>=b>=c and a0<=a<a1, in a-major order."""
    if a1 is None:
        a1 = nvir
    jobs = [(a, b, c) for a in range(a0, a1) for b in range(a + 1) for c in range(b + 1)]
    return np.asarray(jobs, dtype=np.int64).reshape(-1, 3)


def job_factor(jobs: np.ndarray) -> np.ndarray:
    a, b, c = jobs[:, 0], jobs[:, 1], jobs[:, 2]
    fac = np.ones(len(jobs))
    fac[(a == b) | (b == c)] = 0.5
    fac[a == c] = 1.0 / 6.0
    return fac


def _b(tr):
    return (0,) + tuple(t + 1 for t in tr)


def r3(y: np.ndarray) -> np.ndarray:
    return (4 * y + y.transpose(_b((1, 2, 0))) + y.transpose(_b((2, 0, 1)))
            - 2 * y.transpose(_b((2, 1, 0))) - 2 * y.transpose(_b((0, 2, 1)))
            - 2 * y.transpose(_b((1, 0, 2))))


def _orderings(jobs):
    a, b, c = jobs[:, 0], jobs[:, 1], jobs[:, 2]
    return [(a, b, c), (a, c, b), (b, a, c), (b, c, a), (c, a, b), (c, b, a)]


def _wv(L, jobs):
    o = L["t1T"].shape[1]
    t2T, vvop, vooo = L["t2T"], L["vvop"], L["vooo"]
    t1h, fvoh = 0.5 * L["t1T"], 0.5 * L["fvo"]
    nj = len(jobs)
    w = np.zeros((nj, o, o, o))
    v = np.zeros((nj, o, o, o))
    for s, (x, y, z) in enumerate(_orderings(jobs)):
        P = np.einsum("jpf,jfqr->jpqr", vvop[x, y, :, o:], t2T[z], optimize=True)
        P -= np.einsum("jpql,jlr->jpqr", vooo[x], t2T[z, y], optimize=True)
        V = np.einsum("jpq,jr->jpqr", vvop[x, y, :, :o], t1h[z])
        V += np.einsum("jpq,jr->jpqr", t2T[y, x], fvoh[z])
        w += P.transpose(_b(SCATTER_T[s]))
        v += V.transpose(_b(SCATTER_T[s]))
    return w, v


def _d3(L, jobs):
    o = L["t1T"].shape[1]
    e = L["mo_energy"]
    eo = e[:o]
    eijk = eo[:, None, None] + eo[None, :, None] + eo[None, None, :]
    eabc = e[o + jobs[:, 0]] + e[o + jobs[:, 1]] + e[o + jobs[:, 2]]
    fac = job_factor(jobs)
    return fac[:, None, None, None] / (eijk[None] - eabc[:, None, None, None]), fac


def job_energies(L, jobs: np.ndarray, chunk: int = 256) -> np.ndarray:
    """Per-job contributions; E(T) = sum of them (each already carries the 2)."""
    out = np.empty(len(jobs))
    for s in range(0, len(jobs), chunk):
        J = jobs[s:s + chunk]
        w, v = _wv(L, J)
        z = r3(w + v)
        d3, _ = _d3(L, J)
        out[s:s + chunk] = 2.0 * (w * z * d3).sum(axis=(1, 2, 3))
    return out


def energy(L, chunk: int = 256) -> float:
    nvir = L["t1T"].shape[0]
    e = job_energies(L, sorted_jobs(nvir), chunk)
    return float(np.sum(e))


def lno_axis_weights(jobs: np.ndarray, a0: int, a1: int, yz=None) -> np.ndarray:
    """Weights (njobs, 3) of the axis projections P_0, P_1, P_2 of a sorted
    job in the LNO energy restricted to first virtual index x in [a0, a1).

    lnoccsdt_contract (lno_ccsd_t.c:73-138) runs the ordered jobs (x, y, z)
    with y >= z, factor 1/2 when y == z, and projects the occupied index that
    pairs with x (lnoccsdt_get_energy, lno_ccsd_t.c:6-29: cache[i,j,k] =
    sum_l mat[l,i] w[l,j,k]).  On the sorted job's cubes (w, q = z/D indexed
    [p,q,r] for (a,b,c)) the ordering (x,y,z) is the projection on the axis
    that carries x:
      a>b>c:  (a,b,c) axis 0, (b,a,c) axis 1, (c,a,b) axis 2, factor 1 each;
      a>b=c:  (a,b,b) axis 0 x 1/2, (b,a,b) axis 1;
      a=b>c:  (a,a,c) axis 0, (c,a,a) axis 2 x 1/2;
      a=b=c:  (a,a,a) axis 0 x 1/2.
    (An ordering that differs only by exchanging equal values projects an
    axis with the same value as one listed, and w, q are symmetric under
    exchanging those axes.)"""
    a, b, c = jobs[:, 0], jobs[:, 1], jobs[:, 2]
    wt = np.zeros((len(jobs), 3))
    inr = lambda x: (x >= a0) & (x < a1)
    dis = (a > b) & (b > c)
    abc = (a > b) & (b == c)
    aab = (a == b) & (b > c)
    eq = (a == b) & (b == c)
    wt[:, 0] = np.where(inr(a), np.where(dis | aab, 1.0, 0.5), 0.0)
    wt[:, 1] = np.where(inr(b) & (dis | abc), 1.0, 0.0)
    wt[:, 2] = np.where(inr(c), np.where(dis, 1.0, np.where(aab, 0.5, 0.0)), 0.0)
    wt[eq, 1:] = 0.0
    if yz is not None:
        # slab block of the VJP driver (lno_ccsd_t_vjp.c:355-398): the ordering
        # whose first index sits on axis t has (y, z) = the other two values,
        # y >= z; it counts when y in [b0, b1) and z in [c0, c1)
        b0, b1, c0, c1 = yz
        ys = (b, a, a)
        zs = (c, c, b)
        for t in range(3):
            wt[:, t] *= ((ys[t] >= b0) & (ys[t] < b1) & (zs[t] >= c0) & (zs[t] < c1))
    return wt


def lno_job_energies(L, mat: np.ndarray, jobs: np.ndarray, a0: int = 0, a1: int | None = None,
                     chunk: int = 128) -> np.ndarray:
    """LNO energy per sorted job: sum_t weight_t P_t with
    P_0 = sum mat[l,p] w[l,q,r] q[p,q,r], P_1 = sum mat[l,q] w[p,l,r] q[p,q,r],
    P_2 = sum mat[l,r] w[p,q,l] q[p,q,r], q = r3(w + v) / D."""
    nvir = L["t1T"].shape[0]
    if a1 is None:
        a1 = nvir
    o = L["t1T"].shape[1]
    e = L["mo_energy"]
    eo = e[:o]
    eijk = eo[:, None, None] + eo[None, :, None] + eo[None, None, :]
    out = np.empty(len(jobs))
    for s in range(0, len(jobs), chunk):
        J = jobs[s:s + chunk]
        w, v = _wv(L, J)
        z = r3(w + v)
        eabc = e[o + J[:, 0]] + e[o + J[:, 1]] + e[o + J[:, 2]]
        q = z / (eijk[None] - eabc[:, None, None, None])
        P0 = np.einsum("lp,jlqr,jpqr->j", mat, w, q, optimize=True)
        P1 = np.einsum("lq,jplr,jpqr->j", mat, w, q, optimize=True)
        P2 = np.einsum("lr,jpql,jpqr->j", mat, w, q, optimize=True)
        wt = lno_axis_weights(J, a0, a1)
        out[s:s + chunk] = wt[:, 0] * P0 + wt[:, 1] * P1 + wt[:, 2] * P2
    return out


def lno_energy(L, mat: np.ndarray, a0: int = 0, a1: int | None = None) -> float:
    """lnoccsdt_contract's e_tot (without the driver's 2/3) for the slab
    a0 <= x < a1, summed over the sorted jobs that carry such an x."""
    nvir = L["t1T"].shape[0]
    if a1 is None:
        a1 = nvir
    jobs = sorted_jobs(nvir)
    sel = ((jobs >= a0) & (jobs < a1)).any(axis=1)
    return float(np.sum(lno_job_energies(L, mat, jobs[sel], a0, a1)))


def _lno_project(mat, w, wt):
    """A = sum_t wt_t M_t(w), M_0(w)[p,q,r] = sum_l mat[l,p] w[l,q,r] (axes 1, 2 alike)."""
    return (wt[:, 0, None, None, None] * np.einsum("lp,jlqr->jpqr", mat, w, optimize=True)
            + wt[:, 1, None, None, None] * np.einsum("lq,jplr->jpqr", mat, w, optimize=True)
            + wt[:, 2, None, None, None] * np.einsum("lr,jpql->jpqr", mat, w, optimize=True))


def _lno_project_t(mat, q, wt):
    """B = sum_t wt_t M_t^T(q), M_0^T(q)[l,q,r] = sum_p mat[l,p] q[p,q,r] (axes 1, 2 alike)."""
    return (wt[:, 0, None, None, None] * np.einsum("lp,jpqr->jlqr", mat, q, optimize=True)
            + wt[:, 1, None, None, None] * np.einsum("lq,jpqr->jplr", mat, q, optimize=True)
            + wt[:, 2, None, None, None] * np.einsum("lr,jpqr->jpql", mat, q, optimize=True))


def lno_energy_vjp(L, mat: np.ndarray, et_bar: float = 1.0, chunk: int = 128, block=None):
    """(E, mat_bar, grads) of lnoccsdt_energy_vjp over every LNO job, restated
    on sorted jobs.  With A = sum_t wt_t M_t(w), q = z/D and
    B = sum_t wt_t M_t^T(q), the energy is sum A q, and the backward is the
    canonical one (ccsd_t_vjp.c:55-137) with the elementwise products replaced:
    z_bar = eb A / D, w_bar = eb B + r3(z_bar), v_bar = r3(z_bar), and the
    mo_energy bar from tmp = eb A q / D (lno_ccsd_t_vjp.c:73-140);
    mat_bar[l,i] = eb sum_t wt_t sum w q over the other two axes
    (lno_ccsd_t_vjp.c:101-103).  eb = et_bar as passed (no doubling).
    ``block`` = (b0, b1, c0, c1) restricts to one block of the driver's slab
    loop (orderings with y in [b0, b1), z in [c0, c1))."""
    o = L["t1T"].shape[1]
    nvir = L["t1T"].shape[0]
    t2T, vvop, vooo = L["t2T"], L["vvop"], L["vooo"]
    t1h, fvoh = 0.5 * L["t1T"], 0.5 * L["fvo"]
    e = L["mo_energy"]
    eijk = e[:o][:, None, None] + e[:o][None, :, None] + e[:o][None, None, :]
    g = {k: np.zeros_like(val) for k, val in L.items()}
    mat_bar = np.zeros_like(mat)
    eb = et_bar
    jobs_all = sorted_jobs(nvir)
    etot = 0.0
    for s0 in range(0, len(jobs_all), chunk):
        jobs = jobs_all[s0:s0 + chunk]
        w, v = _wv(L, jobs)
        z = r3(w + v)
        D = eijk[None] - (e[o + jobs[:, 0]] + e[o + jobs[:, 1]] + e[o + jobs[:, 2]])[:, None, None, None]
        q = z / D
        wt = lno_axis_weights(jobs, 0, nvir, block)
        A = _lno_project(mat, w, wt)
        B = _lno_project_t(mat, q, wt)
        etot += float((A * q).sum())
        mat_bar += eb * (np.einsum("j,jlqr,jpqr->lp", wt[:, 0], w, q, optimize=True)
                         + np.einsum("j,jplr,jpqr->lq", wt[:, 1], w, q, optimize=True)
                         + np.einsum("j,jpql,jpqr->lr", wt[:, 2], w, q, optimize=True))
        zbar = eb * A / D
        ybar = r3(zbar)
        wbar = eb * B + ybar
        vbar = ybar
        tmp = eb * A * q / D
        occ = -(tmp.sum(axis=(2, 3)) + tmp.sum(axis=(1, 3)) + tmp.sum(axis=(1, 2)))
        np.add.at(g["mo_energy"], np.arange(o), occ.sum(axis=0))
        tt = tmp.sum(axis=(1, 2, 3))
        for col in range(3):
            np.add.at(g["mo_energy"], o + jobs[:, col], tt)
        for s, (x, yy, zz) in enumerate(_orderings(jobs)):
            Wb = wbar.transpose(_b(GATHER_T[s]))
            Vb = vbar.transpose(_b(GATHER_T[s]))
            np.add.at(g["vvop"][:, :, :, o:], (x, yy),
                      np.einsum("jfqr,jpqr->jpf", t2T[zz], Wb, optimize=True))
            np.add.at(g["vooo"], x, -np.einsum("jlr,jpqr->jpql", t2T[zz, yy], Wb, optimize=True))
            np.add.at(g["vvop"][:, :, :, :o], (x, yy), np.einsum("jpqr,jr->jpq", Vb, t1h[zz]))
            np.add.at(g["t1T"], zz, 0.5 * np.einsum("jpqr,jpq->jr", Vb, vvop[x, yy, :, :o]))
            np.add.at(g["t2T"], zz, np.einsum("jpqr,jpf->jfqr", Wb, vvop[x, yy, :, o:], optimize=True))
            np.add.at(g["t2T"], (zz, yy), -np.einsum("jpqr,jpql->jlr", Wb, vooo[x], optimize=True))
            np.add.at(g["t2T"], (yy, x), np.einsum("jpqr,jr->jpq", Vb, fvoh[zz]))
            np.add.at(g["fvo"], zz, 0.5 * np.einsum("jpqr,jpq->jr", Vb, t2T[yy, x]))
    return etot, mat_bar, g


def energy_vjp(L, et_bar: float = 1.0, chunk: int = 256):
    """Returns (E, grads) with grads in the kernel layouts (same keys as L)."""
    o = L["t1T"].shape[1]
    nvir = L["t1T"].shape[0]
    t2T, vvop, vooo = L["t2T"], L["vvop"], L["vooo"]
    t1h, fvoh = 0.5 * L["t1T"], 0.5 * L["fvo"]
    g = {k: np.zeros_like(val) for k, val in L.items()}
    eb = 2.0 * et_bar
    jobs_all = sorted_jobs(nvir)
    etot = 0.0
    for s0 in range(0, len(jobs_all), chunk):
        jobs = jobs_all[s0:s0 + chunk]
        w, v = _wv(L, jobs)
        y = w + v
        z = r3(y)
        d3, fac = _d3(L, jobs)
        etot += 2.0 * float((w * z * d3).sum())
        zbar = eb * w * d3
        d3bar = eb * w * z
        wbar = eb * z * d3
        ybar = r3(zbar)
        wbar += ybar
        vbar = ybar
        tmp = d3bar * d3 * d3 / fac[:, None, None, None]
        occ = -(tmp.sum(axis=(2, 3)) + tmp.sum(axis=(1, 3)) + tmp.sum(axis=(1, 2)))
        np.add.at(g["mo_energy"], np.arange(o), occ.sum(axis=0))
        tt = tmp.sum(axis=(1, 2, 3))
        for col in range(3):
            np.add.at(g["mo_energy"], o + jobs[:, col], tt)
        for s, (x, yy, zz) in enumerate(_orderings(jobs)):
            Wb = wbar.transpose(_b(GATHER_T[s]))
            Vb = vbar.transpose(_b(GATHER_T[s]))
            np.add.at(g["vvop"][:, :, :, o:], (x, yy),
                      np.einsum("jfqr,jpqr->jpf", t2T[zz], Wb, optimize=True))
            np.add.at(g["vooo"], x, -np.einsum("jlr,jpqr->jpql", t2T[zz, yy], Wb, optimize=True))
            np.add.at(g["vvop"][:, :, :, :o], (x, yy), np.einsum("jpqr,jr->jpq", Vb, t1h[zz]))
            np.add.at(g["t1T"], zz, 0.5 * np.einsum("jpqr,jpq->jr", Vb, vvop[x, yy, :, :o]))
            np.add.at(g["t2T"], zz, np.einsum("jpqr,jpf->jfqr", Wb, vvop[x, yy, :, o:], optimize=True))
            np.add.at(g["t2T"], (zz, yy), -np.einsum("jpqr,jpql->jlr", Wb, vooo[x], optimize=True))
            np.add.at(g["t2T"], (yy, x), np.einsum("jpqr,jr->jpq", Vb, fvoh[zz]))
            np.add.at(g["fvo"], zz, 0.5 * np.einsum("jpqr,jpq->jr", Vb, t2T[yy, x]))
    return etot, g


def energy_slow(t1, t2, mo_energy, ovov, ovoo, ovvv, fock) -> float:
    """Direct restatement of pyscfad/cc/ccsd_t_slow.py:29-125 (pyscf layouts),
    looping over a>=b>=c with symmetry factors 6/2/1; small systems only."""
    nocc, nvir = t1.shape
    e_occ, e_vir = mo_energy[:nocc], mo_energy[nocc:]
    eijk = e_occ[:, None, None] + e_occ[None, :, None] + e_occ[None, None, :]
    vvov = ovvv.transpose(1, 3, 0, 2)
    vooo = ovoo.transpose(1, 0, 3, 2)
    vvoo = ovov.transpose(1, 3, 0, 2)
    fvo = fock[nocc:, :nocc]
    t1T = t1.T
    t2T = t2.transpose(2, 3, 0, 1)

    def get_w(a, b, c):
        w = np.einsum("if,fkj->ijk", vvov[a, b], t2T[c, :])
        w -= np.einsum("ijm,mk->ijk", vooo[a, :], t2T[b, c])
        return w

    def get_v(a, b, c):
        return (np.einsum("ij,k->ijk", vvoo[a, b], t1T[c])
                + np.einsum("ij,k->ijk", t2T[a, b], fvo[c]))

    def r3s(w):
        return (4 * w + w.transpose(1, 2, 0) + w.transpose(2, 0, 1)
                - 2 * w.transpose(2, 1, 0) - 2 * w.transpose(0, 2, 1) - 2 * w.transpose(1, 0, 2))

    et = 0.0
    for a in range(nvir):
        for b in range(a + 1):
            for c in range(b + 1):
                fac = 6.0 if a == c else (2.0 if (a == b or b == c) else 1.0)
                d3 = (eijk - e_vir[a] - e_vir[b] - e_vir[c]) * fac
                WW = (get_w(a, b, c) + get_w(a, c, b).transpose(0, 2, 1)
                      + get_w(b, a, c).transpose(1, 0, 2) + get_w(b, c, a).transpose(2, 0, 1)
                      + get_w(c, a, b).transpose(1, 2, 0) + get_w(c, b, a).transpose(2, 1, 0))
                VV = (get_v(a, b, c) + get_v(a, c, b).transpose(0, 2, 1)
                      + get_v(b, a, c).transpose(1, 0, 2) + get_v(b, c, a).transpose(2, 0, 1)
                      + get_v(c, a, b).transpose(1, 2, 0) + get_v(c, b, a).transpose(2, 1, 0))
                ZZ = r3s(WW + .5 * VV) / d3
                et += float(np.einsum("ijk,ijk", WW, ZZ))
    return et * 2
