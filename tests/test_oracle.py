"""CPU: the oracle against the golden fixtures of the reference's own kernels."""
import numpy as np
import pytest

import golden_io
from oracle import ccsd_t_np as onp
from oracle import ref
from pyscfad_b200 import synth

SMALL = ["tiny_o3v7", "small_o4v10_fvo", "edge_o2v3", "edge_o1v4", "mid_o6v17_fvo"]


@pytest.mark.parametrize("name", golden_io.names())
def test_generator_matches_fixture(name):
    meta, _ = golden_io.load(name)
    if meta["nvir"] > 60:
        pytest.skip("large systems are checked by the GPU tests (too slow for the CPU suite)")
    L = synth.reference_layouts(golden_io.system(meta))
    np.testing.assert_allclose(golden_io.checksum(L), meta["checksum"], rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("name", SMALL)
def test_numpy_oracle_energy_and_vjp(name):
    meta, arr = golden_io.load(name)
    L = synth.reference_layouts(golden_io.system(meta))
    e, g = onp.energy_vjp(L, 1.0)
    assert abs(e - meta["e_t"]) <= 1e-12 * max(1.0, abs(meta["e_t"]))
    for k in golden_io.KEYS:
        if f"grad_{k}" in arr:
            np.testing.assert_allclose(g[k], arr[f"grad_{k}"], rtol=1e-10, atol=1e-13)
        proj = [np.vdot(g[k], golden_io.direction(k, g[k].shape, meta["seed"], i))
                for i in range(meta["ndir"])]
        np.testing.assert_allclose(proj, arr[f"proj_{k}"], rtol=1e-9, atol=1e-12)


def test_numpy_oracle_cfg1_energy():
    meta, _ = golden_io.load("cfg1_o8v40")
    L = synth.reference_layouts(golden_io.system(meta))
    e = onp.energy(L)
    assert abs(e - meta["e_t"]) < 1e-10


def test_slow_formula_matches_reference():
    """ccsd_t_slow (pyscf layouts, symmetry factors 6/2/1) equals the C path."""
    meta, _ = golden_io.load("small_o4v10_fvo")
    s = golden_io.system(meta)
    e = onp.energy_slow(s.t1, s.t2, s.mo_energy, s.ovov, s.ovoo, s.ovvv, s.fock)
    assert abs(e - meta["e_t"]) < 1e-13


def test_job_energies_sum():
    meta, _ = golden_io.load("tiny_o3v7")
    L = synth.reference_layouts(golden_io.system(meta))
    jobs = onp.sorted_jobs(meta["nvir"])
    je = onp.job_energies(L, jobs)
    assert len(je) == meta["nvir"] * (meta["nvir"] + 1) * (meta["nvir"] + 2) // 6
    assert abs(je.sum() - meta["e_t"]) < 1e-14


@pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("name", ["tiny_o3v7", "small_o4v10_fvo", "edge_o1v4"])
def test_compiled_reference_reproduces_fixture(name):
    meta, arr = golden_io.load(name)
    L = synth.reference_layouts(golden_io.system(meta))
    assert abs(ref.energy(**L) - meta["e_t"]) <= 1e-13 * max(1.0, abs(meta["e_t"]))
    g = ref.energy_vjp_layouts(**L, et_bar=1.0)
    for k in golden_io.KEYS:
        np.testing.assert_allclose(g[k], arr[f"grad_{k}"], rtol=1e-11, atol=1e-14)


@pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("na,nb", [(3, 2), (4, 3)])
def test_reference_blocked_driver_matches_fixture(na, nb):
    """The driver's slab loop over (a0,a1,b0,b1) blocks reproduces the full VJP."""
    meta, arr = golden_io.load("small_o4v10_fvo")
    L = synth.reference_layouts(golden_io.system(meta))
    g = ref.blocked_vjp(ref.ref_call, L, 2.0, na, nb)
    for k in golden_io.KEYS:
        np.testing.assert_allclose(g[k], arr[f"grad_{k}"], rtol=1e-11, atol=1e-14)


def test_slabs_partition():
    for n, k in [(10, 3), (40, 5), (7, 7), (3, 5)]:
        s = ref.slabs(0, n, k)
        assert s[0][0] == 0 and s[-1][1] == n
        assert all(s[i][1] == s[i + 1][0] for i in range(len(s) - 1))
        assert all(p1 > p0 for p0, p1 in s)


def test_fvo_path_changes_energy():
    base = synth.make_system(4, 10, 30, 7, fvo_sigma=0.0)
    pert = synth.make_system(4, 10, 30, 7, fvo_sigma=1e-2)
    e0 = onp.energy(synth.reference_layouts(base))
    e1 = onp.energy(synth.reference_layouts(pert))
    assert e0 != e1


@pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("name", ["tiny_o3v7", "small_o4v10_fvo", "cfg1_o8v40"])
def test_lno_decomposition_matches_reference(name):
    """The LNO-projected energy with a general projector, restated on sorted
    jobs (three axis projections per job), against the compiled reference's
    lnoccsdt_contract over the full range and partial a-slabs."""
    meta, _ = golden_io.load(name)
    L = synth.reference_layouts(golden_io.system(meta))
    o, v = meta["nocc"], meta["nvir"]
    mat = np.random.default_rng(7).standard_normal((o, o))
    for a0, a1 in [(0, v), (0, 1), (v // 3, v // 2 + 1), (v - 1, v)]:
        er = ref.lno_contract(mat, **L, a0=a0, a1=a1)
        en = onp.lno_energy(L, mat, a0, a1)
        assert abs(er - en) <= 1e-12 * abs(er), (a0, a1, er, en)
    # mat = I gives 3/2 of the canonical energy
    assert abs(ref.lno_contract(np.eye(o), **L) - 1.5 * meta["e_t"]) <= 1e-12 * abs(meta["e_t"])


def test_lno_axis_weights_by_case():
    jobs = np.array([[5, 3, 1], [5, 3, 3], [5, 5, 1], [4, 4, 4]])
    w = onp.lno_axis_weights(jobs, 0, 10)
    np.testing.assert_array_equal(w, [[1, 1, 1], [0.5, 1, 0], [1, 0, 0.5], [0.5, 0, 0]])
    # slab restriction: only orderings whose first index lies in [a0, a1)
    np.testing.assert_array_equal(onp.lno_axis_weights(jobs, 3, 4), [[0, 1, 0], [0, 1, 0], [0, 0, 0], [0, 0, 0]])


@pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("name", ["tiny_o3v7", "edge_o2v3", "small_o4v10_fvo"])
def test_lno_vjp_decomposition_matches_reference(name):
    """The LNO VJP restated on sorted jobs (projected cubes A, B; canonical
    backward with z_bar = eb A/D, w_bar = eb B + r3(z_bar)) against the
    compiled lnoccsdt_energy_vjp over every LNO job."""
    meta, _ = golden_io.load(name)
    L = synth.reference_layouts(golden_io.system(meta))
    o = meta["nocc"]
    mat = np.random.default_rng(5).standard_normal((o, o))
    mb_r, g_r = ref.lno_energy_vjp(mat, **L, et_bar=0.7)
    e, mb, g = onp.lno_energy_vjp(L, mat, 0.7)
    assert abs(e - ref.lno_contract(mat, **L)) <= 1e-13 * abs(e)
    assert np.linalg.norm(mb - mb_r) <= 1e-12 * np.linalg.norm(mb_r)
    for k in golden_io.KEYS:
        assert np.linalg.norm(g[k] - g_r[k]) <= 1e-12 * np.linalg.norm(g_r[k]) + 1e-300, k


@pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("blk", [(7, 10, 7, 10), (7, 10, 0, 7), (3, 6, 0, 2), (2, 5, 2, 5)])
def test_lno_vjp_block_decomposition_matches_reference(blk):
    """One block of the LNO backward's slab loop: orderings with y in [b0,b1),
    z in [c0,c1), against the compiled kernel on the driver's caches."""
    meta, _ = golden_io.load("small_o4v10_fvo")
    L = synth.reference_layouts(golden_io.system(meta))
    o = meta["nocc"]
    mat = np.random.default_rng(5).standard_normal((o, o))
    mb_r, g_r = ref.lno_energy_vjp_block(mat, **L, et_bar=0.7, b0=blk[0], b1=blk[1], c0=blk[2], c1=blk[3])
    _, mb, g = onp.lno_energy_vjp(L, mat, 0.7, block=blk)
    assert np.linalg.norm(mb - mb_r) <= 1e-12 * np.linalg.norm(mb_r)
    for k in golden_io.KEYS:
        assert np.linalg.norm(g[k] - g_r[k]) <= 1e-12 * np.linalg.norm(g_r[k]) + 1e-300, k


@pytest.mark.parametrize("v,bufsize", [(10, 4), (17, 8), (23, 5)])
def test_lno_block_weights_partition_the_full_range(v, bufsize):
    """The LNO backward's slab loop (pyscfad/lno/ccsd_t.py:193-220: diagonal
    blocks over prange(0, v, bufsize) and the blocks below them in steps of
    bufsize//4) covers every ordering exactly once: per sorted job, the block
    weights sum to the full-range weights."""
    jobs = onp.sorted_jobs(v)
    full = onp.lno_axis_weights(jobs, 0, v)
    tot = np.zeros_like(full)
    step = max(1, bufsize // 4)
    for a0 in range(0, v, bufsize):
        a1 = min(v, a0 + bufsize)
        tot += onp.lno_axis_weights(jobs, 0, v, (a0, a1, a0, a1))
        for b0 in range(0, a0, step):
            tot += onp.lno_axis_weights(jobs, 0, v, (a0, a1, b0, min(a0, b0 + step)))
    np.testing.assert_array_equal(tot, full)


def test_lno_kernel_fiber_indexing():
    """The fiber addressing of the LNO projection kernels (ct_fp64.cu:
    fiber f = (f0, f1) of the two fixed indices; base = f, f0*o^2 + f1 or
    f*o and stride o^2, o or 1 for axes 0, 1, 2), restated: every element of
    the cube is visited once per axis, and the fiber sums reproduce the
    projections P_t and the cubes A = M_t(w), B = M_t^T(q)."""
    o = 5
    g = np.random.default_rng(8)
    w = g.standard_normal((o, o, o))
    q = g.standard_normal((o, o, o))
    mat = g.standard_normal((o, o))
    W, Q = w.ravel(), q.ravel()
    for t in range(3):
        st = (o * o, o, 1)[t]
        seen = np.zeros(o ** 3, dtype=int)
        P = 0.0
        A = np.zeros(o ** 3)
        B = np.zeros(o ** 3)
        for f in range(o * o):
            f0, f1 = divmod(f, o)
            base = (f, f0 * o * o + f1, f * o)[t]
            idx = base + st * np.arange(o)
            seen[idx] += 1
            P += W[idx] @ (mat @ Q[idx])                 # sum_l w[l] sum_k mat[l,k] q[k]
            A[idx] += mat.T @ W[idx]                     # A[k] = sum_l mat[l,k] w[l]
            B[idx] += mat @ Q[idx]                       # B[k] = sum_l mat[k,l] q[l]
        assert np.all(seen == 1)
        sub = ("lp,lqr,pqr->", "lq,plr,pqr->", "lr,pql,pqr->")[t]
        np.testing.assert_allclose(P, np.einsum(sub, mat, w, q), rtol=1e-12)
        wt = np.zeros((1, 3))
        wt[0, t] = 1.0
        np.testing.assert_allclose(A.reshape(o, o, o), onp._lno_project(mat, w[None], wt)[0], rtol=1e-12,
                                   atol=1e-14)
        np.testing.assert_allclose(B.reshape(o, o, o), onp._lno_project_t(mat, q[None], wt)[0], rtol=1e-12,
                                   atol=1e-14)


def _perturbed_fock(s, scale, seed):
    """s.fock with small symmetric off-diagonal occupied-occupied and
    virtual-virtual blocks (non-canonical orbitals: the iterative solver then
    needs several cycles)."""
    import dataclasses
    rng = np.random.default_rng(seed)
    o, n = s.nocc, s.nocc + s.nvir
    f = np.array(s.fock, copy=True)
    for lo, hi in ((0, o), (o, n)):
        x = rng.standard_normal((hi - lo, hi - lo)) * scale
        x = 0.5 * (x + x.T)
        np.fill_diagonal(x, 0.0)
        f[lo:hi, lo:hi] += x
    return dataclasses.replace(s, fock=f)


@pytest.mark.parametrize("name", ["tiny_o3v7", "small_o4v10_fvo"])
def test_iterative_oracle_canonical_is_e_t(name):
    """The 6-D iterative restatement (ccsd_t_slow.py:128-293) converges in one
    cycle for canonical orbitals to E(T), which the fixtures hold from the
    compiled reference."""
    from oracle import ccsd_t_iter_np as it
    meta, _ = golden_io.load(name)
    s = golden_io.system(meta)
    conv, e, _, hist = it.iterative_kernel(s.t1, s.t2, s.mo_energy, s.fock, s.ovov, s.ovoo, s.ovvv)
    assert conv and len(hist) == 2
    assert abs(e - meta["e_t"]) <= 1e-12 * abs(meta["e_t"])


def test_iterative_oracle_noncanonical_fixed_point():
    """With off-diagonal Fock blocks the solver iterates to a t3 that its own
    update maps to itself, and the energy moves away from E(T)."""
    from oracle import ccsd_t_iter_np as it
    meta, _ = golden_io.load("small_o4v10_fvo")
    s = _perturbed_fock(golden_io.system(meta), 0.05, 5)
    conv, e, t3, hist = it.iterative_kernel(s.t1, s.t2, s.mo_energy, s.fock, s.ovov, s.ovoo, s.ovvv, tol=1e-12,
                                            tolnormt=1e-11)
    assert conv and len(hist) > 3
    t3n = it.update_amps(s.t1, s.t2, t3, s.mo_energy, s.fock, s.ovov, s.ovoo, s.ovvv)
    assert np.abs(t3n - t3).max() <= 1e-10 * np.abs(t3).max()
    assert abs(e - meta["e_t"]) > 1e-6 * abs(meta["e_t"])
