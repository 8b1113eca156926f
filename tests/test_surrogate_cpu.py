"""CPU: the surrogate's numpy oracle (gradients by finite differences, AdamW,
features) and the host-side job bookkeeping."""
import numpy as np

import golden_io
from oracle import ccsd_t_np as onp
from oracle import mlp_np
from pyscfad_b200 import surrogate, synth


def _params(seed=0, scale=0.3):
    g = np.random.default_rng(seed)
    return scale * g.standard_normal(mlp_np.NPARAM)


def test_param_layout_roundtrip():
    p = _params()
    assert len(p) == mlp_np.NPARAM == 18305
    np.testing.assert_array_equal(mlp_np.pack(*mlp_np.unpack(p)), p)


def test_backward_matches_finite_differences():
    g = np.random.default_rng(1)
    p = _params(1)
    X = g.standard_normal((7, mlp_np.NI))
    t = g.standard_normal(7)

    def loss(q):
        y, _, _ = mlp_np.forward(q, X)
        return mlp_np.mse(y, t)[0]

    y, z1, z2 = mlp_np.forward(p, X)
    _, dy = mlp_np.mse(y, t)
    grad = mlp_np.backward(p, X, z1, z2, dy)
    h = 1e-6
    for idx in list(g.choice(mlp_np.NPARAM, 40, replace=False)) + [mlp_np.NPARAM - 1, 0]:
        e = np.zeros_like(p)
        e[idx] = h
        fd = (loss(p + e) - loss(p - e)) / (2 * h)
        assert abs(fd - grad[idx]) <= 1e-6 * max(1.0, abs(fd)), (idx, fd, grad[idx])


def test_adam_first_step_is_signed_lr():
    p = _params(2)
    gr = np.linspace(-1, 1, mlp_np.NPARAM)
    gr[gr == 0] = 0.5
    q, m, v = mlp_np.adam(p, gr, np.zeros_like(p), np.zeros_like(p), 1, lr=1e-2, eps=0.0)
    np.testing.assert_allclose(p - q, 1e-2 * np.sign(gr), rtol=1e-12)


def test_features_by_definition():
    meta, _ = golden_io.load("small_o4v10_fvo")
    L = synth.reference_layouts(golden_io.system(meta))
    abc = surrogate.sorted_jobs(meta["nvir"])
    F = mlp_np.features(L, abc)
    assert F.shape == (len(abc), 12) and np.all(np.isfinite(F))
    # job (a, b, c) = (5, 3, 3): pairs (5,3), (5,3), (3,3); orbit size 3
    j = int(np.nonzero((abc[:, 0] == 5) & (abc[:, 1] == 3) & (abc[:, 2] == 3))[0][0])
    t2T, vvop, o = L["t2T"], L["vvop"], meta["nocc"]
    assert abs(F[j, 0] - np.log(np.linalg.norm(t2T[5, 3]))) < 1e-12
    assert F[j, 0] == F[j, 1]
    e2 = sum(t2T[5, 3, jj, i] * (2 * vvop[5, 3, i, jj] - vvop[3, 5, i, jj]) for i in range(o) for jj in range(o))
    assert abs(F[j, 3] - np.arcsinh(e2 * 1e4)) < 1e-9
    assert abs(F[j, 11] - np.log(3.0)) < 1e-15
    e = L["mo_energy"]
    assert abs(F[j, 9] - (e[o + 5] + 2 * e[o + 3] - 3 * e[:o].max())) < 1e-12


def test_sorted_jobs_order_matches_kernel_index():
    for v in (1, 2, 5, 13):
        abc = surrogate.sorted_jobs(v)
        assert len(abc) == v * (v + 1) * (v + 2) // 6
        np.testing.assert_array_equal(surrogate.amajor_index(abc), np.arange(len(abc)))
        assert np.all(abc[:, 0] >= abc[:, 1]) and np.all(abc[:, 1] >= abc[:, 2])
    np.testing.assert_array_equal(surrogate.sorted_jobs(4), onp.sorted_jobs(4)[np.argsort(
        surrogate.amajor_index(onp.sorted_jobs(4).astype(np.int32)))])


def test_pack_jobs():
    abc = np.array([[0, 0, 0], [1023, 5, 2], [7, 7, 7]])
    p = surrogate.pack_jobs(abc)
    np.testing.assert_array_equal(p & 1023, abc[:, 0])
    np.testing.assert_array_equal((p >> 10) & 1023, abc[:, 1])
    np.testing.assert_array_equal((p >> 20) & 1023, abc[:, 2])


def test_study_system_ranges():
    specs = surrogate.dataset_systems(range(100, 356))
    assert len(specs) == 256
    o = np.array([s[0] for s in specs])
    v = np.array([s[1] for s in specs])
    assert o.min() >= 6 and o.max() <= 24 and v.min() >= 40 and v.max() <= 200
    assert all(s[2] == 3 * s[1] for s in specs)
    assert len({s[3] for s in specs}) == 256
