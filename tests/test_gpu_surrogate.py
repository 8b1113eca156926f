"""GPU: the surrogate's kernels against the numpy oracle (features, forward,
gradients, AdamW, bf16 inference), the exact pass over a job list, and what the
trained network gains over screening without it.

Tolerances: float32 kernels vs the float64 oracle, 1e-4 relative (forward,
features) and 1e-3 relative to the gradient's norm (backward); bf16 inference
vs float32 forward, 3e-2 relative to the output spread.
"""
import ctypes

import numpy as np
import pytest
import torch

import golden_io
from oracle import mlp_np
from pyscfad_b200 import native, surrogate, synth, triples

pytestmark = pytest.mark.gpu


def dev_layouts(L, dev):
    return {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in L.items()}


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def test_features_match_oracle(cuda_dev):
    meta, _ = golden_io.load("cfg1_o8v40_fvo")
    Lh = synth.reference_layouts(golden_io.system(meta))
    abc = surrogate.sorted_jobs(meta["nvir"])
    F = surrogate.features(dev_layouts(Lh, cuda_dev), abc).cpu().numpy()
    Fo = mlp_np.features(Lh, abc)
    np.testing.assert_allclose(F, Fo, rtol=1e-4, atol=1e-4)


def test_forward_backward_adam_match_oracle(cuda_dev):
    g = np.random.default_rng(3)
    n = 1000                       # not a multiple of the 32-sample tile
    p = 0.2 * g.standard_normal(mlp_np.NPARAM)
    X = g.standard_normal((n, mlp_np.NI))
    t = g.standard_normal(n)
    model = surrogate.MLP(cuda_dev)
    model.params = torch.tensor(p, dtype=torch.float32, device=cuda_dev)
    Xd = torch.tensor(X, dtype=torch.float32, device=cuda_dev)
    Td = torch.tensor(t, dtype=torch.float32, device=cuda_dev)
    Y, Z1, Z2 = model.forward_raw(Xd, keep=True)
    y, z1, z2 = mlp_np.forward(p, X)
    np.testing.assert_allclose(Y.cpu().numpy(), y, rtol=1e-4, atol=1e-4 * np.abs(y).max())
    np.testing.assert_allclose(Z2.cpu().numpy(), z2, rtol=1e-4, atol=1e-4 * np.abs(z2).max())
    loss, grad = model.loss_grad_raw(Xd, Td)
    lo, dy = mlp_np.mse(y, t)
    go = mlp_np.backward(p, X, z1, z2, dy)
    assert abs(float(loss) - lo) <= 1e-4 * lo
    gd = grad.cpu().numpy()
    assert np.linalg.norm(gd - go) <= 1e-3 * np.linalg.norm(go)
    # deterministic: a second backward gives bit-identical gradients
    _, grad2 = model.loss_grad_raw(Xd, Td)
    assert torch.equal(grad, grad2)
    # AdamW step
    m = torch.zeros_like(model.params)
    v = torch.zeros_like(model.params)
    P0 = model.params.clone()
    native.check(native.lib().ct_mlp_adam(_ptr(model.params), _ptr(grad), _ptr(m), _ptr(v), 1, 1e-3, 0.9, 0.999,
                                          1e-8, 1e-4, None))
    po, _, _ = mlp_np.adam(P0.double().cpu().numpy(), gd.astype(np.float64), np.zeros(mlp_np.NPARAM),
                           np.zeros(mlp_np.NPARAM), 1, 1e-3, wd=1e-4)
    np.testing.assert_allclose(model.params.cpu().numpy(), po, rtol=1e-5, atol=1e-6)


def test_bf16_inference_close_to_f32(cuda_dev):
    g = np.random.default_rng(4)
    model = surrogate.MLP(cuda_dev, seed=1)
    F = torch.tensor(g.standard_normal((777, 12)), dtype=torch.float32, device=cuda_dev)
    model.t_mu, model.t_sd = 0.0, 1.0
    yb = torch.asinh(model.predict(F) / surrogate.E_SCALE)
    yf = torch.asinh(model.predict_f32(F) / surrogate.E_SCALE)
    spread = float(yf.max() - yf.min())
    assert float((yb - yf).abs().max()) <= 3e-2 * spread


def test_energy_on_jobs_matches_job_energies(cuda_dev):
    meta, _ = golden_io.load("cfg1_o8v40")
    L = dev_layouts(synth.reference_layouts(golden_io.system(meta)), cuda_dev)
    je = surrogate.exact_job_energies(L).cpu().numpy()
    assert abs(je.sum() - meta["e_t"]) <= 1e-10 * abs(meta["e_t"])
    abc = surrogate.sorted_jobs(meta["nvir"])
    g = np.random.default_rng(5)
    sel = np.sort(g.choice(len(abc), 1234, replace=False))
    e = float(surrogate.energy_on_jobs(L, abc[g.permutation(sel)]))
    assert abs(e - je[sel].sum()) <= 1e-11 * max(1.0, abs(je[sel].sum()))
    e_all = float(surrogate.energy_on_jobs(L, abc[::-1].copy()))
    assert abs(e_all - meta["e_t"]) <= 1e-10 * abs(meta["e_t"])
    with pytest.raises(native.CtError):
        surrogate.energy_on_jobs(L, np.array([[3, 4, 1]], dtype=np.int32))


def test_trained_surrogate_beats_screening_without_it(cuda_dev):
    """Train on 16 small systems, screen 4 held-out ones at 20% exact work:
    the network's ranking plus its estimate of the unscreened 80% is closer
    to the exact E(T) than the same exact work ranked by the MP2 heuristic
    with the rest either dropped or extrapolated from the heuristic scores."""
    specs = surrogate.dataset_systems(range(500, 520), o_range=(6, 12), v_range=(20, 40))
    train, test = specs[:16], specs[16:]
    F, E = surrogate.build_training_set(train, cuda_dev, per_system=None)
    model = surrogate.MLP(cuda_dev, seed=0).fit(F, E, epochs=40, batch=2048, lr=3e-3)
    assert model.history[-1] < 0.2 * model.history[0]
    err_s, err_drop, err_scaled = [], [], []
    for o, v, naux, s in test:
        L = synth.device_layouts(o, v, naux, s, device=cuda_dev)
        e = float(triples.energy(L))
        r = surrogate.screened_energy(L, model, 0.2)
        h = surrogate.screened_energy(L, None, 0.2)
        err_s.append(abs(r.e - e) / abs(e))
        err_drop.append(abs(h.e_exact_part - e) / abs(e))
        err_scaled.append(abs(h.e - e) / abs(e))
        assert r.kept == h.kept
    assert np.median(err_s) < 0.5 * np.median(err_drop), (err_s, err_drop)
    assert np.median(err_s) < np.median(err_scaled), (err_s, err_scaled)
