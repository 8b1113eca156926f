"""Learned block surrogate for screened (T) passes.

A block is one sorted virtual triple (a >= b >= c): the unit of work of the
(T) kernels, whose exact contribution ``triples.energy(..., job_e=...)``
reports per job.  A 12-128-128-1 SiLU MLP (float32 weights, bf16 inference)
maps 12 cheap features of a block (t2 block norms, MP2 pair energies, vvov
block norms of its three virtual pairs; minimum and mean orbital-energy gaps;
its orbit size) to its (T) contribution.  Everything runs on the GPU through
the library's own kernels (csrc/mlp.cu): features, forward, loss, backward,
AdamW and bf16 inference; torch only holds the device buffers.

Screened pass: predict every block, compute the blocks with the largest
predicted |contribution| exactly (``ct_energy_jobs``) and add the predictions
of the rest.  The exact kernel remains the arbiter: ``screened_energy``
returns the exact and predicted parts separately.

The reference has no learned component; this module has no counterpart there.
"""
from __future__ import annotations

import ctypes
import dataclasses
import math
import time

import numpy as np
import torch

from . import native, synth, triples

E_SCALE = 1e-3          # target transform: t = asinh(E_job / E_SCALE)


# ---------------------------------------------------------------- job lists
def sorted_jobs(nvir: int) -> np.ndarray:
    """All (a, b, c), nvir > a >= b >= c >= 0, in a-major order: row J is the
    job whose energy the kernels store at index a(a+1)(a+2)/6 + b(b+1)/2 + c."""
    a = np.repeat(np.arange(nvir), [(x + 1) * (x + 2) // 2 for x in range(nvir)])
    b = np.concatenate([np.repeat(np.arange(x + 1), np.arange(x + 1) + 1) for x in range(nvir)])
    c = np.concatenate([np.arange(y + 1) for x in range(nvir) for y in range(x + 1)])
    return np.stack([a, b, c], axis=1).astype(np.int32)


def amajor_index(abc: np.ndarray) -> np.ndarray:
    a, b, c = (abc[:, q].astype(np.int64) for q in range(3))
    return a * (a + 1) * (a + 2) // 6 + b * (b + 1) // 2 + c


def pack_jobs(abc: np.ndarray) -> np.ndarray:
    abc = np.asarray(abc, dtype=np.int64)
    return (abc[:, 0] | (abc[:, 1] << 10) | (abc[:, 2] << 20)).astype(np.int32)


# ---------------------------------------------------------------- kernels
def _ptr(t: torch.Tensor) -> ctypes.c_void_p:
    return ctypes.c_void_p(t.data_ptr())


def _stream(dev) -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)


def features(L: dict, jobs_abc: np.ndarray | None = None) -> torch.Tensor:
    """(njobs, 12) float32 device features of ``jobs_abc`` (all sorted jobs
    when None) of the device layouts L."""
    nocc, nvir, dev = triples._check_layouts(L)
    if jobs_abc is None:
        jobs_abc = sorted_jobs(nvir)
    packed = torch.from_numpy(pack_jobs(jobs_abc)).to(dev)
    n = packed.numel()
    F = torch.empty((n, native.MLP_IN), dtype=torch.float32, device=dev)
    work = torch.empty(3 * nvir * nvir, dtype=torch.float32, device=dev)
    prob = triples._problem(L, nocc, nvir)
    with torch.cuda.device(dev):
        st = native.lib().ct_surrogate_features(ctypes.byref(prob), _ptr(packed), n, _ptr(work), _ptr(F),
                                                _stream(dev))
    native.check(st, "ct_surrogate_features")
    return F


def exact_job_energies(L: dict, mode="fp64") -> torch.Tensor:
    """Exact per-job contributions (float64, a-major sorted order)."""
    _, nvir, dev = triples._check_layouts(L)
    je = torch.empty(nvir * (nvir + 1) * (nvir + 2) // 6, dtype=torch.float64, device=dev)
    triples.energy(L, mode=mode, job_e=je)
    return je


def energy_on_jobs(L: dict, jobs_abc: np.ndarray, mode="fp64") -> torch.Tensor:
    """Exact E(T) restricted to the listed jobs (0-d float64 device tensor)."""
    nocc, nvir, dev = triples._check_layouts(L)
    abc = np.ascontiguousarray(np.asarray(jobs_abc, dtype=np.int32))
    out = torch.empty((), dtype=torch.float64, device=dev)
    prob = triples._problem(L, nocc, nvir)
    with torch.cuda.device(dev):
        st = native.lib().ct_energy_jobs(ctypes.byref(prob), native.mode_id(mode),
                                         abc.ctypes.data_as(ctypes.c_void_p), len(abc), _ptr(out), None,
                                         _stream(dev))
    native.check(st, "ct_energy_jobs")
    return out


# ---------------------------------------------------------------- model
class MLP:
    """12-128-128-1 SiLU MLP whose training and inference run on the
    library's kernels.  Inputs are standardised features; the target is the
    standardised asinh(E_job / E_SCALE)."""

    def __init__(self, device, seed: int = 0):
        self.dev = torch.device(device)
        g = np.random.default_rng(seed)
        H, I = native.MLP_HIDDEN, native.MLP_IN
        W1 = g.standard_normal((H, I)) * math.sqrt(2.0 / I)
        W2 = g.standard_normal((H, H)) * math.sqrt(2.0 / H)
        W3 = g.standard_normal(H) * math.sqrt(1.0 / H)
        p = np.concatenate([W1.ravel(), np.zeros(H), W2.ravel(), np.zeros(H), W3, [0.0]])
        self.params = torch.tensor(p, dtype=torch.float32, device=self.dev)
        self.x_mu = torch.zeros(I, device=self.dev)
        self.x_sd = torch.ones(I, device=self.dev)
        self.t_mu, self.t_sd = 0.0, 1.0
        self._bf16 = None
        self.history: list[float] = []

    # -- transforms
    def _x(self, F: torch.Tensor) -> torch.Tensor:
        return ((F - self.x_mu) / self.x_sd).contiguous()

    def _t(self, E: torch.Tensor) -> torch.Tensor:
        return ((torch.asinh(E / E_SCALE) - self.t_mu) / self.t_sd).float().contiguous()

    def _e(self, y: torch.Tensor) -> torch.Tensor:
        return E_SCALE * torch.sinh(y.double() * self.t_sd + self.t_mu)

    # -- raw kernel calls (float32 standardised space)
    def forward_raw(self, X: torch.Tensor, keep: bool = False):
        n = X.shape[0]
        Y = torch.empty(n, dtype=torch.float32, device=self.dev)
        Z1 = Z2 = None
        if keep:
            Z1 = torch.empty((n, native.MLP_HIDDEN), dtype=torch.float32, device=self.dev)
            Z2 = torch.empty_like(Z1)
        L = native.lib()
        native.check(L.ct_mlp_forward(_ptr(self.params), _ptr(X), n, _ptr(Z1) if keep else None,
                                      _ptr(Z2) if keep else None, _ptr(Y), _stream(self.dev)), "ct_mlp_forward")
        return Y, Z1, Z2

    def loss_grad_raw(self, X: torch.Tensor, T: torch.Tensor):
        """(loss, grad) of the mean squared error on one batch."""
        n = X.shape[0]
        L = native.lib()
        Y, Z1, Z2 = self.forward_raw(X, keep=True)
        dY = torch.empty_like(Y)
        loss = torch.empty((), dtype=torch.float64, device=self.dev)
        native.check(L.ct_mlp_mse(_ptr(Y), _ptr(T), n, _ptr(dY), _ptr(loss), _stream(self.dev)), "ct_mlp_mse")
        grad = torch.empty_like(self.params)
        work = torch.empty(L.ct_mlp_work_floats(n), dtype=torch.float32, device=self.dev)
        native.check(L.ct_mlp_backward(_ptr(self.params), _ptr(X), _ptr(Z1), _ptr(Z2), _ptr(dY), n, _ptr(grad),
                                       _ptr(work), _stream(self.dev)), "ct_mlp_backward")
        return loss, grad

    def fit(self, F: torch.Tensor, E: torch.Tensor, epochs: int = 30, batch: int = 4096, lr: float = 2e-3,
            weight_decay: float = 1e-5, seed: int = 0, verbose: bool = False):
        """Trains on features F (n, 12) and exact job energies E (n,)."""
        F = F.to(self.dev, torch.float32)
        E = E.to(self.dev, torch.float64)
        self.x_mu = F.mean(0)
        self.x_sd = F.std(0).clamp_min(1e-6)
        t = torch.asinh(E / E_SCALE)
        self.t_mu, self.t_sd = float(t.mean()), max(float(t.std()), 1e-6)
        X, T = self._x(F), self._t(E)
        n = X.shape[0]
        m = torch.zeros_like(self.params)
        v = torch.zeros_like(self.params)
        gen = torch.Generator(device=self.dev)
        gen.manual_seed(seed)
        steps_per_epoch = max(1, n // batch)
        total = epochs * steps_per_epoch
        L = native.lib()
        step = 0
        for ep in range(epochs):
            perm = torch.randperm(n, device=self.dev, generator=gen)
            ep_loss = torch.zeros((), dtype=torch.float64, device=self.dev)
            for s in range(steps_per_epoch):
                idx = perm[s * batch:(s + 1) * batch]
                loss, grad = self.loss_grad_raw(X[idx].contiguous(), T[idx].contiguous())
                ep_loss += loss
                step += 1
                lr_t = lr * 0.5 * (1.0 + math.cos(math.pi * (step - 1) / total))
                native.check(L.ct_mlp_adam(_ptr(self.params), _ptr(grad), _ptr(m), _ptr(v), step, lr_t, 0.9, 0.999,
                                           1e-8, weight_decay, _stream(self.dev)), "ct_mlp_adam")
            self.history.append(float(ep_loss) / steps_per_epoch)
            if verbose:
                print(f"epoch {ep}: loss {self.history[-1]:.4e}", flush=True)
        self._bf16 = None
        return self

    def predict(self, F: torch.Tensor) -> torch.Tensor:
        """Predicted job energies (float64) with bf16 inference."""
        L = native.lib()
        if self._bf16 is None:
            self._bf16 = torch.empty(native.MLP_NPARAM, dtype=torch.bfloat16, device=self.dev)
            native.check(L.ct_mlp_to_bf16(_ptr(self.params), _ptr(self._bf16), _stream(self.dev)), "ct_mlp_to_bf16")
        X = self._x(F.to(self.dev, torch.float32))
        Y = torch.empty(X.shape[0], dtype=torch.float32, device=self.dev)
        native.check(L.ct_mlp_infer_bf16(_ptr(self._bf16), _ptr(X), X.shape[0], _ptr(Y), _stream(self.dev)),
                     "ct_mlp_infer_bf16")
        return self._e(Y)

    def predict_f32(self, F: torch.Tensor) -> torch.Tensor:
        Y, _, _ = self.forward_raw(self._x(F.to(self.dev, torch.float32)))
        return self._e(Y)


# ---------------------------------------------------------------- screening
def heuristic_score(F: torch.Tensor) -> torch.Tensor:
    """The method without the network: orbit size x sum of the |MP2 pair
    energies| of the job's three pairs / its mean denominator."""
    e2 = torch.sinh(F[:, 3:6].double()).abs() * 1e-4
    return torch.exp(F[:, 11].double()) * e2.sum(1) / F[:, 10].double().clamp_min(1e-3)


@dataclasses.dataclass
class ScreenResult:
    e: float                 # screened estimate
    e_exact_part: float      # exact energy of the kept jobs
    e_rest: float            # estimate of the dropped jobs (0 when dropped)
    kept: int
    njobs: int
    ms: float                # device time of the screened pass (features + inference + exact pass)


def screened_energy(L: dict, model: MLP | None, frac: float, mode="fp64", fill_rest: bool = True,
                    F: torch.Tensor | None = None) -> ScreenResult:
    """Exact energy of the top ``frac`` of jobs ranked by the model's
    |prediction| (or, with model None, by ``heuristic_score``), plus an
    estimate of the rest when ``fill_rest``: the model's predictions, or
    without a model the heuristic scores scaled by the kept jobs'
    exact-to-heuristic ratio."""
    _, nvir, dev = triples._check_layouts(L)
    abc = sorted_jobs(nvir)
    n = len(abc)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    ev0.record()
    if F is None:
        F = features(L, abc)
    score = model.predict(F) if model is not None else heuristic_score(F)
    k = max(1, min(n, int(math.ceil(frac * n))))
    order = torch.argsort(score.abs(), descending=True)
    keep = order[:k]
    keep_host = keep.cpu().numpy()
    ex = energy_on_jobs(L, abc[keep_host], mode=mode)
    rest = 0.0
    rest_t = None
    if fill_rest and k < n:
        if model is not None:
            rest_t = score[order[k:]].sum()
        else:
            # E(T) contributions are negative; the heuristic scores are magnitudes
            rest_t = ex * score[order[k:]].sum() / score[keep].sum().clamp_min(1e-300)
    ev1.record()
    torch.cuda.synchronize(dev)
    if rest_t is not None:
        rest = float(rest_t)
    e_ex = float(ex)
    return ScreenResult(e=e_ex + rest, e_exact_part=e_ex, e_rest=rest, kept=k, njobs=n, ms=ev0.elapsed_time(ev1))


# ---------------------------------------------------------------- data sets
def dataset_systems(seeds, o_range=(6, 24), v_range=(40, 200), naux_per_v: int = 3):
    """(nocc, nvir, naux, seed) of the surrogate study systems: nocc and nvir
    drawn uniformly (inclusive) from each seed's own generator."""
    out = []
    for s in seeds:
        g = np.random.default_rng([int(s), 777])
        o = int(g.integers(o_range[0], o_range[1] + 1))
        v = int(g.integers(v_range[0], v_range[1] + 1))
        out.append((o, v, naux_per_v * v, int(s)))
    return out


def system_data(spec, device, per_system: int | None = None, seed: int = 0, mode="fp64"):
    """(features, exact job energies, E(T)) of one system; ``per_system``
    subsamples the jobs (seeded)."""
    o, v, naux, s = spec
    L = synth.device_layouts(o, v, naux, s, device=device)
    je = exact_job_energies(L, mode=mode)
    F = features(L)
    e_tot = float(je.sum())
    if per_system is not None and per_system < je.numel():
        g = torch.Generator(device=device)
        g.manual_seed(seed * 1000003 + s)
        idx = torch.randperm(je.numel(), device=device, generator=g)[:per_system]
        F, je = F[idx], je[idx]
    del L
    return F, je, e_tot


def build_training_set(specs, device, per_system: int | None = 20000, mode="fp64"):
    Fs, Es = [], []
    for spec in specs:
        F, je, _ = system_data(spec, device, per_system=per_system, mode=mode)
        Fs.append(F)
        Es.append(je)
    return torch.cat(Fs), torch.cat(Es)


def study(n_train: int = 192, n_test: int = 64, first_seed: int = 100, per_system: int = 20000,
          fracs=(0.05, 0.1, 0.2, 0.3, 0.5), epochs: int = 30, device="cuda", verbose: bool = False) -> dict:
    """Trains on ``n_train`` systems, evaluates screened passes on ``n_test``
    held-out systems; returns per-fraction errors (relative to the exact E(T))
    and the screened/exact device time ratio."""
    dev = torch.device(device)
    specs = dataset_systems(range(first_seed, first_seed + n_train + n_test))
    tr, te = specs[:n_train], specs[n_train:]
    t0 = time.time()
    F, E = build_training_set(tr, dev, per_system=per_system)
    t_data = time.time() - t0
    t0 = time.time()
    model = MLP(dev, seed=0).fit(F, E, epochs=epochs, verbose=verbose)
    torch.cuda.synchronize(dev)
    t_train = time.time() - t0
    del F, E
    res = {f: {"surrogate": [], "heuristic_drop": [], "heuristic_scaled": [], "surrogate_drop": [], "speedup": []}
           for f in fracs}
    pred_err = []
    for spec in te:
        o, v, naux, s = spec
        L = synth.device_layouts(o, v, naux, s, device=dev)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        ev0.record()
        e_exact = float(triples.energy(L, mode="fp64"))
        ev1.record()
        torch.cuda.synchronize(dev)
        t_exact = ev0.elapsed_time(ev1)
        Fa = features(L)
        pred_err.append(abs(float(model.predict(Fa).sum()) - e_exact) / abs(e_exact))
        for f in fracs:
            r = screened_energy(L, model, f, F=None)
            res[f]["surrogate"].append(abs(r.e - e_exact) / abs(e_exact))
            res[f]["surrogate_drop"].append(abs(r.e_exact_part - e_exact) / abs(e_exact))
            res[f]["speedup"].append(t_exact / r.ms)
            h = screened_energy(L, None, f, F=Fa)
            res[f]["heuristic_drop"].append(abs(h.e_exact_part - e_exact) / abs(e_exact))
            res[f]["heuristic_scaled"].append(abs(h.e - e_exact) / abs(e_exact))
        del L, Fa
        torch.cuda.empty_cache()
    out = {"n_train": n_train, "n_test": n_test, "per_system_jobs": per_system, "epochs": epochs,
           "train_samples": per_system * n_train, "data_s": t_data, "train_s": t_train,
           "final_loss": model.history[-1] if model.history else None,
           "predicted_total_rel_err": {"median": float(np.median(pred_err)), "max": float(np.max(pred_err))},
           "fractions": {}}
    for f in fracs:
        out["fractions"][str(f)] = {k: {"median": float(np.median(vals)), "max": float(np.max(vals))}
                                    for k, vals in res[f].items()}
    return out


if __name__ == "__main__":
    import argparse
    import json
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=192)
    ap.add_argument("--test", type=int, default=64)
    ap.add_argument("--per-system", type=int, default=20000)
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--out", default="")
    a = ap.parse_args()
    r = study(a.train, a.test, per_system=a.per_system, epochs=a.epochs, verbose=True)
    s = json.dumps(r, indent=1)
    print(s)
    if a.out:
        open(a.out, "w").write(s)
