"""Test infrastructure: numpy restatement of the learned block surrogate.

Only tests/ and the smoke check import this module; it is the checker of the
CUDA kernels in pyscfad_b200/csrc/mlp.cu, never a compute path.

The reference has no counterpart to this part (pyscfad ships no learned
component); what it restates is this repository's own specification of the
surrogate: a 12-128-128-1 SiLU MLP over 12 per-job features of a sorted
virtual triple (a >= b >= c), trained with mean-squared error and AdamW.
Everything is float64 here, so the GPU's float32 kernels are compared within
float32 tolerances.

Parameter vector layout: W1[128][12] | b1[128] | W2[128][128] | b2[128] | W3[128] | b3.
"""
from __future__ import annotations

import numpy as np

NI, NH = 12, 128
NPARAM = NH * NI + NH + NH * NH + NH + NH + 1


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    o = 0
    W1 = p[o:o + NH * NI].reshape(NH, NI); o += NH * NI
    b1 = p[o:o + NH]; o += NH
    W2 = p[o:o + NH * NH].reshape(NH, NH); o += NH * NH
    b2 = p[o:o + NH]; o += NH
    W3 = p[o:o + NH]; o += NH
    b3 = p[o]
    return W1, b1, W2, b2, W3, b3


def pack(W1, b1, W2, b2, W3, b3):
    return np.concatenate([W1.ravel(), b1, W2.ravel(), b2, W3, [b3]])


def _sig(z):
    return 1.0 / (1.0 + np.exp(-z))


def silu(z):
    return z * _sig(z)


def dsilu(z):
    s = _sig(z)
    return s * (1.0 + z * (1.0 - s))


def forward(p, X):
    """Returns (y, z1, z2) for features X (n, 12)."""
    W1, b1, W2, b2, W3, b3 = unpack(p)
    X = np.asarray(X, dtype=np.float64)
    z1 = X @ W1.T + b1
    z2 = silu(z1) @ W2.T + b2
    y = silu(z2) @ W3 + b3
    return y, z1, z2


def mse(y, t):
    d = np.asarray(y, np.float64) - np.asarray(t, np.float64)
    return float(np.mean(d * d)), 2.0 * d / len(d)


def backward(p, X, z1, z2, dy):
    """Gradient of sum_s dy[s] y[s] with respect to the parameter vector."""
    W1, b1, W2, b2, W3, b3 = unpack(p)
    X = np.asarray(X, dtype=np.float64)
    a1, a2 = silu(z1), silu(z2)
    d2 = dy[:, None] * W3[None, :] * dsilu(z2)
    d1 = (d2 @ W2) * dsilu(z1)
    return pack(d1.T @ X, d1.sum(0), d2.T @ a1, d2.sum(0), a2.T @ dy, float(dy.sum()))


def adam(p, g, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8, wd=0.0):
    """One AdamW step; returns (p, m, v)."""
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    mh = m / (1 - b1 ** step)
    vh = v / (1 - b2 ** step)
    p = p - lr * (mh / (np.sqrt(vh) + eps) + wd * p)
    return p, m, v


def pair_stats(L):
    """(t2 block norms, MP2 pair energies, vvov block norms), each (v, v), of
    the kernel layouts L (t2T (v,v,o,o) [x,y,j,i], vvop (v,v,o,n))."""
    t2T, vvop = L["t2T"], L["vvop"]
    v, _, o, _ = t2T.shape
    K = vvop[:, :, :, :o]                       # K[x,y,i,j]
    tn = np.sqrt(np.einsum("xyji,xyji->xy", t2T, t2T))
    e2 = np.einsum("xyji,xyij->xy", t2T, 2.0 * K - K.transpose(1, 0, 2, 3))
    vn = np.sqrt(np.einsum("xyip,xyip->xy", vvop[:, :, :, o:], vvop[:, :, :, o:]))
    return tn, e2, vn


def features(L, jobs_abc):
    """The 12 features of each job (a, b, c) (rows of jobs_abc), pairs in the
    order (a,b), (a,c), (b,c):
      0-2 log t2 block norm; 3-5 asinh(MP2 pair energy / 1e-4);
      6-8 log of the (x,y),(y,x) vvov block norms in quadrature;
      9 e_a+e_b+e_c-3 e_homo; 10 e_a+e_b+e_c-3 mean(e_occ); 11 log orbit size."""
    tn, e2, vn = pair_stats(L)
    o = L["t2T"].shape[2]
    e = L["mo_energy"]
    eo, ev = e[:o], e[o:]
    J = np.asarray(jobs_abc, dtype=np.int64)
    a, b, c = J[:, 0], J[:, 1], J[:, 2]
    F = np.zeros((len(J), NI))
    for q, (x, y) in enumerate(((a, b), (a, c), (b, c))):
        F[:, q] = np.log(np.maximum(tn[x, y], 1e-30))
        F[:, 3 + q] = np.arcsinh(e2[x, y] * 1e4)
        F[:, 6 + q] = 0.5 * np.log(np.maximum(vn[x, y] ** 2 + vn[y, x] ** 2, 1e-30))
    eabc = ev[a] + ev[b] + ev[c]
    F[:, 9] = eabc - 3 * eo.max()
    F[:, 10] = eabc - 3 * eo.mean()
    F[:, 11] = np.log(np.where(a == c, 1.0, np.where((a == b) | (b == c), 3.0, 6.0)))
    return F
