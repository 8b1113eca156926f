"""CPU: index algebra of the mixed path's qr-tiled slot layout.

Each o^3 slot of the tcgen05 path's wave scratch stores element (p,q,r) at
p o^2 + (q/8) 8o + (r/8) 64 + (q%8) 8 + r%8 (pyscfad_b200/csrc/ct_mixed.cu).
The GEMM kinds read it through tensor maps whose boxes are written densely in
box order; this test emulates those boxes with numpy on a tiled array and
checks them against the tiles of the plain (p,q,r) array that the same
contraction needs, together with the address formulas the epilogues use.
"""
import numpy as np
import pytest


def tiled_index(o):
    p, q, r = np.meshgrid(np.arange(o), np.arange(o), np.arange(o), indexing="ij")
    return p * o * o + (q // 8) * 8 * o + (r // 8) * 64 + (q % 8) * 8 + (r % 8)


def to_tiled(x):
    """x: (nslot, o, o, o) plain -> flat tiled array."""
    nslot, o = x.shape[0], x.shape[1]
    out = np.zeros(nslot * o ** 3, dtype=x.dtype)
    idx = tiled_index(o)
    for s in range(nslot):
        out[s * o ** 3 + idx] = x[s]
    return out


def box(flat, dims, strides, box_shape, coords):
    """Dense box of a tensor map (dim 0 fastest) with zero fill outside dims;
    returned as rows of box_shape[0] * box_shape[1] elements."""
    rank = len(dims)
    el = np.zeros(box_shape[::-1], dtype=flat.dtype)
    for ix in np.ndindex(*box_shape[::-1]):
        c = [coords[d] + ix[rank - 1 - d] for d in range(rank)]
        if any(c[d] < 0 or c[d] >= dims[d] for d in range(rank)):
            continue
        off = c[0] + sum(c[d] * strides[d - 1] for d in range(1, rank))
        el[ix] = flat[off]
    return el.reshape(-1, box_shape[0] * box_shape[1])


@pytest.mark.parametrize("CK", [32, 64])   # elements per 128-byte row: tf32, bf16
@pytest.mark.parametrize("o", [8, 16, 40, 48])
def test_ob1_gather_box(o, CK):
    rng = np.random.default_rng(o)
    nslot = 3
    nb = o // 8
    x = rng.standard_normal((nslot, o, o, o))
    flat = to_tiled(x)
    dims, strides = [8, nb, 8, nb, nslot * o], [64, 8, 8 * o, o * o]
    for slot in range(nslot):
        for pg in range((o + 15) // 16):
            for Q in range(nb):
                for kr in range((o + CK - 1) // CK):
                    b = box(flat, dims, strides, [8, CK // 8, 8, 1, 16], [0, (CK // 8) * kr, 0, Q, slot * o + 16 * pg])
                    assert b.shape == (8 * 16, CK)
                    for m in range(128):
                        p, qq = 16 * pg + m // 8, 8 * Q + m % 8
                        r0 = CK * kr
                        if p >= o:
                            continue   # rows past the slot: never stored
                        want = np.zeros(CK)
                        n = min(CK, o - r0)
                        want[:n] = x[slot, p, qq, r0:r0 + n]
                        assert np.array_equal(b[m], want), (slot, pg, Q, kr, m)


@pytest.mark.parametrize("CK", [32, 64])
@pytest.mark.parametrize("o", [8, 24, 48])
def test_ob2_gather_boxes(o, CK):
    rng = np.random.default_rng(100 + o)
    nslot, nx = 2, 3
    nb, PK = o // 8, CK // 8
    w = rng.standard_normal((nslot, o, o, o))      # W-bar slots (p, q, r)
    vooo = rng.standard_normal((nx, o, o, o))      # vooo[x, p, q, l]
    wflat = to_tiled(w)
    vflat = vooo.reshape(-1)
    for pk in range(o // PK):
        for Q in range(nb):
            rows = [(PK * pk + m // 8, 8 * Q + m % 8) for m in range(CK)]
            for x in range(nx):
                for c in range((o + CK - 1) // CK):
                    a = box(vflat, [o, 8, nb, nx * o], [o, 8 * o, o * o], [CK, 8, 1, PK], [CK * c, 0, Q, x * o + PK * pk])
                    a = a.reshape(CK, CK)
                    for m, (p, qq) in enumerate(rows):
                        n = min(CK, o - CK * c)
                        assert np.array_equal(a[m, :n], vooo[x, p, qq, CK * c:CK * c + n])
            for slot in range(nslot):
                for c in range((o + CK - 1) // CK):
                    b = box(wflat, [8, nb, 8, nslot * o, nb], [64, 8, o * o, 8 * o], [8, CK // 8, 8, PK, 1],
                            [0, (CK // 8) * c, 0, slot * o + PK * pk, Q])
                    for m, (p, qq) in enumerate(rows):
                        n = min(CK, o - CK * c)
                        assert np.array_equal(b[m, :n], w[slot, p, qq, CK * c:CK * c + n])
                        assert not b[m, n:].any()


@pytest.mark.parametrize("o", [8, 16, 48, 56])
def test_tb_untile_and_f2_address(o):
    idx = tiled_index(o)
    omag = ((1 << 32) + o - 1) // o
    for p in range(0, o, max(1, o // 4)):
        for q in range(o):
            for r in range(o):
                qt = idx[p, q, r] - p * o * o
                Qb = ((qt * omag) >> 32) >> 3
                rem = qt - Qb * 8 * o
                qr = (8 * Qb + ((rem >> 3) & 7)) * o + 8 * (rem >> 6) + (rem & 7)
                assert qr == q * o + r
                pq = p * o + q
                pp = (pq * omag) >> 32
                qq = pq - pp * o
                assert pp * o * o + (qq >> 3) * 8 * o + (r >> 3) * 64 + (qq & 7) * 8 + (r & 7) == idx[p, q, r]


@pytest.mark.parametrize("o", [8, 48])
def test_epilogue_block_rows_contiguous(o):
    """An 8x8x8 block (P,Q,R) of a tiled slot is eight runs of 64 floats at
    (p0+u) o^2 + q0 o + 8 r0, the offsets the epilogue's copies use."""
    idx = tiled_index(o)
    nb = o // 8
    for P in range(nb):
        for Q in range(nb):
            for R in range(nb):
                for u in range(8):
                    p = 8 * P + u
                    run = idx[p, 8 * Q:8 * Q + 8, 8 * R:8 * R + 8].reshape(-1)
                    base = p * o * o + 8 * Q * o + 8 * 8 * R
                    assert np.array_equal(run, base + np.arange(64))


@pytest.mark.parametrize("o", [8, 24, 48])
def test_vterm_tiled_reads(o):
    """The V-term kernel's three axis passes read ybar through tile(j, k)."""
    idx = tiled_index(o)
    tile = lambda j, k: (j >> 3) * 8 * o + (k >> 3) * 64 + (j & 7) * 8 + (k & 7)  # noqa: E731
    for f0 in range(0, o, 3):
        for f1 in range(0, o, 5):
            for r in range(o):
                assert r * o * o + tile(f0, f1) == idx[r, f0, f1]     # axis 0
                assert f0 * o * o + tile(r, f1) == idx[f0, r, f1]     # axis 1
                assert f0 * o * o + tile(f1, r) == idx[f0, f1, r]     # axis 2
