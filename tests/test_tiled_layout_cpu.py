"""CPU: index algebra of the mixed path's qr-tiled slot layout.

Each o^3 slot of the tcgen05 path's wave scratch stores element (p,q,r) at
p o^2 + (q/8) 8o + (r/8) 64 + (q%8) 8 + r%8 (pyscfad_b200/csrc/ct_mixed.cu).
The GEMM kinds that gather r back into 128-byte rows (OB1, OB2) stage their
W-bar tiles piece by piece; this test emulates that staging with numpy on a
tiled array and checks the tiles against those of the plain (p,q,r) array
that the same contraction needs, together with the vooo tensor box of OB2 and
the address formulas the other epilogues use.
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


def stage_ob1(flat, o, CK, slot, pg, Q, kr):
    """Rows (p, q8) x CK r of the OB1 A tile, piece by piece as the producer
    warp copies them (16-byte pieces, zero-fill past the slot or past r = o);
    returned unswizzled (row-major 128-byte rows)."""
    nb, EPP = o // 8, 16 // (128 // CK)
    img = np.zeros((128, CK))
    for pi in range(128 * 8):
        m, c = pi >> 3, pi & 7
        p, q8 = 16 * pg + (m >> 3), m & 7
        R = (CK // 8) * kr + (c if CK == 64 else c >> 1)
        e0 = 0 if CK == 64 else (c & 1) * EPP
        if p < o and R < nb:
            el = slot * o ** 3 + p * o * o + Q * 8 * o + R * 64 + q8 * 8 + e0
            img[m, c * EPP:(c + 1) * EPP] = flat[el:el + EPP]
    return img


def stage_ob2(flat, o, CK, slot, pk, Q, cN):
    """K rows (p, q8) x CK r of one (term, N chunk) region of the OB2 B tile."""
    nb, EPP, PK = o // 8, 16 // (128 // CK), CK // 8
    img = np.zeros((CK, CK))
    for pr in range(CK * 8):
        kr, c = pr >> 3, pr & 7
        p, q8 = PK * pk + (kr >> 3), kr & 7
        R = (CK // 8) * cN + (c if CK == 64 else c >> 1)
        e0 = 0 if CK == 64 else (c & 1) * EPP
        if R < nb:
            el = slot * o ** 3 + p * o * o + Q * 8 * o + R * 64 + q8 * 8 + e0
            img[kr, c * EPP:(c + 1) * EPP] = flat[el:el + EPP]
    return img


@pytest.mark.parametrize("CK", [32, 64])   # elements per 128-byte row: tf32, bf16
@pytest.mark.parametrize("o", [8, 16, 40, 48])
def test_ob1_staged_tile(o, CK):
    rng = np.random.default_rng(o)
    nslot, nb = 3, o // 8
    x = rng.standard_normal((nslot, o, o, o))
    flat = to_tiled(x)
    for slot in range(nslot):
        for pg in range((o + 15) // 16):
            for Q in range(nb):
                for kr in range((o + CK - 1) // CK):
                    img = stage_ob1(flat, o, CK, slot, pg, Q, kr)
                    for m in range(128):
                        p, qq = 16 * pg + m // 8, 8 * Q + m % 8
                        want = np.zeros(CK)
                        if p < o:
                            n = min(CK, o - CK * kr)
                            want[:n] = x[slot, p, qq, CK * kr:CK * kr + n]
                        assert np.array_equal(img[m], want), (slot, pg, Q, kr, m)


@pytest.mark.parametrize("CK", [32, 64])
@pytest.mark.parametrize("o", [8, 24, 48])
def test_ob2_staged_tile_and_vooo_box(o, CK):
    rng = np.random.default_rng(100 + o)
    nslot, nx = 2, 3
    nb, PK = o // 8, CK // 8
    w = rng.standard_normal((nslot, o, o, o))      # W-bar slots (p, q, r)
    vooo = rng.standard_normal((nx, o, o, o))      # vooo[x, p, q, l]
    wflat = to_tiled(w)
    for pk in range(o // PK):
        for Q in range(nb):
            rows = [(PK * pk + m // 8, 8 * Q + m % 8) for m in range(CK)]
            # A: the 4-D tensor box (l, q8, Q, x*o + p) of vooo, inner dimension CK (a full row)
            for x in range(nx):
                for c in range((o + CK - 1) // CK):
                    for m, (p, qq) in enumerate(rows):
                        n = min(CK, o - CK * c)
                        off = CK * c + (qq % 8) * o + Q * 8 * o + (x * o + p) * o * o
                        assert np.array_equal(vooo.reshape(-1)[off:off + n], vooo[x, p, qq, CK * c:CK * c + n])
            for slot in range(nslot):
                for c in range((o + CK - 1) // CK):
                    img = stage_ob2(wflat, o, CK, slot, pk, Q, c)
                    for m, (p, qq) in enumerate(rows):
                        n = min(CK, o - CK * c)
                        assert np.array_equal(img[m, :n], w[slot, p, qq, CK * c:CK * c + n])
                        assert not img[m, n:].any()


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
