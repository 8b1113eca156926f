"""CPU: index algebra of the mixed path's qr-tiled slot layout.

Each o^3 slot of the tcgen05 path's wave scratch stores element (p,q,r) at
p o^2 + (q/8) 8o + (r/8) 64 + (q%8) 8 + r%8 (pyscfad_b200/csrc/ct_mixed.cu).
The six W-bar slots of a job are index permutations of one cube; the GEMM
kinds that need r apart from (p,q) (OB1, OB2) read term t's W-bar from the
slot kRotTerm[t], where it sits as (r, tiled pq).  This test builds the six
slots the way the orbit epilogue fills them (Wbar_s = wbar transposed by the
oracle's gather transpose), emulates the tensor boxes of OB1's A and OB2's B
on the tiled array, and checks them against the plain (p,q,r) cube, together
with the vooo tensor box of OB2, the row/column maps of their epilogues and
the address formulas the other epilogues use.
"""
import numpy as np
import pytest

from oracle.ccsd_t_np import GATHER_T

ROT_TERM = [4, 2, 5, 0, 3, 1]   # kRotTerm in ct_mixed.cu (packed there as 0x130524)


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


def job_slots(rng, o):
    """The six W-bar slots of one job: Wbar_s = wbar.transpose(GATHER_T[s])."""
    wbar = rng.standard_normal((o, o, o))
    return np.stack([wbar.transpose(GATHER_T[s]) for s in range(6)])


def untile_pq(k, o):
    """Tiled position k of a (p,q) plane -> p*o + q, as the OB1/TB epilogues do it."""
    omag = ((1 << 32) + o - 1) // o
    Pb = ((k * omag) >> 32) >> 3
    rem = k - Pb * 8 * o
    return (8 * Pb + ((rem >> 3) & 7)) * o + 8 * (rem >> 6) + (rem & 7)


def test_rot_term_table():
    """kRotTerm[s] holds Wbar_s[p,q,r] at (r,p,q); its packed form decodes to the table."""
    rng = np.random.default_rng(5)
    W = job_slots(rng, 6)
    for s in range(6):
        assert np.array_equal(W[s], W[ROT_TERM[s]].transpose(1, 2, 0))
        assert (0x130524 >> (4 * s)) & 15 == ROT_TERM[s]


def box3(flat, dims, strides, box, coord):
    """A 3-D tensor box (innermost first), zero outside dims: out[b2, b1, b0]."""
    out = np.zeros(box[::-1])
    for i2 in range(box[2]):
        for i1 in range(box[1]):
            for i0 in range(box[0]):
                c = (coord[0] + i0, coord[1] + i1, coord[2] + i2)
                if all(0 <= c[d] < dims[d] for d in range(3)):
                    out[i2, i1, i0] = flat[c[0] + c[1] * strides[0] + c[2] * strides[1]]
    return out


@pytest.mark.parametrize("CK", [32, 64])   # elements per 128-byte row: tf32, bf16
@pytest.mark.parametrize("o", [8, 16, 40])
def test_ob1_rotated_a_tile(o, CK):
    """OB1 A: M-tile mt = 128 tiled pq positions, K rows = all r (o rounded up
    to a whole k-step, kr8), one box of kr8 rows per CK positions from the
    rotated slot (map dims (o^2, o, slots)); row k is Wbar_t[p(k), q(k), :]."""
    rng = np.random.default_rng(o + CK)
    W = job_slots(rng, o)
    flat = to_tiled(W)
    o2 = o * o
    kr8 = (o + 15) // 16 * 16 if CK == 64 else (o + 7) // 8 * 8
    for t in range(6):
        rs = ROT_TERM[t]
        for mt in range((o2 + 127) // 128):
            tile = np.concatenate([box3(flat, (o2, o, 6), (o2, o ** 3), (CK, kr8, 1),
                                        (128 * mt + CK * c, 0, rs))[0]
                                   for c in range(128 // CK)], axis=1)   # [r, k]
            assert tile.shape == (kr8, 128)
            for m in range(128):
                k = 128 * mt + m
                if k >= o2:
                    assert not tile[:, m].any()
                    continue
                pq = untile_pq(k, o)
                p, q = divmod(pq, o)
                assert np.array_equal(tile[:o, m], W[t, p, q, :]), (t, mt, m)
                assert not tile[o:, m].any()


@pytest.mark.parametrize("CK", [32, 64])
@pytest.mark.parametrize("o", [8, 24, 48])
def test_ob2_rotated_b_tile_and_vooo_box(o, CK):
    """OB2: K chunk (pk, Q) = rows (p0 + p_local, 8Q + q8); A is the 4-D vooo
    box, B per term the o rows r of the rotated slot at the CK tiled positions
    from koff (map dims (o^2, o, slots)); columns of term t are t*o + r."""
    rng = np.random.default_rng(100 + o)
    nx = 3
    nb, PK = o // 8, CK // 8
    W = job_slots(rng, o)
    wflat = to_tiled(W)
    vooo = rng.standard_normal((nx, o, o, o))      # vooo[x, p, q, l]
    o2 = o * o
    for pk in range(o // PK):
        for Q in range(nb):
            p0 = PK * pk
            rows = [(p0 + m // 8, 8 * Q + m % 8) for m in range(CK)]
            # A: the 4-D tensor box (l, q8, Q, x*o + p) of vooo, inner dimension CK (a full row)
            for x in range(nx):
                for c in range((o + CK - 1) // CK):
                    for m, (p, qq) in enumerate(rows):
                        n = min(CK, o - CK * c)
                        off = CK * c + (qq % 8) * o + Q * 8 * o + (x * o + p) * o * o
                        assert np.array_equal(vooo.reshape(-1)[off:off + n], vooo[x, p, qq, CK * c:CK * c + n])
            koff = (p0 >> 3) * 8 * o + Q * 64 + (p0 & 7) * 8
            assert koff % 4 == 0                      # 16-byte aligned x coordinate (tf32 and bf16)
            for t in range(6):
                tile = box3(wflat, (o2, o, 6), (o2, o ** 3), (CK, o, 1), (koff, 0, ROT_TERM[t]))[0]   # [r, kk]
                for m, (p, qq) in enumerate(rows):
                    assert np.array_equal(tile[:, m], W[t, p, qq, :]), (pk, Q, t, m)
    # epilogue columns: chunk c0 of 16 spans at most two terms
    for nterms in range(1, 256 // o + 1):
        N = (nterms * o + 15) // 16 * 16
        seen = set()
        for c0 in range(0, N, 16):
            t_lo = c0 // o
            if t_lo >= nterms:
                continue
            for cc in range(16):
                r0 = c0 + cc - t_lo * o
                wrap = r0 >= o
                t = t_lo + wrap
                r = r0 - o if wrap else r0
                if t < nterms:
                    assert 0 <= r < o and (c0 + cc) == t * o + r
                    seen.add((t, r))
        assert len(seen) == nterms * o


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



def plane_pos(q, r, o, qrt):
    """lnoproj::plane_pos in ct_lno.cu: position of (q, r) in one plane."""
    return (q >> 3) * 8 * o + (r >> 3) * 64 + (q & 7) * 8 + (r & 7) if qrt else q * o + r


@pytest.mark.parametrize("NT", [4, 8])
@pytest.mark.parametrize("o,qrt", [(8, True), (16, True), (32, True), (5, False), (13, False), (32, False)])
def test_lno_proj_kernel_indexing(NT, o, qrt):
    """The index arithmetic of lnoproj::proj_kernel (ct_lno.cu), emulated for
    every thread: the staged plane and chunk tiles are written once per tile
    position and read only inside the tile; the plane loads hit every (q, r)
    of a plane once, the chunk loads every (l, position) once; the A12/B12
    writes cover every plane position once and the A0/B0 writes every
    (k, position) once, all inside the cube."""
    R = 8 * NT
    if o > R or (NT == 8 and o <= 32 and o != 32):
        pytest.skip("size handled by the other build")
    S, SC, NTHR, CG = R + 4, 68, 64 * NT, NT // 2
    oo = o * o
    idx = tiled_index(o)[0] if qrt else None
    # staging: tile positions of plane and chunk
    plane_seen, chunk_seen = np.zeros(oo, int), np.zeros(oo, int)
    tile_p, tile_c = set(), set()
    for tid in range(NTHR):
        for k in range(NT):
            i = tid + k * NTHR
            q, r = divmod(i, R)
            assert q * S + r < R * SC
            tile_p.add(q * S + r)
            if q < o and r < o:
                pos = plane_pos(q, r, o, qrt)
                if qrt:
                    assert pos == idx[q, r]
                plane_seen[pos] += 1
        for k in range(8):
            i = tid + k * NTHR
            l, j = i >> 6, i & 63
            tile_c.add(l * SC + j)
            if l < o and j < oo:
                chunk_seen[j] += 1   # chunk 0; other chunks shift the position by 64 ch
    assert len(tile_p) == R * R and len(tile_c) == R * 64
    assert (plane_seen == 1).all()
    assert (chunk_seen[:min(64, oo)] == o).all() and (chunk_seen[min(64, oo):] == 0).all()
    # outputs of every warp (2 NT warps; lane (g, c); tile columns by halves)
    a12 = np.zeros(oo, int)
    nch = (oo + 63) // 64
    a0 = np.zeros((o, nch * 64), int)
    for warp in range(2 * NT):
        mt, half = warp >> 1, warp & 1
        for lane in range(32):
            g, c = lane >> 2, lane & 3
            row = mt * 8 + g
            for kk in range(0, R, 4):   # fragment reads stay inside the tiles
                kr = kk + c
                for j in range(CG):
                    col = (half * CG + j) * 8 + g
                    assert max(row, kr, col) < R
                for j in range(4):
                    assert (half * 4 + j) * 8 + g < 64
            for j in range(CG):
                for h in range(2):
                    r = (half * CG + j) * 8 + 2 * c + h
                    if row < o and r < o:
                        a12[plane_pos(row, r, o, qrt)] += 1
            for ch in range(nch):
                for j in range(4):
                    for h in range(2):
                        P = 64 * ch + (half * 4 + j) * 8 + 2 * c + h
                        if row < o and P < oo:
                            a0[row, P] += 1
    assert (a12 == 1).all()
    assert (a0[:, :oo] == 1).all() and (a0[:, oo:] == 0).all()
