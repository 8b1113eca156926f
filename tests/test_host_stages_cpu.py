"""CPU: the stage split behind the host-pointer block VJP (ct_host.cu:
block_stages, host_block_vjp), restated and checked exhaustively on small
blocks.

A reference slab block (a0, a1, b0, b1) holds the jobs a in [a0, a1),
b in [b0, b1) (b <= a on a diagonal block), c <= b (ccsd_t.c:16-69).  The
host path runs them in stages: stage 0 the jobs with c >= b0, stage k >= 1
those with c in [(k-1) cw, min(k cw, b0)), cw = max(1, max_wave // pairs).
Stage s copies in, before it runs, the t2T / vooo rows of its row range
([b0, a1) for stage 0, the chunk otherwise) and the parts of the block's
vvop caches on those rows (row caches by columns, column caches by rows);
after stage k >= 1 it drains the same rows and parts of the gradients, and
stage 0's parts and rows come back last.  The checks: every job runs once;
everything a job reads was copied by its stage or an earlier one; the caches'
parts tile each cache exactly; and nothing a chunk drains is touched by a
job of any other stage (so it is final when drained).
"""
import itertools

import pytest


def block_jobs(a0, a1, b0, b1):
    diag = b0 == a0 and b1 == a1
    for a in range(a0, a1):
        for b in (range(a0, a + 1) if diag else range(b0, b1)):
            for c in range(b + 1):
                yield a, b, c


def block_stages(a0, a1, b0, b1, max_wave):
    diag = b0 == a0 and b1 == a1
    npair = (a1 - a0) * (a1 - a0 + 1) // 2 if diag else (a1 - a0) * (b1 - b0)
    cw = max(1, max_wave // npair)
    S = 1 + (b0 + cw - 1) // cw
    stages = [[] for _ in range(S)]
    for a, b, c in block_jobs(a0, a1, b0, b1):
        stages[0 if c >= b0 else 1 + c // cw].append((a, b, c))
    return stages, cw


def stage_rows(s, a1, b0, cw):
    return (b0, a1) if s == 0 else ((s - 1) * cw, min(b0, s * cw))


def caches(a0, a1, b0, b1):
    """(x0, x1, y0, y1) of the block's vvop caches (the reference driver's
    cache_row_a, cache_col_a, cache_row_b, cache_col_b, as the host path uses them)."""
    regs = [(a0, a1, 0, a1)]
    if a0 > 0:
        regs.append((0, a0, a0, a1))
    if b1 <= a0:
        regs.append((b0, b1, 0, b1))
        if b0 > 0:
            regs.append((0, b0, b0, b1))
    return regs


def part(reg, r0, r1):
    x0, x1, y0, y1 = reg
    if y0 == 0:
        y0, y1 = max(y0, r0), min(y1, r1)
    else:
        x0, x1 = max(x0, r0), min(x1, r1)
    return (x0, x1, y0, y1) if x1 > x0 and y1 > y0 else None


def terms(a, b, c):
    """(x, y, z) of the six orderings of a job (ccsd_t_vjp.c:32-37)."""
    return [(a, b, c), (a, c, b), (b, a, c), (b, c, a), (c, a, b), (c, b, a)]


def touched(job):
    """vvop pairs and t2T / vooo rows a job reads and whose gradients it writes:
    vvop[x,y] and vooo[x] of each term, t2T[z] (F1/F2, VB/TB, OB1/OB2) and
    t2T[y, x] (the V term)."""
    pairs, rows = set(), set()
    for x, y, z in terms(*job):
        pairs.add((x, y))
        rows.update((x, y, z))
    return pairs, rows


BLOCKS = [(6, 9, 6, 9), (6, 9, 0, 3), (6, 9, 2, 5), (0, 5, 0, 5), (3, 5, 3, 5), (7, 8, 1, 2), (5, 9, 0, 5)]


@pytest.mark.parametrize("blk", BLOCKS)
@pytest.mark.parametrize("max_wave", [1, 3, 7, 40, 10 ** 6])
def test_block_stages(blk, max_wave):
    a0, a1, b0, b1 = blk
    stages, cw = block_stages(a0, a1, b0, b1, max_wave)
    # every job once, in the stage its smallest index selects
    allj = [j for st in stages for j in st]
    assert sorted(allj) == sorted(block_jobs(a0, a1, b0, b1))
    regs = caches(a0, a1, b0, b1)
    copied_pairs, copied_rows = set(), set()
    stage_pairs, stage_rows_set = [], []
    for s, st in enumerate(stages):
        r0, r1 = stage_rows(s, a1, b0, cw)
        rows = set(range(r0, r1))
        pairs = set()
        for reg in regs:
            p = part(reg, r0, r1)
            if p:
                pairs.update(itertools.product(range(p[0], p[1]), range(p[2], p[3])))
        copied_rows |= rows
        copied_pairs |= pairs
        stage_pairs.append(pairs)
        stage_rows_set.append(rows)
        for j in st:
            jp, jr = touched(j)
            assert jp <= copied_pairs, (s, j, jp - copied_pairs)   # inputs there before it runs
            assert jr <= copied_rows, (s, j, jr - copied_rows)
    # the stages' parts tile every cache exactly
    for reg in regs:
        cells = [(x, y) for x in range(reg[0], reg[1]) for y in range(reg[2], reg[3])]
        count = {c: 0 for c in cells}
        for s in range(len(stages)):
            r0, r1 = stage_rows(s, a1, b0, cw)
            p = part(reg, r0, r1)
            if p:
                for c in itertools.product(range(p[0], p[1]), range(p[2], p[3])):
                    count[c] += 1
        assert all(v == 1 for v in count.values()), reg
    # a chunk's drained pairs and rows are touched by its own jobs only
    for k in range(1, len(stages)):
        for s, st in enumerate(stages):
            if s == k:
                continue
            for j in st:
                jp, jr = touched(j)
                assert not (jp & stage_pairs[k]), (k, s, j)
                assert not (jr & stage_rows_set[k]), (k, s, j)
