"""Merkle build plan (host only, no GPU): the stored levels the decommitment
needs, and an index-level simulation of the multi-block reduce kernel
(tree_reduce_kernel in csrc/vx_merkle.cuh) over that plan — every write in
bounds and exactly once, every counter index in range and back at zero, and
exactly one block reaching the root, whatever order the blocks finish in."""
import ctypes as C
import random

import pytest

from vortexstark_b200 import _lib

STAGE_LOG = 8  # kStageLog


def plan(depth):
    h = (C.c_uint32 * 12)()
    n, top, ncnt = C.c_uint32(), C.c_uint32(), C.c_uint32()
    words = C.c_uint64()
    _lib.check(_lib.lib().vx_tree_plan(depth, h, C.byref(n), C.byref(top), C.byref(ncnt), C.byref(words)))
    return list(h[: n.value]), top.value, ncnt.value, words.value


def simulate_reduce(depth, heights, top, n_cnt, seed):
    """Replays the kernel's index arithmetic for every block."""
    stored = {hh: i for i, hh in enumerate(heights) if i >= 1}
    written = {hh: bytearray(1 << (depth - hh)) for hh in stored if hh > heights[top]}
    counters = [0] * n_cnt
    u = depth - heights[top]
    c0 = min(u, STAGE_LOG)
    rng = random.Random(seed)
    # (part, chunks, cbase, h) of every block alive at the current stage
    alive = [(p, 1 << (u - c0), 0, heights[top]) for p in range(1 << (u - c0))]
    roots = 0
    while alive:
        rng.shuffle(alive)
        nxt = []
        for part, chunks, cbase, h in alive:
            c = min(depth - h, STAGE_LOG)
            m = 1 << c
            # inputs: chunk `part` of the level at height h
            assert (part + 1) * m <= 1 << (depth - h)
            for d in range(c):
                half = m >> (d + 1)
                hh = h + d + 1
                if hh in written:
                    lo, hi = part * half, (part + 1) * half
                    assert hi <= len(written[hh])
                    for j in range(lo, hi):
                        assert written[hh][j] == 0, f"level {hh} index {j} written twice"
                        written[hh][j] = 1
            h += c
            if h == depth:
                roots += 1
                continue
            assert h in stored, f"chunk root at height {h} is not a stored level"
            cn = min(depth - h, STAGE_LOG)
            ci = cbase + (part >> cn)
            assert 0 <= ci < n_cnt, (ci, n_cnt)
            counters[ci] += 1
            if counters[ci] == 1 << cn:
                counters[ci] = 0
                nxt.append((part >> cn, chunks >> cn, cbase + (chunks >> cn), h))
            else:
                assert counters[ci] < 1 << cn
        alive = nxt
    assert roots == 1
    assert all(v == 0 for v in counters)
    for hh, w in written.items():
        assert all(w), f"level {hh} not fully written"


@pytest.mark.parametrize("depth", list(range(1, 32)))
def test_tree_plan_shape(depth):
    heights, top, n_cnt, words = plan(depth)
    assert heights[0] == 0 and heights[-1] == depth
    assert len(heights) <= 12
    gaps = [b - a for a, b in zip(heights, heights[1:])]
    assert all(1 <= g <= 4 for g in gaps), gaps  # decommitment re-hashes <= 16 nodes per level
    if depth <= 16:
        assert top == 0
    else:
        assert 1 <= top < len(heights)
        assert 1 << (depth - heights[1]) >= 1 << 16        # leaf kernel threads
        assert depth - heights[top] <= 20                  # reduce launch input <= 2^20 hashes
    # pool = stored hash levels + counters
    assert words == sum(8 << (depth - hh) for hh in heights[1:]) + n_cnt


@pytest.mark.parametrize("depth", [1, 3, 5, 8, 9, 12, 13, 16, 17, 20, 21, 24, 26, 28, 31])
def test_tree_reduce_simulation(depth):
    heights, top, n_cnt, _ = plan(depth)
    for seed in range(3):
        simulate_reduce(depth, heights, top, n_cnt, seed)


def test_tree_plan_rejects_bad_depth():
    for d in (0, 32):
        with pytest.raises(_lib.VortexError):
            plan(d)
