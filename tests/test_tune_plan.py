"""Host-side checks of the plans the autotuner chooses between: every NTT
pass plan covers each butterfly layer once with a pass shape the kernels are
built for, and every Merkle leaf-subtree size gives a consistent tree plan.
No device work."""
import pytest

from vortexstark_b200 import tune
from vortexstark_b200 import _lib
import ctypes as C

# (layers, log2 tile columns) pairs the pass kernels are instantiated for:
# bottom passes on contiguous tiles of up to 2^14 elements, upper passes of
# 3..9 layers on 4096-element tiles, of 10 and 11 layers on 8192-element
# tiles and of 12 layers on 16384-element tiles
BOTTOM_SHAPES = {(r, 0) for r in range(4, 15)}
UPPER_SHAPES = {(r, 12 - r) for r in range(3, 10)} | {(10, 3), (11, 2), (12, 2)}


@pytest.mark.parametrize("bottom", range(9, 15))
@pytest.mark.parametrize("upper", range(3, 13))
def test_every_ntt_plan_is_launchable(bottom, upper):
    for total in range(4, 32):
        plan = tune.ntt_plan(total, bottom, upper)
        start = 0
        for i, (s, r, w) in enumerate(plan):
            assert s == start, (total, plan)
            assert (r, w) in (BOTTOM_SHAPES if i == 0 else UPPER_SHAPES), (total, bottom, upper, plan)
            # an upper pass's 2^w contiguous columns fit between its rows, 2^s apart
            assert w <= s, (total, bottom, upper, plan)
            # an upper pass exceeds `upper` only where the 3-layer minimum merges passes
            if i == 0:
                assert r <= bottom or r == total <= 12  # up to 12 layers: one pass
            else:
                assert r <= max(upper, 5)
                assert w >= 2  # rows of at least 16 bytes (one 16-byte access)
            start += r
        assert start == total


def test_default_ntt_plan_matches_the_built_in_rule():
    assert tune.ntt_plan(24, 12, 12) == [(0, 12, 0), (12, 12, 2)]
    assert tune.ntt_plan(24, 11, 8) == [(0, 11, 0), (11, 7, 5), (18, 6, 6)]
    assert tune.ntt_plan(26, 14, 12) == [(0, 14, 0), (14, 12, 2)]
    assert tune.ntt_plan(24, 13, 11) == [(0, 13, 0), (13, 11, 2)]
    assert tune.ntt_plan(23, 13, 10) == [(0, 13, 0), (13, 10, 3)]
    assert tune.ntt_plan(26, 12, 12) == [(0, 12, 0), (12, 7, 5), (19, 7, 5)]
    assert tune.ntt_plan(28, 12, 10) == [(0, 12, 0), (12, 8, 4), (20, 8, 4)]
    assert tune.ntt_plan(13, 14, 12) == [(0, 13, 0)]
    assert tune.ntt_plan(24, 12, 9) == [(0, 12, 0), (12, 6, 6), (18, 6, 6)]
    assert tune.ntt_plan(14, 12, 9) == [(0, 11, 0), (11, 3, 9)]
    assert tune.ntt_plan(21, 12, 9) == [(0, 12, 0), (12, 9, 3)]
    assert tune.ntt_plan(28, 10, 6) == [(0, 10, 0), (10, 6, 6), (16, 6, 6), (22, 6, 6)]
    # at most 12 layers: one pass whatever the knobs
    assert tune.ntt_plan(11, 10, 6) == [(0, 11, 0)]
    assert tune.ntt_plan(13, 12, 9) == [(0, 10, 0), (10, 3, 9)]


def test_ntt_plan_rejects_unbuilt_shapes():
    for args in ((24, 8, 9), (24, 12, 13), (24, 15, 9), (3, 12, 9), (32, 12, 9)):
        with pytest.raises(_lib.VortexError):
            tune.ntt_plan(*args)


def _tree_plan(depth):
    h = (C.c_uint32 * 12)()
    n, top, nc = C.c_uint32(), C.c_uint32(), C.c_uint32()
    w = C.c_uint64()
    _lib.check(_lib.lib().vx_tree_plan(depth, h, C.byref(n), C.byref(top), C.byref(nc), C.byref(w)))
    return list(h[: n.value]), top.value, w.value


def test_default_leaf_subtree_rule():
    # without a GPU no device knob is set: 2^clamp(depth - 17, 1, 4) leaves per thread
    for depth in range(17, 32):
        heights, top, _ = _tree_plan(depth)
        assert heights[1] == min(max(depth - 17, 1), 4)
    assert _tree_plan(16)[1] == 0  # shallow trees start in the reduce kernel
