"""Per-device autotuner for the NTT pass plans and the Merkle leaf kernel.

The reference launches fixed shapes (src/cuda/circle_ntt.cu: one kernel per
butterfly layer; src/cuda/blake2s.cu: one leaf per thread).  Here the NTT
groups layers into register/shared-memory passes and the Merkle leaf kernel
hashes a subtree of 2^k leaves per thread, and the best grouping depends on
the transform length and tree depth.  ``autotune(max_log)`` times the
candidates on the current device and keeps the fastest; ``set_ntt_plan`` and
``set_leaf_k`` pin a choice by hand.  No choice changes any computed value.
"""
from __future__ import annotations

import ctypes as C
import json

from . import _lib

NTT_PLAN = 0
LEAF_K = 1
FOLD_LEAF_K = 2


def autotune(max_log: int = 24) -> dict:
    """Tune transform lengths 13..max_log and tree depths 17..max_log on the
    current device.  Returns {"ntt": {log: [bottom, upper, ms]},
    "leaf_k": {depth: [k, ms]}, "fold_leaf_k": {depth: [k, ms]}} with int keys."""
    buf = C.create_string_buffer(8192)
    _lib.check(_lib.lib().vx_autotune(max_log, buf, len(buf)))
    raw = json.loads(buf.value.decode())
    return {sec: {int(k): v for k, v in raw[sec].items()} for sec in raw}


def set_ntt_plan(layers: int, bottom: int = 0, upper: int = 0) -> None:
    """Plan of transforms over 2^``layers`` elements (applied to the layers
    such a transform runs): bottom pass of at most ``bottom`` layers (9..14),
    upper passes of at most ``upper`` (3..12); 0 = default."""
    _lib.check(_lib.lib().vx_tune_set(NTT_PLAN, layers, bottom, upper))


def set_leaf_k(depth: int, k: int = 0) -> None:
    """2^k leaves per leaf-kernel thread for narrow-leaf trees of ``depth`` (1..4; 0 = default)."""
    _lib.check(_lib.lib().vx_tune_set(LEAF_K, depth, k, 0))


def set_fold_leaf_k(depth: int, k: int = 0) -> None:
    """The same for wide-leaf trees (FRI layers, lifted rows, their combinations)."""
    _lib.check(_lib.lib().vx_tune_set(FOLD_LEAF_K, depth, k, 0))


def get(kind: int, layers: int) -> tuple[int, int]:
    a, b = C.c_uint32(), C.c_uint32()
    _lib.check(_lib.lib().vx_tune_get(kind, layers, C.byref(a), C.byref(b)))
    return int(a.value), int(b.value)


def ntt_plan(total: int, bottom: int, upper: int) -> list[tuple[int, int, int]]:
    """Host-only pass plan: [(first layer, layers, log2 tile columns)], bottom pass first."""
    s, r, w = (C.c_uint32 * 32)(), (C.c_uint32 * 32)(), (C.c_uint32 * 32)()
    n = C.c_uint32()
    _lib.check(_lib.lib().vx_ntt_plan(total, bottom, upper, s, r, w, C.byref(n)))
    return [(s[i], r[i], w[i]) for i in range(n.value)]


def reset(max_log: int = 31) -> None:
    """Back to the built-in plans for every length and depth."""
    for layers in range(max_log + 1):
        set_ntt_plan(layers)
        set_leaf_k(layers)
        set_fold_leaf_k(layers)
