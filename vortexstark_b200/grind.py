"""Proof-of-work grinding on the B200 (GrindOps::grind, crates/cuda-backend/
src/grind_ops.rs:20-134; kernels grind.cu and grind_m31_output.cu).

``grind(channel, pow_bits)`` returns the smallest nonce (hi << 32) | low,
low < 2^20, hi = 0, 1, ... (stwo's search order) that the channel's
``verify_pow_nonce`` accepts; the search runs on the device through
``vx_grind_pow``.
"""
from __future__ import annotations

import ctypes as C

from . import _lib
from .channel import Channel


def grind_prefixed(prefixed_digest, pow_bits: int, m31_output: bool = False, max_batches: int = 1 << 16,
                   stream=None) -> int:
    """Search from a precomputed prefix digest (8 words)."""
    words = (C.c_uint32 * 8)(*prefixed_digest)
    out = C.c_uint64()
    _lib.check(_lib.lib().vx_grind_pow(words, pow_bits, int(m31_output), max_batches, C.byref(out),
                                       C.c_void_p(stream) if stream else None))
    return int(out.value)


def grind(channel: Channel, pow_bits: int, max_batches: int = 1 << 16) -> int:
    """GrindOps::grind for the standard Blake2s channel."""
    if pow_bits == 0:
        return 0
    return grind_prefixed(channel.pow_prefix(pow_bits), pow_bits, False, max_batches)
