"""Proof-of-work search on the B200 against the oracle (smallest nonce in
stwo's (hi << 32) | low order) and against the reference's own grind
kernels (oracle/_ref)."""
import ctypes as C
import hashlib
import struct

import numpy as np
import pytest

from gpu_util import to_dev
from vortexstark_b200 import _lib
from vortexstark_b200.channel import Channel
from vortexstark_b200.grind import grind, grind_prefixed

pytestmark = pytest.mark.gpu
P = 0x7FFFFFFF


def _channel(seed):
    ch = Channel()
    ch.mix_digest(struct.unpack("<8I", hashlib.blake2s(bytes([seed, 7])).digest()))
    return ch


@pytest.mark.parametrize("m31", [False, True])
@pytest.mark.parametrize("bits", [1, 5, 10, 14, 18, 21])
def test_grind_matches_oracle(oracle, bits, m31):
    for seed in range(2):
        pre = _channel(seed).pow_prefix(bits)
        got = grind_prefixed(pre, bits, m31)
        assert got == oracle.grind_pow(pre, bits, m31), (seed, bits, m31)


def test_grind_channel_accepts_and_pow_zero():
    ch = _channel(3)
    n = grind(ch, 20)
    assert ch.verify_pow_nonce(20, n)
    assert grind(ch, 0) == 0


def test_grind_exhaustion_is_an_error():
    pre = _channel(4).pow_prefix(64)
    with pytest.raises(_lib.VortexError):
        grind_prefixed(pre, 64, False, max_batches=1)


def _batch(fn, pre_dev, bits, offset, n):
    import torch

    res = torch.full((1,), -1, dtype=torch.int64, device="cuda")
    fn(pre_dev.data_ptr(), res.data_ptr(), bits, offset, n)
    torch.cuda.synchronize()
    return int(res.cpu().numpy().view(np.uint64)[0])


@pytest.mark.parametrize("m31", [False, True])
def test_reference_launchers_match_oracle_and_reference_kernels(oracle, m31):
    L = _lib.lib()
    fn = L.cuda_grind_pow_m31_output if m31 else L.cuda_grind_pow
    R = None
    if oracle.ref_available():
        R = oracle.ref_lib()
        for name in ("cuda_grind_pow", "cuda_grind_pow_m31_output"):
            getattr(R, name).argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint64, C.c_uint32]
    for seed, bits in ((5, 8), (6, 12), (7, 15)):
        pre = _channel(seed).pow_prefix(bits)
        want = oracle.grind_pow(pre, bits, m31)  # in batch 0 at these sizes
        pre_dev = to_dev(np.array(pre, np.uint32))
        assert _batch(fn, pre_dev, bits, 0, 1 << 20) == want
        # a window starting past the answer finds the next accepted nonce
        nxt = _batch(fn, pre_dev, bits, want + 1, 1 << 20)
        assert nxt > want and oracle.verify_pow_nonce(pre, bits, nxt, m31)
        if R is not None:
            rfn = R.cuda_grind_pow_m31_output if m31 else R.cuda_grind_pow
            assert _batch(rfn, pre_dev, bits, 0, 1 << 20) == want
