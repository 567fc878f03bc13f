"""Proof of work (channel.rs:140-168, grind.cu, grind_m31_output.cu): the
oracle's prefix digest and nonce search against hashlib, host only."""
import hashlib
import struct

import pytest

from vortexstark_b200.channel import Channel

P = 0x7FFFFFFF


def _tz(prefix, nonce, m31=False):
    h = hashlib.blake2s(struct.pack("<8I", *prefix) + struct.pack("<Q", nonce)).digest()
    w = list(struct.unpack("<4I", h[:16]))
    if m31:
        w = [x % P for x in w]
    v = w[0] | (w[1] << 32) | (w[2] << 64) | (w[3] << 96)
    return (v & -v).bit_length() - 1 if v else 128


def _channel(seed):
    ch = Channel()
    ch.mix_digest(struct.unpack("<8I", hashlib.blake2s(bytes([seed])).digest()))
    return ch


def test_prefix_matches_channel(oracle):
    for seed in range(4):
        ch = _channel(seed)
        for bits in (1, 20, 26):
            assert tuple(oracle.pow_prefix(ch.state_words(), bits)) == ch.pow_prefix(bits)


@pytest.mark.parametrize("m31", [False, True])
@pytest.mark.parametrize("bits", [1, 3, 6, 9])
def test_oracle_grind_is_the_smallest_nonce(oracle, bits, m31):
    for seed in range(3):
        pre = _channel(seed).pow_prefix(bits)
        n = oracle.grind_pow(pre, bits, m31)
        assert n < (1 << 20)  # found in batch 0 at these sizes
        assert _tz(pre, n, m31) >= bits
        assert all(_tz(pre, k, m31) < bits for k in range(n))
        assert oracle.verify_pow_nonce(pre, bits, n, m31)


def test_channel_verify_and_mix(oracle):
    ch = _channel(9)
    n = oracle.grind_pow(ch.pow_prefix(12), 12)
    assert ch.verify_pow_nonce(12, n)
    assert oracle.grind_pow(ch.pow_prefix(5), 0) == 0
    before = ch.state
    ch.mix_u64(n)
    assert ch.state == hashlib.blake2s(before + struct.pack("<Q", n)).digest() and ch.n_draws == 0
