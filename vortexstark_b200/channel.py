"""Fiat-Shamir channel (src/channel.rs:15-185), host side.

The prover runs the same transcript on the device; this host copy is what the
verifier replays.  Blake2s-256 throughout: mix_digest = B(state || root),
squeeze = B(state || n_draws_le32 || 0x00), draw_felt rejection-samples the 8
squeezed words below 2P and keeps words 0..3 mod P, draw_number is the LE u64
of the first 8 squeezed bytes mod bound, mix_felts = B(state || felts).
"""
from __future__ import annotations

import hashlib
import struct

P = 0x7FFFFFFF


def _b2s(data: bytes) -> bytes:
    return hashlib.blake2s(data, digest_size=32).digest()


class Channel:
    def __init__(self):
        self.state = bytes(32)
        self.n_draws = 0

    def mix_digest(self, digest) -> None:
        self.state = _b2s(self.state + struct.pack("<8I", *digest))
        self.n_draws = 0

    def mix_felts(self, felts) -> None:
        if not felts:
            return
        self.state = _b2s(self.state + b"".join(struct.pack("<4I", *f) for f in felts))
        self.n_draws = 0

    def _squeeze(self) -> bytes:
        out = _b2s(self.state + struct.pack("<I", self.n_draws) + b"\x00")
        self.n_draws += 1
        return out

    def draw_felt(self):
        while True:
            w = struct.unpack("<8I", self._squeeze())
            if all(x < 2 * P for x in w):
                return tuple(x % P for x in w[:4])

    def draw_felts(self, n: int):
        return [self.draw_felt() for _ in range(n)]

    def draw_number(self, bound: int) -> int:
        return struct.unpack("<Q", self._squeeze()[:8])[0] % bound

    def draw_query_indices(self, log_domain_size: int, n: int):
        mask = (1 << log_domain_size) - 1
        out = []
        while len(out) < n:
            for w in struct.unpack("<8I", self._squeeze()):
                out.append(w & mask)
                if len(out) == n:
                    break
        return out

    def mix_u64(self, value: int) -> None:
        """channel.rs:120-130: state = B(state || lo_le || hi_le) (a PoW nonce)."""
        self.state = _b2s(self.state + struct.pack("<Q", value))
        self.n_draws = 0

    def pow_prefix(self, pow_bits: int):
        """channel.rs:149-155: B(0x12345678_le || 0^12 || state || pow_bits_le) as 8 LE words."""
        raw = struct.pack("<I", 0x12345678) + bytes(12) + self.state + struct.pack("<I", pow_bits)
        return struct.unpack("<8I", _b2s(raw))

    def verify_pow_nonce(self, pow_bits: int, nonce: int) -> bool:
        """channel.rs:149-168: >= pow_bits trailing zeros in the first 16 bytes
        of B(prefix || nonce_le), read as a LE u128."""
        h = _b2s(struct.pack("<8I", *self.pow_prefix(pow_bits)) + struct.pack("<Q", nonce))
        v = int.from_bytes(h[:16], "little")
        tz = (v & -v).bit_length() - 1 if v else 128
        return tz >= pow_bits

    def state_words(self):
        return struct.unpack("<8I", self.state)
