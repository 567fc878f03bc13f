"""Seeded synthetic inputs for the benchmark and the parity tests.

There is no public dataset on this path; every input is derived from a
SplitMix64 stream per seed.  M31 values are ``next() >> 33`` with the value P
rejected, so they are uniform on [0, 2^31 - 1).
"""
from __future__ import annotations

P = 0x7FFFFFFF
_MASK = (1 << 64) - 1


class SplitMix64:
    def __init__(self, seed: int):
        self.s = seed & _MASK

    def next(self) -> int:
        self.s = (self.s + 0x9E3779B97F4A7C15) & _MASK
        z = self.s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _MASK
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _MASK
        return z ^ (z >> 31)

    def m31(self) -> int:
        while True:
            v = self.next() >> 33
            if v != P:
                return v

    def uniform(self) -> float:
        return (self.next() >> 11) * (1.0 / (1 << 53))


def fib_inputs(seed: int, count: int):
    """(a0, a1) pairs uniform in [0, P)."""
    g = SplitMix64(seed)
    return [(g.m31(), g.m31()) for _ in range(count)]


def m31_array(seed: int, n: int):
    """n uniform M31 words as a numpy uint32 array (vectorised SplitMix64)."""
    import numpy as np

    idx = np.arange(1, n + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = (np.uint64(seed) + idx * np.uint64(0x9E3779B97F4A7C15))
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    v = (z >> np.uint64(33)).astype(np.uint32)
    v[v == P] = 0  # the one value outside the field maps to 0 (probability 2^-31)
    return v


def served_stream(seed: int, n_requests: int = 512, sizes=(16, 18, 20, 22, 24),
                  weights=(0.40, 0.25, 0.20, 0.10, 0.05)):
    """Mixed-size request stream: (log_n, a, b) per request, log_n drawn with
    the given weights."""
    g = SplitMix64(seed)
    cum, acc = [], 0.0
    for w in weights:
        acc += w
        cum.append(acc)
    out = []
    for _ in range(n_requests):
        u = g.uniform() * acc
        k = next(i for i, c in enumerate(cum) if u < c)
        out.append((sizes[k], g.m31(), g.m31()))
    return out
