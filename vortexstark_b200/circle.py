"""Circle group over M31, cosets and GPU twiddle tables.

Mirrors src/circle.rs: ``CirclePoint`` (generator (2, 1268011823), group law
circle.rs:33-39), ``Coset`` constructors (subgroup 101-109, half_coset 113-122,
half_odds 132-143, ``at`` 183-185) and the GPU twiddle builders
(``compute_forward_twiddles_gpu`` 454-521, ``compute_inverse_twiddles_gpu``
525-550), which chain the exported launchers cuda_compute_coset_points,
cuda_extract_and_squash and cuda_batch_inverse_m31 exactly as the reference does.
"""
from __future__ import annotations

from dataclasses import dataclass

from . import _lib

P = 0x7FFFFFFF


@dataclass(frozen=True)
class CirclePoint:
    x: int
    y: int

    def mul(self, o: "CirclePoint") -> "CirclePoint":
        return CirclePoint((self.x * o.x - self.y * o.y) % P, (self.x * o.y + self.y * o.x) % P)

    def double(self) -> "CirclePoint":
        return self.mul(self)

    def repeated_double(self, n: int) -> "CirclePoint":
        p = self
        for _ in range(n):
            p = p.double()
        return p

    def mul_scalar(self, k: int) -> "CirclePoint":
        r, b = IDENTITY, self
        while k:
            if k & 1:
                r = r.mul(b)
            b = b.double()
            k >>= 1
        return r

    def conjugate(self) -> "CirclePoint":
        return CirclePoint(self.x, (-self.y) % P)


IDENTITY = CirclePoint(1, 0)
GENERATOR = CirclePoint(2, 1268011823)


@dataclass(frozen=True)
class Coset:
    initial: CirclePoint
    step: CirclePoint
    log_size: int

    @staticmethod
    def subgroup(log_size: int) -> "Coset":
        assert log_size <= 31
        return Coset(IDENTITY, GENERATOR.repeated_double(31 - log_size), log_size)

    @staticmethod
    def half_coset(log_size: int) -> "Coset":
        assert log_size <= 30
        return Coset(GENERATOR.repeated_double(30 - log_size), GENERATOR.repeated_double(31 - log_size), log_size)

    @staticmethod
    def half_odds(log_size: int) -> "Coset":
        assert log_size <= 30
        return Coset(GENERATOR.repeated_double(max(29 - log_size, 0)), GENERATOR.repeated_double(31 - log_size),
                     log_size)

    def size(self) -> int:
        return 1 << self.log_size

    def at(self, i: int) -> CirclePoint:
        return self.initial.mul(self.step.mul_scalar(i & 0xFFFFFFFF))


def eval_domain(log_size: int) -> Coset:
    """half_coset up to 30, subgroup(31) at 31 (prover.rs:655-659)."""
    return Coset.half_coset(log_size) if log_size <= 30 else Coset.subgroup(log_size)


def _u32(n, device="cuda"):
    import torch

    return torch.empty(max(int(n), 1), dtype=torch.int32, device=device)


def compute_forward_twiddles_gpu(coset: Coset):
    """circle.rs:454-521 — returns (line, circle, layer_offsets, layer_sizes);
    line and circle are device tensors (int32 storage of u32 words)."""
    L = _lib.lib()
    n = coset.size()
    n_line = coset.log_size - 1 if coset.log_size > 0 else 0
    xs, ys = _u32(n), _u32(n)
    L.cuda_compute_coset_points(coset.initial.x, coset.initial.y, coset.step.x, coset.step.y,
                                xs.data_ptr(), ys.data_ptr(), n)
    circle = ys[: n // 2].clone()
    line = _u32(n - 1)
    offsets, sizes = [], []
    cur, cur_n, off = xs, n, 0
    for _ in range(n_line):
        ls = cur_n // 2
        offsets.append(off)
        sizes.append(ls)
        sq = _u32(ls)
        L.cuda_extract_and_squash(cur.data_ptr(), line.data_ptr() + 4 * off, sq.data_ptr(), ls)
        off += ls
        cur, cur_n = sq, ls
    return line, circle, offsets, sizes


def compute_inverse_twiddles_gpu(coset: Coset):
    """circle.rs:525-550 — forward tables, then batch inverse (0 -> 0)."""
    L = _lib.lib()
    line, circle, offsets, sizes = compute_forward_twiddles_gpu(coset)
    n = coset.size()
    iline, icircle = _u32(n - 1), _u32(n // 2)
    if n - 1 > 0:
        L.cuda_batch_inverse_m31(line.data_ptr(), iline.data_ptr(), n - 1)
    if n // 2 > 0:
        L.cuda_batch_inverse_m31(circle.data_ptr(), icircle.data_ptr(), n // 2)
    return iline, icircle, offsets, sizes
