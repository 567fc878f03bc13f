"""FRI folds on the B200.

Mirrors src/fri.rs: ``SecureColumn`` (SoA QM31, 13-69), fold twiddles
(``compute_fold_twiddles_on_demand`` / ``_async``, 73-139, and
``precompute_fri_twiddles`` 143-160), ``fold_circle_into_line_with_twiddles``
(163-191) and ``fold_line_with_twiddles`` (194-224):
  line:   out[i] = (f0 + f1) + alpha * (tw[i] * (f0 - f1))
  circle: dst[i] = dst[i] * alpha^2 + (f0 + f1) + alpha * (tw[i] * (f0 - f1))
with f0 = src[2i], f1 = src[2i + 1].
"""
from __future__ import annotations

import ctypes as C

from . import _lib
from .circle import Coset
from .field import qm31_mul


def _empty(n):
    import torch

    return torch.empty(max(int(n), 1), dtype=torch.int32, device="cuda")


class SecureColumn:
    def __init__(self, cols, length: int):
        self.cols = cols
        self.len = length

    @classmethod
    def zeros(cls, length: int) -> "SecureColumn":
        import torch

        return cls([torch.zeros(max(length, 1), dtype=torch.int32, device="cuda") for _ in range(4)], length)

    @classmethod
    def alloc(cls, length: int) -> "SecureColumn":
        return cls([_empty(length) for _ in range(4)], length)

    @classmethod
    def from_words(cls, cols_np) -> "SecureColumn":
        import numpy as np
        import torch

        cols = [torch.from_numpy(np.ascontiguousarray(c, dtype=np.uint32).view(np.int32)).cuda() for c in cols_np]
        return cls(cols, int(cols_np[0].shape[0]))

    def to_words(self):
        import numpy as np

        return np.stack([c[: self.len].cpu().numpy().view(np.uint32) for c in self.cols])


def compute_fold_twiddles_on_demand(domain: Coset, extract_y: bool):
    """fri.rs:73-139: tw[i] = 1 / coord(domain.at(brev(2i, log))), i < n/2."""
    L = _lib.lib()
    n = domain.size()
    src = _empty(n // 2)
    L.cuda_compute_fold_twiddle_sources(domain.initial.x, domain.initial.y, domain.step.x, domain.step.y,
                                        src.data_ptr(), n, domain.log_size, 1 if extract_y else 0)
    out = _empty(n // 2)
    L.cuda_batch_inverse_m31(src.data_ptr(), out.data_ptr(), n // 2)
    return out


def precompute_fri_twiddles(start_log_size: int, stop_log_size: int):
    """fri.rs:143-160"""
    res = [compute_fold_twiddles_on_demand(Coset.half_coset(start_log_size), True)]
    log_size = start_log_size - 1
    while log_size > stop_log_size:
        res.append(compute_fold_twiddles_on_demand(Coset.half_odds(log_size), False))
        log_size -= 1
    return res


def _host4(v):
    return (C.c_uint32 * 4)(*[int(x) for x in v])


def fold_circle_into_line_with_twiddles(dst: SecureColumn, src: SecureColumn, alpha, d_twiddles) -> None:
    half = src.len // 2
    alpha_sq = qm31_mul(alpha, alpha)
    _lib.lib().cuda_fold_circle_into_line_soa(*[c.data_ptr() for c in dst.cols], *[c.data_ptr() for c in src.cols],
                                              d_twiddles.data_ptr(), _host4(alpha), _host4(alpha_sq), half)


def fold_line_with_twiddles(ev: SecureColumn, alpha, d_twiddles) -> SecureColumn:
    half = ev.len // 2
    out = SecureColumn.alloc(half)
    _lib.lib().cuda_fold_line_soa(*[c.data_ptr() for c in ev.cols], d_twiddles.data_ptr(),
                                  *[c.data_ptr() for c in out.cols], _host4(alpha), half)
    return out


def fold_circle_into_line(dst: SecureColumn, src: SecureColumn, alpha, domain: Coset) -> None:
    fold_circle_into_line_with_twiddles(dst, src, alpha, compute_fold_twiddles_on_demand(domain, True))


def fold_line(ev: SecureColumn, alpha, domain: Coset) -> SecureColumn:
    return fold_line_with_twiddles(ev, alpha, compute_fold_twiddles_on_demand(domain, False))
