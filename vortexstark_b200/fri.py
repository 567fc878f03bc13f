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


class FriChain:
    """FRI of a QM31 codeword on half_coset(log_size) with a commitment per
    layer, down to 2 values (vx_fri_chain_*): the proof's FRI
    (prover.rs:860-926) as one device call."""

    def __init__(self, log_size: int):
        self.log_size = log_size
        self._h = C.c_void_p()
        _lib.check(_lib.lib().vx_fri_chain_create(log_size, C.byref(self._h)))
        self.layers = int(_lib.lib().vx_fri_chain_layers(self._h))

    def commit_async(self, cols, state_words, stream=None) -> None:
        """cols: 4 device tensors of 2^log_size words; state_words: 8 ints."""
        ptrs = (C.c_void_p * 4)(*[c.data_ptr() for c in cols])
        st = (C.c_uint32 * 8)(*[int(x) for x in state_words])
        _lib.check(_lib.lib().vx_fri_chain_commit_async(self._h, ptrs, st, C.c_void_p(stream) if stream else None))

    def result(self, stream=None):
        """(roots [layers][8], alphas [layers][4], last [2][4]) after the stream drains."""
        nl = self.layers
        roots, alphas, last = (C.c_uint32 * (8 * nl))(), (C.c_uint32 * (4 * nl))(), (C.c_uint32 * 8)()
        _lib.check(_lib.lib().vx_fri_chain_fetch(self._h, roots, alphas, last, C.c_void_p(stream) if stream else None))
        return ([tuple(roots[8 * k: 8 * k + 8]) for k in range(nl)],
                [tuple(alphas[4 * k: 4 * k + 4]) for k in range(nl)],
                [tuple(last[0:4]), tuple(last[4:8])])

    def launches(self) -> int:
        return int(_lib.lib().vx_fri_chain_launches(self._h))

    def close(self) -> None:
        if self._h:
            _lib.lib().vx_fri_chain_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
