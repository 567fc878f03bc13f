"""Circle NTT on the B200: evaluate / interpolate with cached twiddles.

Mirrors src/ntt.rs: ``TwiddleCache`` / ``ForwardTwiddleCache`` /
``InverseTwiddleCache`` (ntt.rs:10-91), ``evaluate`` / ``interpolate``
(145-180), ``bit_reverse`` (183-188) and the batched forms (191-281).  Data
are device tensors of u32 words (int32 storage), transformed in place.
"""
from __future__ import annotations

import ctypes as C

from . import _lib
from .circle import Coset, compute_forward_twiddles_gpu, compute_inverse_twiddles_gpu


def _host_u32(vals):
    arr = (C.c_uint32 * max(len(vals), 1))(*vals)
    return arr


class ForwardTwiddleCache:
    def __init__(self, coset: Coset):
        self.log_n = coset.log_size
        self.d_twiddles, self.d_circle_twids, self.layer_offsets, self.layer_sizes = compute_forward_twiddles_gpu(coset)


class InverseTwiddleCache:
    def __init__(self, coset: Coset):
        self.log_n = coset.log_size
        self.d_itwiddles, self.d_circle_itwids, self.layer_offsets, self.layer_sizes = compute_inverse_twiddles_gpu(coset)


class TwiddleCache:
    def __init__(self, coset: Coset):
        f = ForwardTwiddleCache(coset)
        i = InverseTwiddleCache(coset)
        self.log_n = coset.log_size
        self.d_twiddles, self.d_circle_twids = f.d_twiddles, f.d_circle_twids
        self.d_itwiddles, self.d_circle_itwids = i.d_itwiddles, i.d_circle_itwids
        self.layer_offsets, self.layer_sizes = f.layer_offsets, f.layer_sizes


def evaluate(d_data, cache) -> None:
    """ntt.rs:145-161 — coefficients -> values, in place."""
    n = 1 << cache.log_n
    nl = max(cache.log_n - 1, 0)
    _lib.lib().cuda_circle_ntt_evaluate(d_data.data_ptr(), cache.d_twiddles.data_ptr(), cache.d_circle_twids.data_ptr(),
                                        _host_u32(cache.layer_offsets), _host_u32(cache.layer_sizes), nl, n)


def interpolate(d_data, cache) -> None:
    """ntt.rs:164-180 — values -> coefficients (with the 1/n scale), in place."""
    n = 1 << cache.log_n
    nl = max(cache.log_n - 1, 0)
    _lib.lib().cuda_circle_ntt_interpolate(d_data.data_ptr(), cache.d_itwiddles.data_ptr(),
                                           cache.d_circle_itwids.data_ptr(), _host_u32(cache.layer_offsets),
                                           _host_u32(cache.layer_sizes), nl, n)


def _ptr_array(cols):
    import torch

    return torch.tensor([c.data_ptr() for c in cols], dtype=torch.int64, device=cols[0].device)


def evaluate_batch(columns, cache) -> None:
    """ntt.rs:191-236 — forward NTT of equal-size columns."""
    if not columns:
        return
    ptrs = _ptr_array(columns)
    n = 1 << cache.log_n
    _lib.lib().cuda_circle_ntt_evaluate_batch(ptrs.data_ptr(), cache.d_twiddles.data_ptr(),
                                              cache.d_circle_twids.data_ptr(), _host_u32(cache.layer_offsets),
                                              _host_u32(cache.layer_sizes), max(cache.log_n - 1, 0), n, len(columns))


def interpolate_batch(columns, cache) -> None:
    """ntt.rs:238-281 — inverse NTT of equal-size columns."""
    if not columns:
        return
    ptrs = _ptr_array(columns)
    n = 1 << cache.log_n
    _lib.lib().cuda_circle_ntt_interpolate_batch(ptrs.data_ptr(), cache.d_itwiddles.data_ptr(),
                                                 cache.d_circle_itwids.data_ptr(), _host_u32(cache.layer_offsets),
                                                 _host_u32(cache.layer_sizes), max(cache.log_n - 1, 0), n,
                                                 len(columns))


def bit_reverse(d_data, log_n: int) -> None:
    """ntt.rs:183-188"""
    _lib.lib().cuda_bit_reverse_m31(d_data.data_ptr(), log_n)
    _lib.lib().cuda_device_sync()


def permute_hc_to_canonic_brt(src, dst, log_n: int) -> None:
    _lib.lib().cuda_permute_hc_to_canonic_brt(src.data_ptr(), dst.data_ptr(), 1 << log_n, log_n)


def permute_canonic_brt_to_hc_natural(src, dst, log_n: int) -> None:
    _lib.lib().cuda_permute_canonic_brt_to_hc_natural(src.data_ptr(), dst.data_ptr(), 1 << log_n, log_n)


# ---- stwo format (ntt.rs:288-379, circle_ntt_stwo.cu, circle_ntt_stwo_batch.cu) ----
class StwoNttCache:
    """ntt.rs:288-362 — stwo twiddles of CanonicCoset(log_n)'s circle domain
    (the layout of CpuBackend::precompute_twiddles), built on the device
    (vx_stwo_twiddles) instead of on the CPU and uploaded."""

    def __init__(self, log_n: int):
        import torch

        self.log_n = log_n
        half = 1 << (log_n - 1)
        self.d_fwd_twiddles = torch.empty(half, dtype=torch.int32, device="cuda")
        self.d_inv_twiddles = torch.empty(half, dtype=torch.int32, device="cuda")
        L = _lib.lib()
        _lib.check(L.vx_stwo_twiddles(log_n, 0, self.d_fwd_twiddles.data_ptr(), None))
        _lib.check(L.vx_stwo_twiddles(log_n, 1, self.d_inv_twiddles.data_ptr(), None))
        torch.cuda.synchronize()


def evaluate_stwo(d_data, cache: StwoNttCache) -> None:
    """ntt.rs:365-371 — coefficients -> values in bit-reversed circle-domain order."""
    _lib.clear_error()
    _lib.lib().cuda_stwo_ntt_evaluate(d_data.data_ptr(), cache.d_fwd_twiddles.data_ptr(), 1 << cache.log_n)
    _lib.raise_if_error()


def interpolate_stwo(d_data, cache: StwoNttCache) -> None:
    """ntt.rs:373-379 — values -> coefficients (with the 1/n scale)."""
    _lib.clear_error()
    _lib.lib().cuda_stwo_ntt_interpolate(d_data.data_ptr(), cache.d_inv_twiddles.data_ptr(), 1 << cache.log_n)
    _lib.raise_if_error()


def _host_ptrs(cols):
    return (C.c_void_p * len(cols))(*[c.data_ptr() for c in cols])


def evaluate_stwo_batch(columns, cache: StwoNttCache) -> None:
    """poly_ops.rs:676-770 (cuda_stwo_ntt_batch_evaluate) — equal-size columns."""
    if columns:
        _lib.clear_error()
        _lib.lib().cuda_stwo_ntt_batch_evaluate(_host_ptrs(columns), cache.d_fwd_twiddles.data_ptr(),
                                                1 << cache.log_n, len(columns))
        _lib.raise_if_error()


def interpolate_stwo_batch(columns, cache: StwoNttCache) -> None:
    """poly_ops.rs:772-830 (cuda_stwo_ntt_batch_interpolate) — equal-size columns."""
    if columns:
        _lib.clear_error()
        _lib.lib().cuda_stwo_ntt_batch_interpolate(_host_ptrs(columns), cache.d_inv_twiddles.data_ptr(),
                                                   1 << cache.log_n, len(columns))
        _lib.raise_if_error()
