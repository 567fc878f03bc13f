"""stwo-format launchers and the batched lifted commitment on the B200,
against the oracle and against the reference's own kernels (oracle/_ref)
on the same inputs and tables."""
import ctypes as C

import numpy as np
import pytest

from gpu_util import empty, to_dev, to_host
from vortexstark_b200 import _lib
from vortexstark_b200.lifted import LiftedCommitter, commit_lifted, verify_lifted

pytestmark = pytest.mark.gpu
P = 0x7FFFFFFF


def _rand(seed, n):
    return np.random.default_rng(seed).integers(0, P, n, dtype=np.uint32)


def _ref(oracle):
    if not oracle.ref_available():
        pytest.skip("oracle/_ref not built")
    R = oracle.ref_lib()
    vp, u32 = C.c_void_p, C.c_uint32
    R.cuda_stwo_ntt_evaluate.argtypes = [vp, vp, u32]
    R.cuda_stwo_ntt_interpolate.argtypes = [vp, vp, u32]
    R.cuda_stwo_ntt_batch_evaluate.argtypes = [vp, vp, u32, u32]
    R.cuda_stwo_ntt_batch_interpolate.argtypes = [vp, vp, u32, u32]
    R.cuda_bit_reverse_qm31.argtypes = [vp, vp, u32, u32]
    R.cuda_accumulate_lift.argtypes = [vp, vp, u32, u32]
    R.cuda_pack_leaves.argtypes = [vp, vp, u32]
    return R


@pytest.mark.parametrize("L", [2, 3, 5, 10, 16, 21])
def test_stwo_twiddles_built_on_device(oracle, L):
    for inv in (0, 1):
        out = empty(1 << (L - 1))
        _lib.check(_lib.lib().vx_stwo_twiddles(L, inv, out.data_ptr(), None))
        assert (to_host(out) == oracle.stwo_twiddles(L, bool(inv))).all(), (L, inv)


@pytest.mark.parametrize("L", [3, 8, 16, 22])
def test_stwo_fold_circle_twiddles_on_device(oracle, L):
    out = empty(1 << (L - 1))
    _lib.check(_lib.lib().vx_stwo_fold_circle_twiddles(L, out.data_ptr(), None))
    assert (to_host(out) == oracle.stwo_fold_circle_twiddles(L)).all()


@pytest.mark.parametrize("L", [2, 3, 4, 5, 8, 11, 12, 13, 14, 15, 16, 20, 22])
def test_stwo_ntt_matches_oracle(oracle, L):
    x = _rand(L, 1 << L)
    tw, itw = to_dev(oracle.stwo_twiddles(L)), to_dev(oracle.stwo_twiddles(L, True))
    d = to_dev(x)
    _lib.clear_error()
    _lib.lib().cuda_stwo_ntt_evaluate(d.data_ptr(), tw.data_ptr(), 1 << L)
    _lib.raise_if_error()
    ev = oracle.stwo_ntt_evaluate(x)
    assert (to_host(d) == ev).all()
    _lib.lib().cuda_stwo_ntt_interpolate(d.data_ptr(), itw.data_ptr(), 1 << L)
    _lib.raise_if_error()
    assert (to_host(d) == x).all()


@pytest.mark.parametrize("L", [4, 12, 17])
def test_stwo_ntt_batch_matches_oracle(oracle, L):
    cols = [_rand(100 * L + c, 1 << L) for c in range(5)]
    tw, itw = to_dev(oracle.stwo_twiddles(L)), to_dev(oracle.stwo_twiddles(L, True))
    ds = [to_dev(c) for c in cols]
    ptrs = (C.c_void_p * 5)(*[d.data_ptr() for d in ds])
    _lib.clear_error()
    _lib.lib().cuda_stwo_ntt_batch_evaluate(ptrs, tw.data_ptr(), 1 << L, 5)
    _lib.raise_if_error()
    for d, c in zip(ds, cols):
        assert (to_host(d) == oracle.stwo_ntt_evaluate(c)).all()
    _lib.lib().cuda_stwo_ntt_batch_interpolate(ptrs, itw.data_ptr(), 1 << L, 5)
    for d, c in zip(ds, cols):
        assert (to_host(d) == c).all()


def test_stwo_ntt_rejects_bad_sizes(oracle):
    tw = to_dev(oracle.stwo_twiddles(4))
    d = to_dev(_rand(1, 16))
    for n in (2, 24):
        _lib.clear_error()
        _lib.lib().cuda_stwo_ntt_evaluate(d.data_ptr(), tw.data_ptr(), n)
        with pytest.raises(_lib.VortexError):
            _lib.raise_if_error()


@pytest.mark.parametrize("L", [2, 4, 9, 10, 12, 16, 20])
def test_stwo_ntt_matches_reference_kernels(oracle, L):
    R = _ref(oracle)
    x = _rand(1000 + L, 1 << L)
    tw, itw = to_dev(oracle.stwo_twiddles(L)), to_dev(oracle.stwo_twiddles(L, True))
    ours, theirs = to_dev(x), to_dev(x)
    _lib.lib().cuda_stwo_ntt_evaluate(ours.data_ptr(), tw.data_ptr(), 1 << L)
    R.cuda_stwo_ntt_evaluate(theirs.data_ptr(), tw.data_ptr(), 1 << L)
    assert (to_host(ours) == to_host(theirs)).all()
    _lib.lib().cuda_stwo_ntt_interpolate(ours.data_ptr(), itw.data_ptr(), 1 << L)
    R.cuda_stwo_ntt_interpolate(theirs.data_ptr(), itw.data_ptr(), 1 << L)
    assert (to_host(ours) == to_host(theirs)).all() and (to_host(ours) == x).all()
    # batched, three columns
    cols = [_rand(2000 + L + c, 1 << L) for c in range(3)]
    a = [to_dev(c) for c in cols]
    b = [to_dev(c) for c in cols]
    pa = (C.c_void_p * 3)(*[t.data_ptr() for t in a])
    pb = (C.c_void_p * 3)(*[t.data_ptr() for t in b])
    _lib.lib().cuda_stwo_ntt_batch_evaluate(pa, tw.data_ptr(), 1 << L, 3)
    R.cuda_stwo_ntt_batch_evaluate(pb, tw.data_ptr(), 1 << L, 3)
    for s, t in zip(a, b):
        assert (to_host(s) == to_host(t)).all()


@pytest.mark.parametrize("L", [1, 4, 9, 10, 11, 16, 21])
def test_bit_reverse_qm31(oracle, L):
    x = _rand(3000 + L, 4 << L)
    src, dst = to_dev(x), empty(4 << L)
    _lib.clear_error()
    _lib.lib().cuda_bit_reverse_qm31(src.data_ptr(), dst.data_ptr(), 1 << L, L)
    _lib.raise_if_error()
    want = oracle.bit_reverse_qm31(x)
    assert (to_host(dst) == want).all()
    if oracle.ref_available():
        R = _ref(oracle)
        d2 = empty(4 << L)
        R.cuda_bit_reverse_qm31(src.data_ptr(), d2.data_ptr(), 1 << L, L)
        assert (to_host(d2) == want).all()


def test_bit_reverse_qm31_unaligned(oracle):
    L = 12
    x = _rand(11, (4 << L) + 1)
    src, dst = to_dev(x), empty((4 << L) + 1)
    # one word in: not 16-byte aligned, the untiled kernel runs
    _lib.lib().cuda_bit_reverse_qm31(src.data_ptr() + 4, dst.data_ptr() + 4, 1 << L, L)
    assert (to_host(dst)[1:] == oracle.bit_reverse_qm31(x[1:])).all()


@pytest.mark.parametrize("col_log,ratio", [(4, 0), (10, 1), (12, 3), (20, 2), (21, 6)])
def test_accumulate_lift(oracle, col_log, ratio):
    col = _rand(4000 + col_log, 1 << col_log)
    curr = _rand(5000 + ratio, 1 << (col_log - ratio))
    want = oracle.accumulate_lift(col, curr)
    dc, ds = to_dev(col), to_dev(curr)
    _lib.lib().cuda_accumulate_lift(dc.data_ptr(), ds.data_ptr(), 1 << col_log, ratio)
    assert (to_host(dc) == want).all()
    # an odd length runs the scalar kernel
    dc2 = to_dev(col)
    _lib.lib().cuda_accumulate_lift(dc2.data_ptr(), ds.data_ptr(), (1 << col_log) - 1, ratio)
    got = to_host(dc2)
    assert (got[:-1] == want[:-1]).all() and got[-1] == col[-1]
    if oracle.ref_available():
        R = _ref(oracle)
        dc3 = to_dev(col)
        R.cuda_accumulate_lift(dc3.data_ptr(), ds.data_ptr(), 1 << col_log, ratio)
        assert (to_host(dc3) == want).all()


@pytest.mark.parametrize("n", [16, 48, 1024, (1 << 20) + 16])
def test_pack_leaves(oracle, n):
    import torch

    cols = [_rand(6000 + n + c, n) for c in range(4)]
    want = oracle.pack_leaves(cols)
    ins = [to_dev(c) for c in cols]
    outs = [empty(n // 16) for _ in range(64)]
    pin = torch.tensor([t.data_ptr() for t in ins], dtype=torch.int64, device="cuda")
    pout = torch.tensor([t.data_ptr() for t in outs], dtype=torch.int64, device="cuda")
    _lib.lib().cuda_pack_leaves(pin.data_ptr(), pout.data_ptr(), n)
    for i in range(64):
        assert (to_host(outs[i], n // 16) == want[i]).all(), i
    if oracle.ref_available():
        R = _ref(oracle)
        outs2 = [empty(n // 16) for _ in range(64)]
        pout2 = torch.tensor([t.data_ptr() for t in outs2], dtype=torch.int64, device="cuda")
        R.cuda_pack_leaves(pin.data_ptr(), pout2.data_ptr(), n)
        for i in range(64):
            assert (to_host(outs2[i], n // 16) == want[i]).all(), i


def _cols(seed, logs):
    rng = np.random.default_rng(seed)
    return [rng.integers(0, P, 1 << L, dtype=np.uint32) for L in logs]


@pytest.mark.parametrize("logs,B,nq", [
    ([2], 2, 8), ([3, 3], 1, 5), ([4, 4, 6], 2, 16), ([2, 5, 7], 3, 33), ([6] * 8, 2, 80),
    ([8] * 8 + [10] * 16 + [12] * 10, 2, 80),
    ([5] * 17 + [9] * 20, 2, 40),
])
def test_commit_lifted_matches_oracle(oracle, logs, B, nq):
    cols = _cols(sum(logs) + B, logs)
    got = commit_lifted(cols, B, nq)
    assert got == oracle.commit_lifted(cols, B, nq)
    verify_lifted(got, nq)


def test_commit_lifted_graph_and_uploads(oracle):
    import torch

    logs = [7] * 4 + [9] * 6 + [11] * 3
    com = LiftedCommitter(logs, 2, 80)
    stream = torch.cuda.Stream()
    for seed in (1, 2):
        cols = _cols(seed, logs)
        pinned = [torch.from_numpy(c.view(np.int32).copy()).pin_memory() for c in cols]
        for graph in (False, True, True):
            com.upload_async([t.data_ptr() for t in pinned], stream.cuda_stream)
            com.commit_async(stream.cuda_stream, graph=graph)
            com.fetch_async(stream.cuda_stream)
            stream.synchronize()
            assert com.result_bytes() == oracle.commit_lifted(cols, 2, 80), (seed, graph)
        # the uploaded column is where vx_lifted_column says
        probe = torch.empty(1 << logs[0], dtype=torch.int32, device="cuda")
        assert com.column_ptr(0) != 0 and probe.numel() == len(cols[0])
    assert com.launches() > 0 and com.device_bytes() > 0
    com.close()
