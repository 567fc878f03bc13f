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
    # the smallest size group (8 LDE rows), and eight size groups in the group combination
    ([2, 2, 3], 1, 6), ([2, 3, 4, 5, 6, 7, 8, 9], 2, 20),
    # size groups of 15..21 layers share one NTT launch per pass (up to four groups per launch); the others
    # run on their own: all merged, mixed, and more mergeable groups than one launch takes
    ([15] * 2 + [17] * 3 + [19] * 2, 2, 40),
    ([12] * 3 + [15] * 2 + [21], 1, 40),
    ([14] + [16] * 2 + [18] * 2 + [20] * 2 + [21] * 2, 1, 30),
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


def test_two_commitments_in_flight_on_two_streams(oracle):
    """Two contexts of one shape, each on its own stream with different
    columns, enqueued alternately without synchronising (the pipelined
    end-to-end loop): each context's words equal the oracle's for its own
    columns."""
    import torch

    logs = [10] * 3 + [12] * 4 + [14] * 2
    coms = [LiftedCommitter(logs, 2, 40) for _ in range(2)]
    streams = [torch.cuda.Stream() for _ in range(2)]
    cols = [_cols(40 + i, logs) for i in range(2)]
    pinned = [[torch.from_numpy(c.view(np.int32).copy()).pin_memory() for c in cs] for cs in cols]
    for _ in range(3):
        for com, st, pin in zip(coms, streams, pinned):
            com.upload_async([t.data_ptr() for t in pin], st.cuda_stream)
            com.commit_async(st.cuda_stream, graph=True)
            com.fetch_async(st.cuda_stream)
    torch.cuda.synchronize()
    for com, cs in zip(coms, cols):
        assert com.result_bytes() == oracle.commit_lifted(cs, 2, 40)
        com.close()


def _qm(rng, n):
    return rng.integers(0, P, (n, 4), dtype=np.uint32)


@pytest.mark.parametrize("log_n", [0, 1, 3, 10, 11, 12, 13, 16, 20, 21, 22, 23])
def test_eval_at_point_matches_oracle_and_reference(oracle, log_n):
    """cuda_eval_at_point (PolyOps::eval_at_point, poly_ops.rs:382-443)."""
    import ctypes as C
    rng = np.random.default_rng(40 + log_n)
    n = 1 << log_n
    coeffs = rng.integers(0, P, n, dtype=np.uint32)
    factors = _qm(rng, max(log_n, 1))
    want = oracle.eval_at_point(coeffs, factors[:log_n])
    d_c, d_f = to_dev(coeffs), to_dev(factors.reshape(-1))
    s1, s2 = empty(2 * n + 8), empty(2 * n + 8)
    res = (C.c_uint32 * 4)()
    _lib.clear_error()
    _lib.lib().cuda_eval_at_point(d_c.data_ptr(), d_f.data_ptr(), res, n, s1.data_ptr(), s2.data_ptr())
    _lib.raise_if_error()
    assert list(res) == want.tolist()
    if oracle.ref_available() and log_n >= 1:  # the reference's launcher needs n >= 2
        R = oracle.ref_lib()
        R.cuda_eval_at_point.argtypes = [C.c_void_p] * 3 + [C.c_uint32, C.c_void_p, C.c_void_p]
        ref = (C.c_uint32 * 4)()
        R.cuda_eval_at_point(d_c.data_ptr(), d_f.data_ptr(), ref, n, s1.data_ptr(), s2.data_ptr())
        assert list(ref) == want.tolist()


def test_eval_at_point_rejects_non_power_of_two():
    import ctypes as C
    d = empty(8)
    res = (C.c_uint32 * 4)()
    _lib.clear_error()
    _lib.lib().cuda_eval_at_point(d.data_ptr(), d.data_ptr(), res, 6, d.data_ptr(), d.data_ptr())
    with pytest.raises(_lib.VortexError):
        _lib.raise_if_error()


@pytest.mark.parametrize("n,n_blocks", [(1, 1), (255, 1), (1000, 3), (1 << 16, 64), (1 << 20, 256), (12345, 256)])
def test_barycentric_partials_match_oracle_and_reference(oracle, n, n_blocks):
    """cuda_barycentric_eval (poly_ops.rs:449-497): the per-block partial sums."""
    import ctypes as C
    rng = np.random.default_rng(n + n_blocks)
    evals = rng.integers(0, P, n, dtype=np.uint32)
    weights = _qm(rng, n)
    want = oracle.barycentric_partials(evals, weights, n_blocks)
    d_e, d_w, out = to_dev(evals), to_dev(weights.reshape(-1)), empty(4 * n_blocks)
    _lib.clear_error()
    _lib.lib().cuda_barycentric_eval(d_e.data_ptr(), d_w.data_ptr(), n, out.data_ptr(), n_blocks)
    _lib.raise_if_error()
    assert np.array_equal(to_host(out, 4 * n_blocks).reshape(-1, 4), want)
    if oracle.ref_available():
        R = oracle.ref_lib()
        R.cuda_barycentric_eval.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32]
        out2 = empty(4 * n_blocks)
        R.cuda_barycentric_eval(d_e.data_ptr(), d_w.data_ptr(), n, out2.data_ptr(), n_blocks)
        assert np.array_equal(to_host(out2, 4 * n_blocks).reshape(-1, 4), want)


def test_gathers_and_forge_aliases(oracle):
    """cuda_gather_u32 / _u256 (gather.cu) and their bounded _forge forms;
    cuda_bit_reverse_qm31_forge == cuda_bit_reverse_qm31."""
    import ctypes as C
    L = _lib.lib()
    rng = np.random.default_rng(9)
    src = rng.integers(0, 1 << 32, 5000, dtype=np.uint64).astype(np.uint32)
    idx = rng.integers(0, 5000, 777, dtype=np.uint32)
    d_src, d_idx = to_dev(src), to_dev(idx)
    out = empty(777)
    L.cuda_gather_u32(d_src.data_ptr(), d_idx.data_ptr(), out.data_ptr(), 777)
    assert np.array_equal(to_host(out, 777), src[idx])
    idx8 = rng.integers(0, 5000 // 8, 300, dtype=np.uint32)
    d_idx8 = to_dev(idx8)
    out8 = empty(8 * 300)
    L.cuda_gather_u256(d_src.data_ptr(), d_idx8.data_ptr(), out8.data_ptr(), 300)
    want8 = src[: (5000 // 8) * 8].reshape(-1, 8)[idx8].reshape(-1)
    assert np.array_equal(to_host(out8, 8 * 300), want8)
    # bounded forms: in-range the same, out-of-range elements left as they were
    bad = idx.copy()
    bad[::5] = 6000
    d_bad = to_dev(bad)
    outf = to_dev(np.full(777, 0xABCD, np.uint32))
    L.cuda_gather_u32_forge(d_src.data_ptr(), d_bad.data_ptr(), outf.data_ptr(), 777, 5000)
    got = to_host(outf, 777)
    ok = bad < 5000
    assert np.array_equal(got[ok], src[bad[ok]]) and (got[~ok] == 0xABCD).all()
    outf8 = empty(8 * 300)
    L.cuda_gather_u256_forge(d_src.data_ptr(), d_idx8.data_ptr(), outf8.data_ptr(), 300, 5000)
    assert np.array_equal(to_host(outf8, 8 * 300), want8)
    if oracle.ref_available():
        R = oracle.ref_lib()
        R.cuda_gather_u32.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32]
        out_r = empty(777)
        R.cuda_gather_u32(d_src.data_ptr(), d_idx.data_ptr(), out_r.data_ptr(), 777)
        assert np.array_equal(to_host(out_r, 777), src[idx])
    q = rng.integers(0, P, 4 * 1024, dtype=np.uint32)
    a, b = empty(4 * 1024), empty(4 * 1024)
    dq = to_dev(q)
    L.cuda_bit_reverse_qm31(dq.data_ptr(), a.data_ptr(), 1024, 10)
    L.cuda_bit_reverse_qm31_forge(dq.data_ptr(), b.data_ptr(), 1024, 10)
    assert np.array_equal(to_host(a), to_host(b))


def test_eval_and_barycentric_unaligned_inputs(oracle):
    """The scalar-load forms: coefficients and weights one word off 16-byte alignment."""
    import ctypes as C
    rng = np.random.default_rng(77)
    n = 1 << 13
    coeffs = rng.integers(0, P, n + 1, dtype=np.uint32)
    factors = _qm(rng, 13)
    d_c, d_f = to_dev(coeffs), to_dev(factors.reshape(-1))
    s1, s2 = empty(2 * n + 8), empty(2 * n + 8)
    res = (C.c_uint32 * 4)()
    _lib.clear_error()
    _lib.lib().cuda_eval_at_point(d_c.data_ptr() + 4, d_f.data_ptr(), res, n, s1.data_ptr(), s2.data_ptr())
    _lib.raise_if_error()
    assert list(res) == oracle.eval_at_point(coeffs[1:], factors).tolist()
    # an unaligned first scratch buffer takes the chunk fold
    _lib.lib().cuda_eval_at_point(d_c.data_ptr() + 4, d_f.data_ptr(), res, n, s1.data_ptr() + 4, s2.data_ptr())
    _lib.raise_if_error()
    assert list(res) == oracle.eval_at_point(coeffs[1:], factors).tolist()
    m = 5000
    evals = rng.integers(0, P, m, dtype=np.uint32)
    weights = rng.integers(0, P, 4 * m + 1, dtype=np.uint32)
    d_e, d_w, out = to_dev(evals), to_dev(weights), empty(4 * 7)
    _lib.lib().cuda_barycentric_eval(d_e.data_ptr(), d_w.data_ptr() + 4, m, out.data_ptr(), 7)
    _lib.raise_if_error()
    want = oracle.barycentric_partials(evals, weights[1:].reshape(m, 4), 7)
    assert np.array_equal(to_host(out, 28).reshape(-1, 4), want)
