"""Every reference-compatible launcher of libvortex_b200 against the oracle.

Bit-exact equality on seeded inputs (all arithmetic is exact integer work).
"""
import ctypes as C

import numpy as np
import pytest

from gpu_util import empty, to_dev, to_host
from vortexstark_b200 import _lib
from vortexstark_b200.workload import m31_array

pytestmark = pytest.mark.gpu
P = 0x7FFFFFFF


@pytest.fixture(scope="module")
def L():
    # test_no_launch_errors checks the launch errors of this module's tests
    # only: clear what earlier modules left (some test rejected arguments)
    _lib.lib().vx_clear_error()
    return _lib.lib()


def _cos(oracle, kind, k):
    from vortexstark_b200.circle import Coset
    pc = {"half_coset": Coset.half_coset, "half_odds": Coset.half_odds, "subgroup": Coset.subgroup}[kind](k)
    return pc, oracle.coset(kind, k)


@pytest.mark.parametrize("kind", ["half_coset", "half_odds", "subgroup"])
@pytest.mark.parametrize("k", [1, 2, 3, 5, 8, 12])
def test_twiddle_tables(oracle, kind, k):
    from vortexstark_b200.circle import compute_forward_twiddles_gpu, compute_inverse_twiddles_gpu
    pc, oc = _cos(oracle, kind, k)
    line, circ, offs, sizes = compute_forward_twiddles_gpu(pc)
    oline, ocirc, ooffs = oracle.twiddles(oc, False)
    assert np.array_equal(to_host(circ, 1 << (k - 1)), ocirc)
    # the flat line table has 2^k - 1 slots of which the layers fill 2^k - 2
    # (circle.rs:479); the last slot is never written or read
    assert np.array_equal(to_host(line, (1 << k) - 2), oline[:(1 << k) - 2])
    assert list(offs) == ooffs.tolist()
    il, ic, _, _ = compute_inverse_twiddles_gpu(pc)
    oil, oic, _ = oracle.twiddles(oc, True)
    assert np.array_equal(to_host(ic, 1 << (k - 1)), oic)
    assert np.array_equal(to_host(il, (1 << k) - 2), oil[:(1 << k) - 2])


@pytest.mark.parametrize("kind", ["half_coset", "half_odds", "subgroup"])
@pytest.mark.parametrize("k", [1, 2, 4, 7, 11, 12, 13, 16, 20])
def test_ntt_evaluate_interpolate(oracle, kind, k):
    from vortexstark_b200 import ntt
    pc, oc = _cos(oracle, kind, k)
    cache = ntt.TwiddleCache(pc)
    x = m31_array(1000 + k, 1 << k)
    d = to_dev(x)
    ntt.evaluate(d, cache)
    ev = to_host(d)
    assert np.array_equal(ev, oracle.ntt_evaluate(x, oc))
    ntt.interpolate(d, cache)
    assert np.array_equal(to_host(d), oracle.ntt_interpolate(ev, oc))
    if kind == "half_coset":
        assert np.array_equal(to_host(d), x)  # round trip (ntt.rs:386-449)


def test_ntt_large_round_trip(oracle):
    from vortexstark_b200 import ntt
    from vortexstark_b200.circle import Coset
    k = 24
    cache = ntt.TwiddleCache(Coset.half_coset(k))
    x = m31_array(24, 1 << k)
    d = to_dev(x)
    ntt.evaluate(d, cache)
    ev = to_host(d)
    assert np.array_equal(ev[:4096], oracle.ntt_evaluate(x, oracle.coset("half_coset", k))[:4096])
    ntt.interpolate(d, cache)
    assert np.array_equal(to_host(d), x)


@pytest.mark.parametrize("k", [6, 13])
def test_ntt_batch(oracle, k):
    from vortexstark_b200 import ntt
    pc, oc = _cos(oracle, "half_coset", k)
    cache = ntt.TwiddleCache(pc)
    xs = [m31_array(50 + i, 1 << k) for i in range(5)]
    ds = [to_dev(x) for x in xs]
    ntt.evaluate_batch(ds, cache)
    evs = [to_host(d) for d in ds]
    for x, e in zip(xs, evs):
        assert np.array_equal(e, oracle.ntt_evaluate(x, oc))
    ntt.interpolate_batch(ds, cache)
    for x, d in zip(xs, ds):
        assert np.array_equal(to_host(d), x)


def test_ntt_single_layers(oracle, L):
    """prover.rs:2491-2574 through cuda_circle_ntt_layer."""
    from vortexstark_b200.circle import Coset, compute_forward_twiddles_gpu
    k = 10
    line, circ, offs, sizes = compute_forward_twiddles_gpu(Coset.half_coset(k))
    x = m31_array(7, 1 << k)
    d = to_dev(x)
    for l in range(k - 2, -1, -1):
        L.cuda_circle_ntt_layer(d.data_ptr(), line.data_ptr() + 4 * offs[l], l + 1, 1 << k, 1)
    L.cuda_circle_ntt_layer(d.data_ptr(), circ.data_ptr(), 0, 1 << k, 1)
    assert np.array_equal(to_host(d), oracle.ntt_evaluate(x, oracle.coset("half_coset", k)))


@pytest.mark.parametrize("k", [1, 5, 9, 10, 11, 12, 13, 17, 22])
def test_bit_reverse_and_permute(oracle, L, k):
    x = m31_array(k, 1 << k)
    d = to_dev(x)
    L.cuda_bit_reverse_m31(d.data_ptr(), k)
    assert np.array_equal(to_host(d), oracle.bit_reverse(x))
    s, t = to_dev(x), empty(1 << k)
    L.cuda_permute_hc_to_canonic_brt(s.data_ptr(), t.data_ptr(), 1 << k, k)
    assert np.array_equal(to_host(t, 1 << k), oracle.permute_hc_to_canonic_brt(x))
    u = empty(1 << k)
    L.cuda_permute_canonic_brt_to_hc_natural(t.data_ptr(), u.data_ptr(), 1 << k, k)
    assert np.array_equal(to_host(u, 1 << k), x)


def test_batch_inverse(oracle, L):
    x = m31_array(5, 10000)
    x[0] = 0
    x[640] = 0
    x[777] = 0
    x[9999] = 0
    d, o = to_dev(x), empty(len(x))
    L.cuda_batch_inverse_m31(d.data_ptr(), o.data_ptr(), len(x))
    assert np.array_equal(to_host(o, len(x)), oracle.batch_inverse(x))


@pytest.mark.parametrize("n", [1, 63, 64, 65, 4095, 4096, 4097, 8192 + 64, (1 << 20) + 3])
def test_batch_inverse_sizes_and_in_place(oracle, L, n):
    """Chunk (64) and block (4096) boundaries, zeros in first and other slots, in place."""
    x = m31_array(90 + n % 1000, n)
    x[::97] = 0
    want = oracle.batch_inverse(x)
    d, o = to_dev(x), empty(n)
    L.cuda_batch_inverse_m31(d.data_ptr(), o.data_ptr(), n)
    assert np.array_equal(to_host(o, n), want)
    L.cuda_batch_inverse_m31(d.data_ptr(), d.data_ptr(), n)
    assert np.array_equal(to_host(d, n), want)


@pytest.mark.parametrize("kind,ey", [("half_coset", 1), ("half_odds", 0), ("subgroup", 1), ("half_coset", 0)])
@pytest.mark.parametrize("k", [2, 7, 15])
def test_fold_twiddles(oracle, kind, ey, k):
    from vortexstark_b200.fri import compute_fold_twiddles_on_demand
    pc, oc = _cos(oracle, kind, k)
    got = to_host(compute_fold_twiddles_on_demand(pc, bool(ey)), 1 << (k - 1))
    assert np.array_equal(got, oracle.fold_twiddles(oc, bool(ey)))


def test_zero_pad_and_quotient(oracle, L):
    n, N = 1 << 10, 1 << 12
    x = m31_array(3, n)
    s, d = to_dev(x), empty(N)
    L.cuda_zero_pad(s.data_ptr(), d.data_ptr(), n, N)
    pad = to_host(d, N)
    assert np.array_equal(pad[:n], x) and not pad[n:].any()
    ev = m31_array(4, N)
    alpha = (123, 456, 789, 1011)
    dev = to_dev(ev)
    q = [empty(N) for _ in range(4)]
    L.cuda_fibonacci_quotient(dev.data_ptr(), *[c.data_ptr() for c in q], (C.c_uint32 * 4)(*alpha), N)
    want = oracle.fibonacci_quotient(ev, alpha)
    for c in range(4):
        assert np.array_equal(to_host(q[c], N), want[c])
    qc = [empty(512) for _ in range(4)]
    L.cuda_fibonacci_quotient_chunk(dev.data_ptr(), *[c.data_ptr() for c in qc], (C.c_uint32 * 4)(*alpha), N - 512,
                                    512, N)
    for c in range(4):
        assert np.array_equal(to_host(qc[c], 512), want[c][N - 512:])


@pytest.mark.parametrize("n,N,shift", [(1, 1, 0), (5, 13, 0), (1024, 4096, 0), (1001, 4099, 0), (6, 11, 1)])
def test_zero_pad_sizes(L, n, N, shift):
    """Ragged lengths, a straddling group, and an unaligned (word-offset) source and destination."""
    x = m31_array(70 + n, n + shift)
    s, d = to_dev(x), to_dev(np.full(N + shift, 0xDEAD, np.uint32))
    L.cuda_zero_pad(s.data_ptr() + 4 * shift, d.data_ptr() + 4 * shift, n, N)
    got = to_host(d, N + shift)[shift:]
    assert np.array_equal(got[:n], x[shift:shift + n]) and not got[n:].any()


def test_quotient_chunk_unaligned(oracle, L):
    """A chunk whose offset and length are not multiples of 4 (the scalar form), ending at the wrap."""
    N = 1000
    ev = m31_array(61, N)
    alpha = (9, 10, 11, 12)
    dev = to_dev(ev)
    want = oracle.fibonacci_quotient(ev, alpha)
    for off, cnt in ((3, 10), (N - 7, 7), (0, 999)):
        q = [empty(cnt) for _ in range(4)]
        L.cuda_fibonacci_quotient_chunk(dev.data_ptr(), *[c.data_ptr() for c in q], (C.c_uint32 * 4)(*alpha), off,
                                        cnt, N)
        for c in range(4):
            assert np.array_equal(to_host(q[c], cnt), want[c][off:off + cnt])


@pytest.mark.parametrize("N", [1, 2, 3, 5])
def test_quotient_tiny_domains(oracle, L, N):
    """(i + 1) mod N and (i + 2) mod N where i + 2 can pass 2N."""
    ev = m31_array(40 + N, N)
    alpha = (5, 6, 7, 8)
    dev = to_dev(ev)
    q = [empty(N) for _ in range(4)]
    L.cuda_fibonacci_quotient(dev.data_ptr(), *[c.data_ptr() for c in q], (C.c_uint32 * 4)(*alpha), N)
    want = oracle.fibonacci_quotient(ev, alpha)
    for c in range(4):
        assert np.array_equal(to_host(q[c], N), want[c])


def _ptrs(ts):
    import torch
    return torch.tensor([t.data_ptr() for t in ts], dtype=torch.int64, device="cuda")


def _tree_levels(oracle, cols):
    """Oracle leaf and node hashes level by level (list of (n, 8) arrays)."""
    from oracle import pyoracle as Y
    nc = min(len(cols), 16)
    leaves = np.array([Y.leaf([int(c[i]) for c in cols[:nc]]) for i in range(len(cols[0]))], np.uint32)
    levels = [leaves]
    while len(levels[-1]) > 1:
        lv = levels[-1]
        levels.append(np.array([Y.node(list(lv[2 * i]), list(lv[2 * i + 1])) for i in range(len(lv) // 2)], np.uint32))
    return levels


@pytest.mark.parametrize("ncols", [1, 2, 4, 7, 8, 16, 20])
def test_merkle_leaves_nodes(oracle, L, ncols):
    n = 256
    cols = [m31_array(100 * ncols + i, n) for i in range(ncols)]
    dcols = [to_dev(c) for c in cols]
    lv = _tree_levels(oracle, cols)
    out = empty(8 * n)
    L.cuda_merkle_hash_leaves(_ptrs(dcols).data_ptr(), out.data_ptr(), ncols, n)
    assert np.array_equal(to_host(out).reshape(-1, 8), lv[0])
    if ncols in (1, 4):
        o2 = empty(8 * n)
        if ncols == 1:
            L.cuda_merkle_hash_leaves_forge_single(dcols[0].data_ptr(), o2.data_ptr(), n)
        else:
            L.cuda_merkle_hash_leaves_forge_quad(*[c.data_ptr() for c in dcols], o2.data_ptr(), n)
        assert np.array_equal(to_host(o2).reshape(-1, 8), lv[0])
    par = empty(4 * n)
    L.cuda_merkle_hash_nodes(out.data_ptr(), par.data_ptr(), n // 2)
    assert np.array_equal(to_host(par).reshape(-1, 8), lv[1])
    root = empty(8)
    L.cuda_merkle_reduce_to_root(par.data_ptr(), root.data_ptr(), n // 2)
    assert np.array_equal(to_host(root, 8), lv[-1][0])


def test_merkle_soa4_variants(oracle, L):
    n = 2048
    cols = [m31_array(900 + i, n) for i in range(4)]
    d = [to_dev(c) for c in cols]
    lv = _tree_levels(oracle, cols)
    root = empty(8)
    L.cuda_merkle_commit_small_soa4(*[c.data_ptr() for c in d], root.data_ptr(), n)
    assert np.array_equal(to_host(root, 8), lv[-1][0])
    par = empty(4 * n)
    L.cuda_merkle_hash_leaves_merge_soa4(*[c.data_ptr() for c in d], par.data_ptr(), n)
    assert np.array_equal(to_host(par).reshape(-1, 8), lv[1])
    sub = empty(16)
    L.cuda_merkle_tiled_soa4(*[c.data_ptr() for c in d], sub.data_ptr(), n)
    assert np.array_equal(to_host(sub).reshape(-1, 8), lv[10])
    sub2 = empty(16)
    L.cuda_merkle_tiled_generic(_ptrs(d).data_ptr(), sub2.data_ptr(), 4, n)
    assert np.array_equal(to_host(sub2).reshape(-1, 8), lv[10])


@pytest.mark.parametrize("ncols", [1, 2, 3, 8])
def test_merkle_tiled_generic_column_counts(oracle, L, ncols):
    """1024-leaf subtree roots for the compile-time column counts and the generic fallback (3)."""
    n = 4096
    cols = [m31_array(300 + 10 * ncols + i, n) for i in range(ncols)]
    d = [to_dev(c) for c in cols]
    lv = _tree_levels(oracle, cols)
    sub = empty(8 * (n // 1024))
    L.cuda_merkle_tiled_generic(_ptrs(d).data_ptr(), sub.data_ptr(), ncols, n)
    assert np.array_equal(to_host(sub).reshape(-1, 8), lv[10])


@pytest.mark.parametrize("log_n,ncols", [(12, 1), (16, 4), (20, 1)])
def test_merkle_tree_root_and_paths(oracle, log_n, ncols):
    from vortexstark_b200.merkle import MerkleTree, hash_leaf, verify_auth_path
    cols = [m31_array(7 * log_n + i, 1 << log_n) for i in range(ncols)]
    d = [to_dev(c) for c in cols]
    want = oracle.merkle_root(cols)
    r1, subs = MerkleTree.commit_root_only_with_subtrees(d, log_n)
    assert r1 == tuple(want.tolist())
    t = MerkleTree.commit(d, log_n)
    assert t.root() == tuple(want.tolist())
    idx = [0, 1, 5, (1 << log_n) - 1, 12345 % (1 << log_n)]
    for i, pth in zip(idx, t.batch_auth_paths(idx)):
        assert verify_auth_path(want.tolist(), hash_leaf([int(c[i]) for c in cols]), i, pth)


def test_lifted_leaves(oracle):
    from vortexstark_b200.merkle import build_leaves_lifted
    sizes = [6] * 3 + [8] * 17 + [10] * 14   # 34 columns, ascending sizes
    cols = [m31_array(300 + i, 1 << s) for i, s in enumerate(sizes)]
    out = build_leaves_lifted([to_dev(c) for c in cols], 10)
    assert np.array_equal(to_host(out).reshape(-1, 8), oracle.lifted_leaves(cols, 10))


@pytest.mark.parametrize("k", [2, 3, 4, 9, 16, 20])
def test_folds(oracle, k):
    from vortexstark_b200 import fri
    from vortexstark_b200.circle import Coset
    src = np.stack([m31_array(40 * k + c, 1 << k) for c in range(4)])
    alpha = (42, 99, 7, 13)
    col = fri.SecureColumn.from_words(src)
    tw = fri.compute_fold_twiddles_on_demand(Coset.half_odds(k), False)
    out = fri.fold_line_with_twiddles(col, alpha, tw)
    want = oracle.fold_line(src, oracle.fold_twiddles(oracle.coset("half_odds", k), False), alpha)
    assert np.array_equal(out.to_words(), want)
    dst = fri.SecureColumn.zeros(1 << (k - 1))
    twc = fri.compute_fold_twiddles_on_demand(Coset.half_coset(k), True)
    fri.fold_circle_into_line_with_twiddles(dst, col, alpha, twc)
    wantc = oracle.fold_circle_into_line(np.zeros((4, 1 << (k - 1)), np.uint32), src,
                                         oracle.fold_twiddles(oracle.coset("half_coset", k), True), alpha)
    assert np.array_equal(dst.to_words(), wantc)
    # accumulate into a non-zero destination (dst * alpha^2 + f')
    prev = np.stack([m31_array(7 + c, 1 << (k - 1)) for c in range(4)])
    dst2 = fri.SecureColumn.from_words(prev)
    fri.fold_circle_into_line_with_twiddles(dst2, col, alpha, twc)
    want2 = oracle.fold_circle_into_line(prev, src, oracle.fold_twiddles(oracle.coset("half_coset", k), True), alpha)
    assert np.array_equal(dst2.to_words(), want2)


def test_folds_unaligned_match_aligned(oracle, L):
    """The scalar fold kernels (pointers only 4-byte aligned) and the
    vectorised ones give the same words."""
    import ctypes as C

    import torch

    k = 12
    src = np.stack([m31_array(900 + c, 1 << k) for c in range(4)])
    tw = np.asarray(oracle.fold_twiddles(oracle.coset("half_odds", k), False), np.uint32)
    want = oracle.fold_line(src, tw, (5, 6, 7, 8))
    alpha = (C.c_uint32 * 4)(5, 6, 7, 8)
    for off in (0, 1):
        ins = [torch.from_numpy(np.concatenate([np.zeros(off, np.uint32), c]).view(np.int32)).cuda() for c in src]
        t = torch.from_numpy(np.concatenate([np.zeros(off, np.uint32), tw]).view(np.int32)).cuda()
        outs = [torch.zeros((1 << (k - 1)) + off, dtype=torch.int32, device="cuda") for _ in range(4)]
        L.cuda_fold_line_soa(*[x.data_ptr() + 4 * off for x in ins], t.data_ptr() + 4 * off,
                             *[o.data_ptr() + 4 * off for o in outs], alpha, 1 << (k - 1))
        got = np.stack([to_host(o)[off:] for o in outs])
        assert np.array_equal(got, want), off


def test_no_launch_errors(L):
    import torch
    torch.cuda.synchronize()
    assert _lib.last_error() == ""


@pytest.mark.parametrize("log_n,ncols", [(1, 1), (4, 4), (12, 1), (12, 3), (17, 1), (18, 4), (20, 16), (21, 1)])
def test_fused_root_only_commit(oracle, log_n, ncols):
    """vx_merkle_root_cols against the oracle's Merkle root (merkle.rs:142-312)."""
    from vortexstark_b200.merkle import FusedRoot
    cols = [m31_array(11 * log_n + i, 1 << log_n) for i in range(ncols)]
    want = tuple(oracle.merkle_root(cols).tolist())
    fr = FusedRoot(log_n)
    d = [to_dev(c) for c in cols]
    assert fr.commit(d) == want
    assert fr.commit(d) == want  # workspace reused


def test_fused_root_workspace_bounds(oracle, L):
    import ctypes as C

    from vortexstark_b200.merkle import FusedRoot
    log_n = 20
    col = m31_array(5, 1 << log_n)
    want = tuple(oracle.merkle_root([col]).tolist())
    d = to_dev(col)
    fr = FusedRoot(log_n)
    ptrs = (C.c_void_p * 1)(d.data_ptr())
    # a workspace sized for the largest leaf subtree (smallest stored level) still works
    small = L.vx_merkle_workspace_words(log_n)
    for k in (4, 3, 2, 1):
        from vortexstark_b200 import tune
        tune.set_leaf_k(log_n, k)
        small = min(small, int(L.vx_merkle_workspace_words(log_n)))
    tune.set_leaf_k(log_n, 1)  # the device prefers a bigger pool than given
    _lib.check(L.vx_merkle_root_cols(ptrs, 1, log_n, fr.workspace.data_ptr(), small, fr.root_dev.data_ptr(), None))
    assert tuple(int(x) for x in to_host(fr.root_dev)) == want
    with pytest.raises(_lib.VortexError):
        _lib.check(L.vx_merkle_root_cols(ptrs, 1, log_n, fr.workspace.data_ptr(), small - 1, fr.root_dev.data_ptr(),
                                         None))
    with pytest.raises(_lib.VortexError):
        _lib.check(L.vx_merkle_root_cols(ptrs, 17, log_n, fr.workspace.data_ptr(), small, fr.root_dev.data_ptr(),
                                         None))
    tune.set_leaf_k(log_n, 0)


@pytest.mark.parametrize("L", [3, 4, 8, 13, 17, 20])
def test_fri_chain_matches_oracle(oracle, L):
    """vx_fri_chain against the oracle's composition of the proof's FRI
    pieces (circle fold, line folds, 4-word-leaf trees, transcript)."""
    from vortexstark_b200.fri import FriChain
    src = np.stack([m31_array(70 * L + c, 1 << L) for c in range(4)])
    state = [int(x) for x in m31_array(3 + L, 8)]
    want_roots, want_alphas, want_last = oracle.fri_chain(src, state)
    ch = FriChain(L)
    assert ch.layers == L - 1
    cols = [to_dev(c) for c in src]
    for _ in range(2):  # reusable: the second run must give the same words
        ch.commit_async(cols, state)
        roots, alphas, last = ch.result()
        assert np.array_equal(np.array(alphas, np.uint32), want_alphas)
        assert np.array_equal(np.array(roots, np.uint32), want_roots)
        assert np.array_equal(np.array(last, np.uint32), want_last)
    assert ch.launches() >= L
    ch.close()


def test_forge_forms_match_plain(oracle, L):
    """The forge-feature symbols of ntt.rs / blake2s_m31.rs: batched NTT with a host pointer array, the
    single layer and the batch inverse give the plain forms' words."""
    from vortexstark_b200 import ntt
    from vortexstark_b200.circle import Coset
    k, ncol = 12, 3
    n = 1 << k
    cache = ntt.TwiddleCache(Coset.half_coset(k))
    cols = [m31_array(500 + c, n) for c in range(ncol)]
    d1, d2 = [to_dev(c) for c in cols], [to_dev(c) for c in cols]
    ntt.evaluate_batch(d1, cache)
    hp = (C.c_void_p * ncol)(*[d.data_ptr() for d in d2])
    off = (C.c_uint32 * len(cache.layer_offsets))(*cache.layer_offsets)
    sz = (C.c_uint32 * len(cache.layer_sizes))(*cache.layer_sizes)
    L.cuda_circle_ntt_evaluate_batch_forge(hp, cache.d_twiddles.data_ptr(), cache.d_circle_twids.data_ptr(), off, sz,
                                           k - 1, n, ncol)
    for a, b in zip(d1, d2):
        assert np.array_equal(to_host(a, n), to_host(b, n))
    L.cuda_circle_ntt_interpolate_batch_forge(hp, cache.d_itwiddles.data_ptr(), cache.d_circle_itwids.data_ptr(), off,
                                              sz, k - 1, n, ncol)
    for c, b in zip(cols, d2):
        assert np.array_equal(to_host(b, n), c)
    x1, x2 = to_dev(cols[0]), to_dev(cols[0])
    tw = cache.d_twiddles.data_ptr() + 4 * cache.layer_offsets[2]
    L.cuda_circle_ntt_layer(x1.data_ptr(), tw, 3, n, 1)
    L.cuda_circle_ntt_layer_forge(x2.data_ptr(), tw, 3, n, 1)
    assert np.array_equal(to_host(x1, n), to_host(x2, n))
    z = m31_array(77, 1000)
    z[::50] = 0
    dz, oz = to_dev(z), empty(1000)
    L.cuda_batch_inverse_m31_forge(dz.data_ptr(), oz.data_ptr(), 1000)
    assert np.array_equal(to_host(oz, 1000), oracle.batch_inverse(z))


@pytest.mark.parametrize("n_line", [0, 3, 8])
def test_batched_ntt_partial_layer_count(oracle, L, n_line):
    """A layer count below the full transform (circle_ntt.cu:314-404,
    circle_ntt_batch_forge.cu:95-185): exactly n_line line layers and the
    circle layer, then for the inverse the 2^-log_n scale, in both batched
    forms (device pointer array and the forge host array)."""
    from vortexstark_b200 import ntt
    from vortexstark_b200.circle import Coset
    k, ncol = 10, 3
    n = 1 << k
    cache = ntt.TwiddleCache(Coset.half_coset(k))
    oline, ocirc, ooffs = oracle.twiddles(oracle.coset("half_coset", k), False)
    iline, icirc, _ = oracle.twiddles(oracle.coset("half_coset", k), True)
    cols = [m31_array(900 + c, n) for c in range(ncol)]
    want_e = []
    for x in cols:
        for l in range(n_line - 1, -1, -1):
            x = oracle.ntt_layer(x, oline[ooffs[l]:], l + 1, True)
        want_e.append(oracle.ntt_layer(x, ocirc, 0, True))
    want_i = []
    for x in want_e:
        x = oracle.ntt_layer(x, icirc, 0, False)
        for l in range(n_line):
            x = oracle.ntt_layer(x, iline[ooffs[l]:], l + 1, False)
        e = (30 * k) % 31
        want_i.append(np.array([(int(v) << e) % P for v in x], np.uint32))
    off = (C.c_uint32 * len(cache.layer_offsets))(*cache.layer_offsets)
    sz = (C.c_uint32 * len(cache.layer_sizes))(*cache.layer_sizes)
    d1, d2 = [to_dev(c) for c in cols], [to_dev(c) for c in cols]
    ptrs = ntt._ptr_array(d1)
    hp = (C.c_void_p * ncol)(*[d.data_ptr() for d in d2])
    L.cuda_circle_ntt_evaluate_batch(ptrs.data_ptr(), cache.d_twiddles.data_ptr(), cache.d_circle_twids.data_ptr(),
                                     off, sz, n_line, n, ncol)
    L.cuda_circle_ntt_evaluate_batch_forge(hp, cache.d_twiddles.data_ptr(), cache.d_circle_twids.data_ptr(), off, sz,
                                           n_line, n, ncol)
    for a, b, w in zip(d1, d2, want_e):
        assert np.array_equal(to_host(a, n), w) and np.array_equal(to_host(b, n), w)
    L.cuda_circle_ntt_interpolate_batch(ptrs.data_ptr(), cache.d_itwiddles.data_ptr(),
                                        cache.d_circle_itwids.data_ptr(), off, sz, n_line, n, ncol)
    L.cuda_circle_ntt_interpolate_batch_forge(hp, cache.d_itwiddles.data_ptr(), cache.d_circle_itwids.data_ptr(), off,
                                              sz, n_line, n, ncol)
    for a, b, w in zip(d1, d2, want_i):
        assert np.array_equal(to_host(a, n), w) and np.array_equal(to_host(b, n), w)
