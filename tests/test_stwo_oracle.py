"""The oracle's stwo-format path and batched lifted commitment, pinned
without a GPU.

stwo (the reference's dependency that owns these conventions) is not in the
reference tree, so the stwo NTT is pinned to the mathematics it computes: a
circle polynomial in stwo's basis  y^b0 * x^b1 * pi(x)^b2 * ...  (pi(x) =
2x^2 - 1), evaluated on CanonicCoset(L)'s circle domain in bit-reversed
order (poly_ops.rs:718, ntt.rs:539-585).  The lifted commitment is pinned by
its algebra (lifted columns have low degree, the FRI last layer is a
degree-1 line polynomial) and by an independent host verifier
(vortexstark_b200.lifted.verify_lifted).
"""
import numpy as np
import pytest

from vortexstark_b200.lifted import LiftedVerificationError, lifted_size, parse_lifted, verify_lifted

P = 0x7FFFFFFF
G = (2, 1268011823)


def _mul(p, q):
    return ((p[0] * q[0] - p[1] * q[1]) % P, (p[0] * q[1] + p[1] * q[0]) % P)


def _pow(p, e):
    r = (1, 0)
    while e:
        if e & 1:
            r = _mul(r, p)
        p = _mul(p, p)
        e >>= 1
    return r


def _brev(i, b):
    r = 0
    for _ in range(b):
        r = (r << 1) | (i & 1)
        i >>= 1
    return r


def _domain_at(L, k):
    """CanonicCoset(L).circle_domain().at(k): half_odds(L-1), then its conjugate."""
    ini, st = _pow(G, 1 << (29 - (L - 1))), _pow(G, 1 << (31 - (L - 1)))
    h = 1 << (L - 1)
    if k < h:
        return _mul(ini, _pow(st, k))
    p = _mul(ini, _pow(st, k - h))
    return (p[0], (-p[1]) % P)


def _eval_poly(c, pt):
    x, y = pt
    L = len(c).bit_length() - 1
    fs = [y]
    xx = x
    for _ in range(1, L):
        fs.append(xx)
        xx = (2 * xx * xx - 1) % P
    tot = 0
    for i, ci in enumerate(c):
        t = int(ci)
        for j in range(L):
            if (i >> j) & 1:
                t = t * fs[j] % P
        tot = (tot + t) % P
    return tot


@pytest.mark.parametrize("L", [3, 4, 5, 6])
def test_stwo_evaluate_is_circle_polynomial_evaluation(oracle, L):
    rng = np.random.default_rng(100 + L)
    c = rng.integers(0, P, 1 << L, dtype=np.uint32)
    got = oracle.stwo_ntt_evaluate(c)
    want = [_eval_poly(c, _domain_at(L, _brev(j, L))) for j in range(1 << L)]
    assert got.tolist() == want


@pytest.mark.parametrize("L", [3, 5])
def test_stwo_lde_is_the_same_polynomial_on_the_bigger_domain(oracle, L):
    rng = np.random.default_rng(200 + L)
    c = np.zeros(1 << (L + 2), np.uint32)
    c[: 1 << L] = rng.integers(0, P, 1 << L, dtype=np.uint32)
    got = oracle.stwo_ntt_evaluate(c)
    want = [_eval_poly(c, _domain_at(L + 2, _brev(j, L + 2))) for j in range(1 << (L + 2))]
    assert got.tolist() == want


def test_stwo_log2_reads_the_padding_as_y(oracle):
    # The reference kernel derives the circle layer from pairs of level 0;
    # at 4 points level 0 has one word and the pair's y is the padding 1
    # (circle_ntt_stwo.cu:202-249).  The oracle keeps that behaviour.
    tw = oracle.stwo_twiddles(2)
    assert tw[1] == 1
    c = np.array([5, 7, 11, 13], np.uint32)
    x = int(tw[0])
    d = [5, 7, 11, 13]
    # line layer (h = 0, t = x), then circle layer with t = [1, -1, -x, x]
    t = x * d[2] % P; d[2] = (d[0] - t) % P; d[0] = (d[0] + t) % P
    t = x * d[3] % P; d[3] = (d[1] - t) % P; d[1] = (d[1] + t) % P
    for tid, tv in ((0, 1), (1, P - 1)):
        t = tv * d[2 * tid + 1] % P
        d[2 * tid + 1] = (d[2 * tid] - t) % P
        d[2 * tid] = (d[2 * tid] + t) % P
    assert oracle.stwo_ntt_evaluate(c).tolist() == d


@pytest.mark.parametrize("L", range(2, 14))
def test_stwo_round_trip(oracle, L):
    rng = np.random.default_rng(L)
    x = rng.integers(0, P, 1 << L, dtype=np.uint32)
    assert (oracle.stwo_ntt_interpolate(oracle.stwo_ntt_evaluate(x)) == x).all()


@pytest.mark.parametrize("L", [2, 3, 8, 12])
def test_stwo_twiddle_layout(oracle, L):
    """ntt.rs:300-341: level j = x of the first half of half_odds(L-1)
    doubled j times, bit-reversed within the level; then a 1."""
    tw = oracle.stwo_twiddles(L)
    assert len(tw) == 1 << (L - 1) and tw[-1] == 1
    off = 0
    for j in range(L - 1):
        lvl = L - 1 - j  # log size of the level's coset
        half = 1 << (lvl - 1)
        ini, st = _pow(G, 1 << (29 - lvl)), _pow(G, 1 << (31 - lvl))
        bits = lvl - 1
        for i in range(half):
            assert tw[off + (_brev(i, bits) if bits else 0)] == _mul(ini, _pow(st, i))[0]
        off += half
    inv = oracle.stwo_twiddles(L, True)
    assert all(int(a) * int(b) % P == 1 for a, b in zip(tw, inv))


def test_stwo_fold_circle_twiddles(oracle):
    for L in (3, 6, 9):
        tw = oracle.stwo_fold_circle_twiddles(L)
        for i in range(1 << (L - 1)):
            y = _domain_at(L, _brev(i << 1, L))[1]
            assert int(tw[i]) * y % P == 1


def test_accumulate_lift_and_bit_reverse_and_pack(oracle):
    rng = np.random.default_rng(7)
    col = rng.integers(0, P, 64, dtype=np.uint32)
    for r in (0, 1, 3):
        curr = rng.integers(0, P, 64 >> r, dtype=np.uint32)
        i = np.arange(64)
        src = ((i >> (r + 1)) << 1) | (i & 1)
        want = (col.astype(np.uint64) + curr[src]) % P
        assert (oracle.accumulate_lift(col, curr) == want).all()
    q = rng.integers(0, P, 4 * 32, dtype=np.uint32)
    br = oracle.bit_reverse_qm31(q).reshape(32, 4)
    for k in range(32):
        assert (br[_brev(k, 5)] == q.reshape(32, 4)[k]).all()
    cols = [rng.integers(0, P, 64, dtype=np.uint32) for _ in range(4)]
    pk = oracle.pack_leaves(cols)
    for c in range(4):
        for i in range(64):
            assert pk[c * 16 + i % 16][i // 16] == cols[c][i]


def _cols(seed, logs):
    rng = np.random.default_rng(seed)
    return [rng.integers(0, P, 1 << L, dtype=np.uint32) for L in logs]


def test_lifted_columns_have_low_degree(oracle):
    logs, B = [3, 4, 5], 2
    ldes = oracle.lifted_lde(_cols(1, logs), B)
    S = max(logs) + B
    i = np.arange(1 << S)
    for c in ldes:
        Lc = len(c).bit_length() - 1
        lifted = c if Lc == S else c[((i >> (S - Lc + 1)) << 1) | (i & 1)]
        co = oracle.stwo_ntt_interpolate(lifted)
        assert not co[1 << (S - B):].any()


def test_lifted_commitment_verifies_and_last_layer_is_linear(oracle):
    logs = [3, 3, 4, 5, 5]
    words = oracle.commit_lifted(_cols(2, logs), 2, 24)
    assert len(words) == oracle.lifted_size(logs, 2, 24) == lifted_size(logs, 2, 24)
    c = verify_lifted(words, 24)
    # the last layer (8 values on half_odds(3), bit-reversed) is a + b x
    ini, st = _pow(G, 1 << 26), _pow(G, 1 << 28)
    xs = [_mul(ini, _pow(st, _brev(j, 3)))[0] for j in range(8)]
    for comp in range(4):
        v = [c.last_layer[j][comp] for j in range(8)]
        b = (v[1] - v[0]) * pow((xs[1] - xs[0]) % P, P - 2, P) % P
        a = (v[0] - b * xs[0]) % P
        assert all((a + b * xs[j] - v[j]) % P == 0 for j in range(8))


def test_lifted_commitment_tampering_is_rejected(oracle):
    words = oracle.commit_lifted(_cols(3, [4, 4, 6]), 2, 16)
    verify_lifted(words)
    n = len(words) // 4
    rng = np.random.default_rng(5)
    header = 5 + 3
    for w in list(rng.integers(header, n, 25)) + [header, header + 8, n - 1]:
        bad = bytearray(words)
        bad[4 * int(w)] ^= 0x10
        with pytest.raises((LiftedVerificationError, ValueError)):
            verify_lifted(bytes(bad))


def test_lifted_shapes_rejected(oracle):
    assert oracle.lifted_size([5, 4], 2, 8) == 0      # not ascending
    assert oracle.lifted_size([1, 4], 2, 8) == 0      # too small
    assert oracle.lifted_size([27], 2, 8) == 0        # LDE above 2^28
    assert lifted_size([5, 4], 2, 8) == 0 and lifted_size([1], 2, 8) == 0
    with pytest.raises(ValueError):
        oracle.commit_lifted(_cols(4, [5, 4]), 2, 8)
    assert parse_lifted(oracle.commit_lifted(_cols(4, [4, 5]), 1, 8)).lifting_log == 6


def test_eval_at_point_fold_is_the_weighted_sum():
    """The level-by-level fold equals sum_i c[i] prod(f_(k-1-b) for the set bits b of i)."""
    import numpy as np

    from oracle import oracle as O
    P = (1 << 31) - 1
    rng = np.random.default_rng(3)
    k = 5
    c = rng.integers(0, P, 1 << k, dtype=np.uint32)
    f = rng.integers(0, P, (k, 4), dtype=np.uint32)
    acc = np.zeros(4, np.uint32)
    for i in range(1 << k):
        w = np.array([1, 0, 0, 0], np.uint32)
        for b in range(k):
            if (i >> b) & 1:
                w = O.qm31_mul(w, f[k - 1 - b])
        term = np.array([(int(x) * int(c[i])) % P for x in w], np.uint32)
        acc = np.array([(int(x) + int(y)) % P for x, y in zip(acc, term)], np.uint32)
    assert np.array_equal(O.eval_at_point(c, f), acc)
