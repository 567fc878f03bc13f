"""The oracle itself, pinned before it is trusted (CPU only).

Pins: Blake2s against hashlib; the reference's own known-answer tests
(circle.rs:586-622 group facts, channel.rs:346-381 mix_felts, fri.rs:513-580
last-layer polynomial round trip); the C oracle against the independent
Python restatement and the committed golden fixtures; verifier acceptance and
tamper rejection (verifier.rs:319-410).
"""
import hashlib
import json
import os
import struct

import numpy as np
import pytest

from oracle import pyoracle as Y

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("n", [0, 1, 3, 4, 16, 36, 37, 63, 64, 65, 127, 128, 129, 160, 300])
def test_blake2s_matches_hashlib(oracle, n):
    data = bytes((i * 31 + 7) & 0xFF for i in range(n))
    assert oracle.blake2s(data) == hashlib.blake2s(data).digest()


def test_generator_facts(oracle):
    """circle.rs:586-622"""
    L = oracle.lib()
    g = oracle.Point(2, 1268011823)
    assert (g.x * g.x + g.y * g.y) % Y.P == 1
    r = L.vxo_point_pow(g, 1 << 31)
    assert (r.x, r.y) == (1, 0)
    half = L.vxo_point_pow(g, 1 << 30)
    assert (half.x, half.y) != (1, 0)
    sg = oracle.coset("subgroup", 2)
    r = L.vxo_point_pow(sg.step, 4)
    assert (r.x, r.y) == (1, 0)
    c = L.vxo_point_mul(g, oracle.Point(g.x, (Y.P - g.y) % Y.P))
    assert (c.x, c.y) == (1, 0)


def test_mix_felts_kat():
    """channel.rs:346-381: mix_felts is one Blake2s over state || all felts."""
    felts = [tuple(range(4 * i + 1, 4 * i + 5)) for i in range(9)]
    ch = Y.Channel()
    ch.mix_felts(felts)
    expect = hashlib.blake2s(bytes(32) + b"".join(struct.pack("<4I", *f) for f in felts)).digest()
    assert ch.state == expect
    from vortexstark_b200.channel import Channel
    c2 = Channel()
    c2.mix_felts(felts)
    assert c2.state == expect


@pytest.mark.parametrize("coeffs", [[(42, 0, 0, 0), (17, 0, 0, 0)],
                                    [(42, 0, 0, 0), (17, 0, 0, 0), (99, 0, 0, 0), (7, 0, 0, 0)]])
def test_last_layer_poly_kat(coeffs):
    """fri.rs:513-580: BRT evaluations on half_odds(3) of a known line
    polynomial recover its coefficients (pins the half_odds convention)."""
    dom = Y.half_odds(3)
    ev = []
    for j in range(8):
        x = Y.at(dom, Y.brev(j, 3))[0]
        dx = (2 * x * x - 1) % Y.P
        basis = [1, x, dx, x * dx % Y.P]
        acc = (0, 0, 0, 0)
        for c, bb in zip(coeffs, basis):
            acc = Y.qadd(acc, Y.qmulm(c, bb))
        ev.append(acc)
    got = Y.last_layer_poly_coeffs(ev)
    assert got[:len(coeffs)] == [tuple(c) for c in coeffs]
    assert all(v == (0, 0, 0, 0) for v in got[len(coeffs):])
    for j in range(8):
        assert Y.eval_last_layer_poly(got, j, 3) == ev[j]


def test_golden_proofs_match_c_oracle(oracle):
    for c in json.load(open(os.path.join(GOLDEN, "proofs.json"))):
        blob = oracle.prove(c["a"], c["b"], c["log_n"], c["blowup_bits"], c["n_queries"])
        assert len(blob) == c["len"]
        assert hashlib.sha256(blob).hexdigest() == c["sha256"], c
        tr, qr, fr = oracle.prove_roots(c["a"], c["b"], c["log_n"])
        assert tr.tolist() == c["trace_root"] and qr.tolist() == c["quotient_root"]
        assert fr.tolist() == c["fri_roots"]


def test_golden_bin(oracle):
    blob = open(os.path.join(GOLDEN, "proof_4_1_1.bin"), "rb").read()
    assert oracle.prove(1, 1, 4) == blob
    assert Y.prove(1, 1, 4) == blob


@pytest.mark.parametrize("log_n,a,b", [(6, 1, 1), (7, 2, 3), (8, 42, 99), (9, 1000, 2000)])
def test_c_oracle_equals_python_restatement(oracle, log_n, a, b):
    assert oracle.prove(a, b, log_n) == Y.prove(a, b, log_n)


def test_blowup_one_matches_python(oracle):
    assert oracle.prove(3, 5, 6, blowup_bits=1) == Y.prove(3, 5, 6, blowup_bits=1)


@pytest.mark.parametrize("log_n", [4, 5, 6, 8, 10, 14])
def test_oracle_verifier_accepts(oracle, log_n):
    """verifier.rs:319-360"""
    for a, b in [(1, 1), (2, 3), (42, 99), (1000, 2000)]:
        blob = oracle.prove(a, b, log_n)
        assert oracle.verify(blob) == (0, "")


@pytest.mark.parametrize("log_n,blowup", [(4, 1), (5, 3), (7, 2), (8, 1), (10, 2), (13, 3), (16, 2)])
def test_lean_prove_equals_full_prove(oracle, log_n, blowup):
    """The memory-lean prove (recomputed quotient, trees stored from height
    8 up) that generates the largest proofs' fixtures gives the same bytes as
    the full prove, below and above the stored height."""
    for a, b in [(1, 1), (123456789, 987654321)]:
        assert oracle.prove_lean(a, b, log_n, blowup) == oracle.prove(a, b, log_n, blowup)


def test_large_proof_fixtures(oracle):
    """tests/golden/large_proofs.json holds the oracle's 2^30- and 2^31-point
    proofs (log_n = 28 / blowup 2 and log_n = 30 / blowup 1) for the inputs
    the GPU test proves."""
    from vortexstark_b200.workload import fib_inputs

    data = json.load(open(os.path.join(GOLDEN, "large_proofs.json")))
    for log_n, blowup in [(28, 2), (30, 1)]:
        e = data[f"{log_n}_{blowup}"]
        assert (e["a"], e["b"]) == fib_inputs(9000 + log_n, 1)[0]
        assert e["len"] == oracle.proof_size(log_n, blowup) and len(e["sha256"]) == 64


def test_oracle_verifier_rejects_tampering(oracle):
    """verifier.rs:324-367 (trace / quotient / FRI values, commitments) plus
    random words of the decommitments.  Words 3 and 4 (the public inputs) are
    excluded: the reference verifier only range-checks them (verifier.rs:46-49)
    and the transcript does not bind them, so a changed in-range input is
    accepted there too."""
    blob = oracle.prove(7, 11, 6)
    w = np.frombuffer(blob, dtype=np.uint32)
    rng = np.random.default_rng(1)
    positions = sorted(set([2, 5, 13, 22, 40] + rng.integers(60, len(w), 40).tolist()))
    for pos in positions:
        t = w.copy()
        t[pos] ^= 1
        rc, msg = oracle.verify(t.tobytes())
        assert rc != 0, (pos, msg)


def test_kernel_goldens(oracle):
    g = json.load(open(os.path.join(GOLDEN, "kernels.json")))
    x = np.array([(i * 7 + 13) % Y.P for i in range(64)], np.uint32)
    for kind in ("half_coset", "half_odds", "subgroup"):
        cs = oracle.coset(kind, 6)
        assert oracle.ntt_evaluate(x, cs).tolist() == g[f"evaluate_{kind}_6"]
        if kind != "subgroup":
            assert oracle.ntt_interpolate(x, cs).tolist() == g[f"interpolate_{kind}_6"]
    assert oracle.fold_twiddles(oracle.coset("half_coset", 6), True).tolist() == g["fold_tw_circle_half_coset_6"]
    assert oracle.fold_twiddles(oracle.coset("half_odds", 6), False).tolist() == g["fold_tw_line_half_odds_6"]


@pytest.mark.parametrize("log_n", [1, 2, 4, 9, 14, 18])
def test_oracle_ntt_round_trip(oracle, log_n):
    """ntt.rs:386-449"""
    from vortexstark_b200.workload import m31_array
    x = m31_array(log_n, 1 << log_n)
    cs = oracle.coset("half_coset", log_n)
    assert np.array_equal(oracle.ntt_interpolate(oracle.ntt_evaluate(x, cs), cs), x)


def test_layerwise_matches_standard(oracle):
    """prover.rs:2491-2574: layer-by-layer application of the extract-and-squash
    tables equals the standard evaluate (pins the twiddle layout)."""
    log_n = 8
    cs = oracle.coset("half_coset", log_n)
    x = np.array([(i * 7 + 13) % Y.P for i in range(1 << log_n)], np.uint32)
    line, circ, offs = oracle.twiddles(cs, False)
    d = x.copy()
    sizes = [(1 << log_n) >> (l + 1) for l in range(log_n - 1)]
    for l in range(log_n - 2, -1, -1):
        d = oracle.ntt_layer(d, line[offs[l]:offs[l] + sizes[l]], l + 1, True)
    d = oracle.ntt_layer(d, circ, 0, True)
    assert np.array_equal(d, oracle.ntt_evaluate(x, cs))


def test_batch_inverse_chunk_semantics(oracle):
    """batch_inverse.cu:8-41: 0 -> 0, and a zero in a chunk's first slot zeroes
    the whole chunk."""
    x = np.arange(1, 200, dtype=np.uint32)
    inv = oracle.batch_inverse(x)
    assert all(int(a) * int(b) % Y.P == 1 for a, b in zip(x, inv))
    y = x.copy()
    y[5] = 0
    y[64] = 0
    inv = oracle.batch_inverse(y)
    assert inv[5] == 0 and all(inv[64:128] == 0)
    assert all(int(a) * int(b) % Y.P == 1 for a, b in zip(y[:5], inv[:5]))
    assert all(int(a) * int(b) % Y.P == 1 for a, b in zip(y[128:], inv[128:]))


def test_fibonacci_trace_parallel_equals_sequential(oracle):
    t = oracle.fibonacci_trace(5, 8, 18)
    assert t.tolist()[:64] == Y.fib_trace(5, 8, 64)
    seq = [5, 8]
    for _ in range((1 << 18) - 2):
        seq.append((seq[-1] + seq[-2]) % Y.P)
    assert t.tolist() == seq


def test_lifted_leaves(oracle):
    """merkle_leaves_lifted.cu:25-98: leaf = Blake2s over every column's lifted row."""
    from vortexstark_b200.workload import m31_array
    cols = [m31_array(1, 4), m31_array(2, 8), m31_array(3, 8), m31_array(4, 16)] + [m31_array(10 + i, 16) for i in range(14)]
    S = 4
    got = oracle.lifted_leaves(cols, S)
    for idx in range(16):
        words = []
        for c in cols:
            L = len(c).bit_length() - 1
            row = idx if L == S else ((idx >> (S - L + 1)) << 1) | (idx & 1)
            words.append(int(c[row]))
        h = struct.unpack("<8I", hashlib.blake2s(struct.pack(f"<{len(words)}I", *words)).digest())
        assert tuple(got[idx].tolist()) == h


def test_fri_chain_composition():
    """vxo_fri_chain against a composition of the oracle's fold and tree
    functions with the host channel restatement (channel.rs): the order of
    draws, folds, commitments and mixes."""
    import struct

    import numpy as np

    from oracle import oracle as O
    from vortexstark_b200.channel import Channel

    L = 7
    rng = np.random.default_rng(11)
    src = rng.integers(0, (1 << 31) - 1, (4, 1 << L), dtype=np.uint32)
    state = [int(x) for x in rng.integers(0, 1 << 32, 8, dtype=np.uint64)]
    roots, alphas, last = O.fri_chain(src, state)
    ch = Channel()
    ch.state = struct.pack("<8I", *state)
    cur = src
    for k in range(L - 1):
        a = ch.draw_felt()
        assert tuple(alphas[k]) == tuple(a), k
        if k == 0:
            tw = O.fold_twiddles(O.coset("half_coset", L), True)
            cur = O.fold_circle_into_line(np.zeros((4, 1 << (L - 1)), np.uint32), cur, tw, a)
        else:
            l = L - k
            cur = O.fold_line(cur, O.fold_twiddles(O.coset("half_odds", l), False), a)
        r = O.merkle_root([cur[c] for c in range(4)])
        assert np.array_equal(r, roots[k]), k
        ch.mix_digest(tuple(int(x) for x in r))
    assert np.array_equal(cur.T, last)
