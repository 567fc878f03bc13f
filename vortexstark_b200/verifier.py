"""Verifier of the Fibonacci STARK (src/verifier.rs:39-310), host side.

Replays the transcript, re-derives the query indices, checks every Merkle
authentication path and the circle-fold and line-fold equations down to the
last layer.  Raises ``VerificationError`` on the first failure, with the same
checks in the same order as the reference.
"""
from __future__ import annotations

from .channel import Channel
from .circle import Coset, eval_domain
from .field import P, m31_inv, qm31_add, qm31_mul, qm31_mul_m31, qm31_sub
from .merkle import hash_leaf, verify_auth_path
from .proof import BLOWUP_BITS, N_QUERIES, StarkProof


class VerificationError(ValueError):
    pass


def _brev(x: int, bits: int) -> int:
    r = 0
    for _ in range(bits):
        r = (r << 1) | (x & 1)
        x >>= 1
    return r


def fold_twiddle_at(domain: Coset, folded_index: int, circle: bool) -> int:
    """verifier.rs:27-37"""
    p = domain.at(_brev(folded_index << 1, domain.log_size))
    return m31_inv(p.y if circle else p.x)


def _fold_pair(f0, f1, alpha, tw):
    return qm31_add(qm31_add(f0, f1), qm31_mul(alpha, qm31_mul_m31(qm31_sub(f0, f1), tw)))


def _check_paths(root, values, svals, paths, spaths, indices, label, width):
    if len(values) != N_QUERIES or len(paths) != N_QUERIES:
        raise VerificationError(f"{label} decommitment size mismatch")
    for q, qi in enumerate(indices):
        v = [values[q]] if width == 1 else values[q]
        if not verify_auth_path(root, hash_leaf(v), qi, paths[q]):
            raise VerificationError(f"{label} auth path invalid at query {q} (index {qi})")
        s = [svals[q]] if width == 1 else svals[q]
        if not verify_auth_path(root, hash_leaf(s), qi ^ 1, spaths[q]):
            raise VerificationError(f"{label} sibling auth path invalid at query {q} (sibling index {qi ^ 1})")


def verify(proof: StarkProof, blowup_bits: int = BLOWUP_BITS) -> None:
    log_n = proof.log_trace_size
    a, b = proof.public_inputs
    le = log_n + blowup_bits
    n_eval = 1 << le
    if a >= P or b >= P:
        raise VerificationError("Public inputs out of M31 range")
    if len(proof.query_indices) != N_QUERIES:
        raise VerificationError(f"Expected {N_QUERIES} queries, got {len(proof.query_indices)}")
    ch = Channel()
    ch.mix_digest(proof.trace_commitment)
    ch.draw_felt()
    ch.mix_digest(proof.quotient_commitment)
    alphas = [ch.draw_felt()]
    for c in proof.fri_commitments:
        ch.mix_digest(c)
        alphas.append(ch.draw_felt())
    if len(proof.fri_commitments) != max(le - 3, 0):
        raise VerificationError(f"Expected {le - 3} FRI layers, got {len(proof.fri_commitments)}")
    if len(proof.fri_last_layer) != 8:
        raise VerificationError(f"Expected 8 FRI last layer values, got {len(proof.fri_last_layer)}")
    ch.mix_felts(proof.fri_last_layer)
    expected = [ch.draw_number(n_eval) for _ in range(N_QUERIES)]
    if list(proof.query_indices) != expected:
        raise VerificationError("Query indices don't match Fiat-Shamir derivation")
    if tuple(proof.trace_commitment) == (0,) * 8:
        raise VerificationError("Trace commitment is zero")
    if tuple(proof.quotient_commitment) == (0,) * 8:
        raise VerificationError("Quotient commitment is zero")
    td, qd = proof.trace_decommitment, proof.quotient_decommitment
    _check_paths(proof.trace_commitment, td.values, td.sibling_values, td.auth_paths, td.sibling_auth_paths,
                 proof.query_indices, "trace", 1)
    _check_paths(proof.quotient_commitment, qd.values, qd.sibling_values, qd.auth_paths, qd.sibling_auth_paths,
                 proof.query_indices, "quotient", 4)
    folded = [qi // 2 for qi in proof.query_indices]
    for layer, (d, c) in enumerate(zip(proof.fri_decommitments, proof.fri_commitments)):
        _check_paths(c, d.values, d.sibling_values, d.auth_paths, d.sibling_auth_paths, folded, f"FRI layer {layer}", 4)
        folded = [i // 2 for i in folded]
    nfd = len(proof.fri_decommitments)
    for q, qi in enumerate(proof.query_indices):
        cur, cl = qi, le
        dom = eval_domain(cl)
        v, s = qd.values[q], qd.sibling_values[q]
        f0, f1 = (v, s) if cur % 2 == 0 else (s, v)
        exp = _fold_pair(f0, f1, alphas[0], fold_twiddle_at(dom, cur // 2, True))
        if exp != tuple(proof.fri_decommitments[0].values[q]):
            raise VerificationError(f"Circle fold mismatch at query {q} (qi={qi})")
        cur, cl = cur // 2, cl - 1
        for layer in range(max(nfd - 1, 0)):
            d = proof.fri_decommitments[layer]
            v, s = d.values[q], d.sibling_values[q]
            f0, f1 = (v, s) if cur % 2 == 0 else (s, v)
            exp = _fold_pair(f0, f1, alphas[layer + 1], fold_twiddle_at(Coset.half_odds(cl), cur // 2, False))
            if exp != tuple(proof.fri_decommitments[layer + 1].values[q]):
                raise VerificationError(f"Line fold mismatch at query {q}, layer {layer}->{layer + 1} (log={cl})")
            cur, cl = cur // 2, cl - 1
        if nfd:
            if cur >= len(proof.fri_last_layer):
                raise VerificationError(f"FRI last layer index {cur} out of bounds")
            if tuple(proof.fri_decommitments[-1].values[q]) != tuple(proof.fri_last_layer[cur]):
                raise VerificationError(f"FRI last layer mismatch at query {q} (index {cur})")
