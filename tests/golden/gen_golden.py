"""Generate the golden fixtures in this directory.

Run from the repository root:  python tests/golden/gen_golden.py

Source of truth: oracle/pyoracle.py, a pure-Python restatement of the
reference's Fibonacci commitment path that hashes with hashlib.blake2s.  The
fixtures pin the C oracle and the GPU path to it:
  proofs.json   — for small (log_n, a, b): proof length, SHA-256 of the proof
                  bytes, trace / quotient / FRI roots, the query indices.
  proof_4_1_1.bin — complete proof bytes of (log_n=4, a=1, b=1).
  kernels.json  — NTT evaluate / interpolate, fold twiddles and folds on
                  fixed small inputs.
"""
import hashlib
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle import pyoracle as Y  # noqa: E402

CASES = [(4, 1, 1), (4, 2, 3), (5, 42, 99), (5, 1000, 2000), (6, 1, 1), (6, 123456789, 987654321), (7, 5, 8),
         (8, 2147483646, 0)]


def proofs():
    out = []
    for log_n, a, b in CASES:
        blob = Y.prove(a, b, log_n)
        w = Y.words(blob)
        nf = w[21]
        qoff = 22 + 8 * nf + 1 + 32
        out.append({
            "log_n": log_n, "a": a, "b": b, "blowup_bits": 2, "n_queries": 80,
            "len": len(blob), "sha256": hashlib.sha256(blob).hexdigest(),
            "trace_root": w[5:13], "quotient_root": w[13:21],
            "fri_roots": [w[22 + 8 * k:30 + 8 * k] for k in range(nf)],
            "query_indices": w[qoff + 1:qoff + 1 + 80],
        })
        if (log_n, a, b) == (4, 1, 1):
            open(os.path.join(HERE, "proof_4_1_1.bin"), "wb").write(blob)
    return out


def kernels():
    out = {}
    x = [(i * 7 + 13) % Y.P for i in range(64)]  # prover.rs:2497 input pattern
    for kind, cs in (("half_coset", Y.half_coset(6)), ("half_odds", Y.half_odds(6)), ("subgroup", Y.subgroup(6))):
        d = list(x)
        Y.evaluate(d, cs)
        out[f"evaluate_{kind}_6"] = d
        if kind != "subgroup":
            e = list(x)
            Y.interpolate(e, cs)
            out[f"interpolate_{kind}_6"] = e
    out["fold_tw_circle_half_coset_6"] = Y.fold_tw(Y.half_coset(6), True)
    out["fold_tw_line_half_odds_6"] = Y.fold_tw(Y.half_odds(6), False)
    vals = [((i * 3 + 1) % Y.P, (i * 5 + 2) % Y.P, (i * 7 + 3) % Y.P, (i * 11 + 4) % Y.P) for i in range(64)]
    alpha = (42, 99, 7, 13)  # fri.rs:599
    out["fold_line_half_odds_6"] = [list(v) for v in Y.fold(vals, Y.fold_tw(Y.half_odds(6), False), alpha)]
    out["fold_circle_half_coset_6"] = [list(v) for v in Y.fold(vals, Y.fold_tw(Y.half_coset(6), True), alpha)]
    return out


if __name__ == "__main__":
    json.dump(proofs(), open(os.path.join(HERE, "proofs.json"), "w"), indent=1)
    json.dump(kernels(), open(os.path.join(HERE, "kernels.json"), "w"))
    print("wrote", os.listdir(HERE))
