"""Whole proofs from the device-resident prover against the oracle.

Bit-exact: the proof bytes (roots, FRI commitments, last layer, query
indices, every decommitted value and authentication path) must equal the
oracle's for the same (log_n, a, b), and both verifiers must accept them.
"""
import hashlib
import json
import os

import pytest

from vortexstark_b200 import prover
from vortexstark_b200.proof import deserialize_proof
from vortexstark_b200.verifier import verify
from vortexstark_b200.workload import fib_inputs

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_golden_proofs():
    for c in json.load(open(os.path.join(GOLDEN, "proofs.json"))):
        blob = prover.prove_bytes(c["a"], c["b"], c["log_n"], c["blowup_bits"], c["n_queries"])
        assert len(blob) == c["len"]
        assert hashlib.sha256(blob).hexdigest() == c["sha256"], (c["log_n"], c["a"], c["b"])
    assert prover.prove_bytes(1, 1, 4) == open(os.path.join(GOLDEN, "proof_4_1_1.bin"), "rb").read()


@pytest.mark.parametrize("log_n", [9, 10, 11, 12, 13, 14, 16, 18])
def test_matches_oracle(oracle, log_n):
    for a, b in fib_inputs(log_n, 2):
        assert prover.prove_bytes(a, b, log_n) == oracle.prove(a, b, log_n), (log_n, a, b)


@pytest.mark.parametrize("log_n,bb", [(6, 1), (12, 1), (10, 3)])
def test_other_blowups(oracle, log_n, bb):
    a, b = fib_inputs(77 + log_n, 1)[0]
    assert prover.prove_bytes(a, b, log_n, bb) == oracle.prove(a, b, log_n, bb)


def test_edge_inputs(oracle):
    for a, b in [(0, 0), (0x7FFFFFFE, 0x7FFFFFFE), (0, 1), (1, 0)]:
        assert prover.prove_bytes(a, b, 8) == oracle.prove(a, b, 8)


def test_log_n_20_matches_and_verifies(oracle):
    a, b = fib_inputs(20, 1)[0]
    blob = prover.prove_bytes(a, b, 20)
    assert blob == oracle.prove(a, b, 20)
    verify(deserialize_proof(blob))


def test_log_n_24_headline(oracle):
    """The single-proof configuration (2^24 rows, 2^26-point LDE), bit-exact."""
    a, b = fib_inputs(2024, 1)[0]
    blob = prover.prove_bytes(a, b, 24)
    assert oracle.verify(blob) == (0, "")
    assert blob == oracle.prove(a, b, 24)


def test_cache_reuse_and_sizes(oracle):
    """prover.rs:2373-2391: cached / pipeline proofs equal the plain ones."""
    c12 = prover.ProverCache(12)
    c14 = prover.ProverCache(14)
    for (a, b) in fib_inputs(5, 3):
        x = prover.prove_cached_bytes(a, b, c12)
        y = prover.prove_cached_bytes(a, b, c14)
        assert x == oracle.prove(a, b, 12)
        assert y == oracle.prove(a, b, 14)
    pipe = prover.ProverPipeline(10)
    ins = fib_inputs(9, 3)
    for (a, b), p in zip(ins, pipe.prove_batch(ins)):
        verify(p)
        assert p.public_inputs == (a, b)


def test_concurrent_slots_on_streams(oracle):
    """Proofs in flight at once on separate streams give the same bytes."""
    import torch
    sizes = [12, 14, 12, 16]
    ins = fib_inputs(31, len(sizes))
    caches = [prover.ProverCache(s) for s in sizes]
    streams = [torch.cuda.Stream() for _ in sizes]
    for c, s, (a, b) in zip(caches, streams, ins):
        c.prove_async(a, b, s.cuda_stream)
    torch.cuda.synchronize()
    for c, s, (a, b) in zip(caches, sizes, ins):
        assert c.result_bytes() == oracle.prove(a, b, s)
