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


@pytest.mark.parametrize("log_n,count", [(8, 1), (8, 2), (10, 5), (12, 11), (14, 4), (18, 3)])
def test_prove_batch_matches_single_proofs(oracle, log_n, count):
    """vx_prove_fib_batch (ProverPipeline::prove_batch, prover.rs:2305) gives the
    proofs that vx_prove_fib and the oracle give, in input order."""
    inputs = fib_inputs(900 + log_n, count)
    got = prover.prove_batch_bytes(inputs, log_n)
    assert len(got) == count
    for (a, b), blob in zip(inputs, got):
        assert blob == prover.prove_bytes(a, b, log_n)
    for (a, b), blob in list(zip(inputs, got))[:2]:
        assert blob == oracle.prove(a, b, log_n)


def test_prove_batch_slots_grow_between_calls():
    """A size first batched with one proof, then with more: the cached context
    grows to more slots in flight and every proof stays byte-identical."""
    for count in (1, 3, 9):
        inputs = fib_inputs(1700 + count, count)
        got = prover.prove_batch_bytes(inputs, 9)
        assert [blob == prover.prove_bytes(a, b, 9) for (a, b), blob in zip(inputs, got)] == [True] * count


def test_prove_batch_arguments():
    import ctypes as C

    from vortexstark_b200 import _lib
    assert prover.prove_batch_bytes([], 8) == []
    size = prover.proof_size(8)
    a = (C.c_uint32 * 2)(1, 2)
    b = (C.c_uint32 * 2)(3, 0x7FFFFFFF)  # the second input is not canonical
    buf = (C.c_uint8 * (2 * size))()
    n = C.c_size_t()
    L = _lib.lib()
    with pytest.raises(_lib.VortexError):
        _lib.check(L.vx_prove_fib_batch(a, b, 2, 8, 2, 80, buf, 2 * size, C.byref(n)))
    with pytest.raises(_lib.VortexError):
        _lib.check(L.vx_prove_fib_batch(a, a, 2, 8, 2, 80, buf, 2 * size - 1, C.byref(n)))
