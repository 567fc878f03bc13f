"""Largest single proofs, fully HBM-resident: log_n=28 at blowup 4 (2^30-point
LDE) and log_n=30 at blowup 2 (2^31 points, the whole M31 circle group;
the eval domain becomes subgroup(31), prover.rs:655-659).

Parity is bit-exact: the proof's SHA-256 equals the oracle's for the same
inputs, recorded in tests/golden/large_proofs.json by
tests/golden/gen_large.py (the oracle's memory-lean prove, minutes of CPU time
and tens of GB of host memory per proof, so it is generated once rather than
on every run).  The oracle's verifier (verifier.rs:39-310) also accepts the
proof, and the bytes are deterministic.
"""
import hashlib
import json
import os

import pytest

from vortexstark_b200 import _lib, prover
from vortexstark_b200.workload import fib_inputs

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "large_proofs.json")


def _free():
    import torch
    _lib.lib().vx_release_all()
    torch.cuda.synchronize()
    torch.cuda.empty_cache()


@pytest.mark.parametrize("log_n,blowup", [(28, 2), (30, 1)])
def test_max_size_proof_matches_oracle(oracle, log_n, blowup):
    want = json.load(open(GOLDEN))[f"{log_n}_{blowup}"]
    _free()
    a, b = fib_inputs(9000 + log_n, 1)[0]
    assert (a, b) == (want["a"], want["b"])
    blob = prover.prove_bytes(a, b, log_n, blowup)
    assert len(blob) == want["len"] == oracle.proof_size(log_n, blowup)
    assert hashlib.sha256(blob).hexdigest() == want["sha256"]
    rc, msg = oracle.verify(blob, blowup)
    assert rc == 0, msg
    again = prover.prove_bytes(a, b, log_n, blowup)
    assert hashlib.sha256(again).digest() == hashlib.sha256(blob).digest()
    _free()


def test_lifted_commitment_full_shape_matches_oracle(oracle):
    """The batched workload at its full size: 34 columns (8 x 2^16,
    16 x 2^18, 10 x 2^20), blowup 4, 80 queries, S = 22."""
    import bench
    from vortexstark_b200.lifted import commit_lifted, verify_lifted

    cols = bench.lifted_workload(bench.SEED)
    got = commit_lifted(cols, 2, 80)
    assert got == oracle.commit_lifted(cols, 2, 80)
    verify_lifted(got, 80)
