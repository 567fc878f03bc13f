"""Largest single proofs, fully HBM-resident: log_n=28 at blowup 4 (2^30-point
LDE) and log_n=30 at blowup 2 (2^31 points, the whole M31 circle group;
the eval domain becomes subgroup(31), prover.rs:655-659).

At these sizes the CPU oracle would need minutes to hours, so parity rests on
size-independent properties: the oracle's verifier (verifier.rs:39-310)
accepts the proof (every authentication path and every fold equation of all
80 queries), the proof has the exact layout and size, and the bytes are
deterministic.  Bit-exact equality with the oracle is tested at every smaller
size in test_gpu_prover.py.
"""
import hashlib

import pytest

from vortexstark_b200 import _lib, prover
from vortexstark_b200.workload import fib_inputs

pytestmark = pytest.mark.gpu


def _free():
    import torch
    _lib.lib().vx_release_all()
    torch.cuda.synchronize()
    torch.cuda.empty_cache()


@pytest.mark.parametrize("log_n,blowup", [(28, 2), (30, 1)])
def test_max_size_proof_verifies(oracle, log_n, blowup):
    _free()
    a, b = fib_inputs(9000 + log_n, 1)[0]
    blob = prover.prove_bytes(a, b, log_n, blowup)
    assert len(blob) == oracle.proof_size(log_n, blowup)
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
