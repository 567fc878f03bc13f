"""Host-side logic and the C ABI surface (CPU only, no kernel launches)."""
import os

import numpy as np
import pytest

import vortexstark_b200
from vortexstark_b200 import _lib
from vortexstark_b200.proof import deserialize_proof, serialize_proof
from vortexstark_b200.verifier import VerificationError, verify

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_library_exports_every_declared_symbol(vx):
    names = _lib.header_symbols()
    assert len(names) >= 45
    missing = [n for n in names if not hasattr(vx, n)]
    assert not missing, missing


def test_binding_table_covers_header():
    assert set(_lib.header_symbols()) == set(_lib._SIGS), set(_lib.header_symbols()) ^ set(_lib._SIGS)


@pytest.mark.parametrize("log_n,bb", [(4, 2), (6, 2), (10, 2), (16, 2), (24, 2), (28, 2), (30, 1), (20, 1)])
def test_proof_size_matches_oracle(vx, oracle, log_n, bb):
    assert vx.vx_proof_size(log_n, bb, 80) == oracle.proof_size(log_n, bb, 80)


def test_proof_size_rejects_bad_sizes(vx):
    assert vx.vx_proof_size(3, 2, 80) == 0
    assert vx.vx_proof_size(30, 2, 80) == 0


def test_serialize_round_trip():
    blob = open(os.path.join(GOLDEN, "proof_4_1_1.bin"), "rb").read()
    p = deserialize_proof(blob)
    assert p.log_trace_size == 4 and p.public_inputs == (1, 1) and len(p.query_indices) == 80
    assert len(p.fri_commitments) == 3 and len(p.fri_decommitments) == 3
    assert serialize_proof(p) == blob


def test_host_verifier_accepts_oracle_proofs(oracle):
    for log_n, a, b in [(4, 1, 1), (5, 2, 3), (6, 42, 99), (8, 1000, 2000)]:
        verify(deserialize_proof(oracle.prove(a, b, log_n)))


def test_host_verifier_rejects(oracle):
    """verifier.rs:324-367"""
    blob = oracle.prove(1, 1, 6)
    p = deserialize_proof(blob)
    p.trace_decommitment.values[0] ^= 1
    with pytest.raises(VerificationError):
        verify(p)
    p = deserialize_proof(blob)
    p.quotient_decommitment.values[0] = (p.quotient_decommitment.values[0][0] ^ 1,) + p.quotient_decommitment.values[0][1:]
    with pytest.raises(VerificationError):
        verify(p)
    p = deserialize_proof(blob)
    v = p.fri_decommitments[0].values[0]
    p.fri_decommitments[0].values[0] = (v[0] ^ 1,) + v[1:]
    with pytest.raises(VerificationError):
        verify(p)
    p = deserialize_proof(blob)
    p.trace_commitment = (p.trace_commitment[0] ^ 1,) + p.trace_commitment[1:]
    with pytest.raises(VerificationError):
        verify(p)
    p = deserialize_proof(blob)
    p.fri_commitments.pop()
    with pytest.raises(VerificationError):
        verify(p)


def test_deserialize_rejects_garbage():
    with pytest.raises(ValueError):
        deserialize_proof(b"\x00" * 16)
    blob = open(os.path.join(GOLDEN, "proof_4_1_1.bin"), "rb").read()
    with pytest.raises(ValueError):
        deserialize_proof(blob[:-4])
    with pytest.raises(ValueError):
        deserialize_proof(blob + b"\x00" * 4)


def test_prover_rejects_bad_inputs():
    from vortexstark_b200 import prover
    with pytest.raises(ValueError):
        prover.prove_bytes(0x7FFFFFFF, 1, 8)
    with pytest.raises(ValueError):
        prover.prove_bytes(1, 1, 3)
    with pytest.raises(ValueError):
        prover.prove_bytes(1, 1, 30, blowup_bits=2)


def test_workload_streams_are_seeded():
    from vortexstark_b200.workload import fib_inputs, m31_array, served_stream
    assert fib_inputs(7, 4) == fib_inputs(7, 4)
    assert all(0 <= a < 0x7FFFFFFF and 0 <= b < 0x7FFFFFFF for a, b in fib_inputs(1, 100))
    x = m31_array(3, 1 << 12)
    assert x.dtype == np.uint32 and int(x.max()) < 0x7FFFFFFF
    s = served_stream(11)
    assert len(s) == 512 and {r[0] for r in s} <= {16, 18, 20, 22, 24}
    frac16 = sum(r[0] == 16 for r in s) / 512
    assert 0.3 < frac16 < 0.5


def test_package_imports_no_oracle():
    """The product package never reaches into oracle/ (the oracle)."""
    root = os.path.dirname(vortexstark_b200.__file__)
    for dirpath, _, files in os.walk(root):
        for f in files:
            if f.endswith((".py", ".cu", ".cuh", ".h")):
                txt = open(os.path.join(dirpath, f)).read()
                assert "from oracle" not in txt and "import oracle" not in txt and "vx_oracle" not in txt, f
