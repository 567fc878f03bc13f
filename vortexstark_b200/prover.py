"""Fibonacci STARK prover on the B200 (host side).

Mirrors the reference's prover entry points (src/prover.rs:172-319, 2278-2319):
``prove``, ``prove_lean``, ``prove_cached`` with a ``ProverCache`` and the
``ProverPipeline`` batch loop.  All of them produce the same proof, as the
reference's variants do; the whole commitment path runs on the device in
libvortex_b200 (trace, LDE, trace/quotient/FRI commitments, transcript, query
decommitment), and the host receives the finished proof bytes.
"""
from __future__ import annotations

import ctypes as C

from . import _lib
from .proof import BLOWUP_BITS, N_QUERIES, StarkProof, deserialize_proof

P = 0x7FFFFFFF


def proof_size(log_n: int, blowup_bits: int = BLOWUP_BITS, n_queries: int = N_QUERIES) -> int:
    return int(_lib.lib().vx_proof_size(log_n, blowup_bits, n_queries))


def _check_inputs(a: int, b: int, log_n: int, blowup_bits: int) -> None:
    if not (0 <= a < P and 0 <= b < P):
        raise ValueError("public inputs must be canonical M31 values in [0, 2^31 - 1)")
    if log_n < 4:
        raise ValueError("trace too small (log_n >= 4 required, prover.rs:266)")
    if blowup_bits < 1 or log_n + blowup_bits > 31:
        raise ValueError("log_n + blowup_bits must be <= 31 (the M31 circle group has order 2^31)")


def prove_bytes(a: int, b: int, log_n: int, blowup_bits: int = BLOWUP_BITS, n_queries: int = N_QUERIES) -> bytes:
    """Whole proof through the C ABI (vx_prove_fib) into a host buffer."""
    _check_inputs(a, b, log_n, blowup_bits)
    L = _lib.lib()
    size = proof_size(log_n, blowup_bits, n_queries)
    buf = bytearray(size)
    n = C.c_size_t()
    _lib.check(L.vx_prove_fib(a, b, log_n, blowup_bits, n_queries, C.addressof((C.c_uint8 * size).from_buffer(buf)),
                              size, C.byref(n)))
    return bytes(memoryview(buf)[: n.value])


def prove_batch_bytes(inputs, log_n: int, blowup_bits: int = BLOWUP_BITS, n_queries: int = N_QUERIES,
                      out: bytearray | None = None) -> list[bytes]:
    """ProverPipeline::prove_batch (prover.rs:2305-2311) through the C ABI
    (vx_prove_fib_batch): the proofs of [(a, b), ...], two in flight."""
    pairs = list(inputs)
    for a, b in pairs:
        _check_inputs(a, b, log_n, blowup_bits)
    size = proof_size(log_n, blowup_bits, n_queries)
    n = len(pairs)
    buf = out if out is not None and len(out) >= n * size else bytearray(max(n, 1) * size)
    av = (C.c_uint32 * max(n, 1))(*[p[0] for p in pairs])
    bv = (C.c_uint32 * max(n, 1))(*[p[1] for p in pairs])
    got = C.c_size_t()
    _lib.check(_lib.lib().vx_prove_fib_batch(av, bv, n, log_n, blowup_bits, n_queries,
                                              C.addressof((C.c_uint8 * len(buf)).from_buffer(buf)), len(buf),
                                              C.byref(got)))
    mv = memoryview(buf)
    return [bytes(mv[i * size:(i + 1) * size]) for i in range(n)]


def prove(a: int, b: int, log_n: int) -> StarkProof:
    """prover.rs:221 — prove the Fibonacci AIR with public inputs (a, b)."""
    return deserialize_proof(prove_bytes(a, b, log_n))


def prove_lean(a: int, b: int, log_n: int) -> StarkProof:
    """prover.rs:249 — same proof as ``prove`` (the device path is already lean)."""
    return prove(a, b, log_n)


class ProverCache:
    """Device-resident state for repeated proofs of one size (prover.rs:172-210):
    twiddle tables shared per size, plus one proof slot (all buffers of one
    in-flight proof) and a pinned host buffer for its bytes."""

    def __init__(self, log_n: int, blowup_bits: int = BLOWUP_BITS, n_queries: int = N_QUERIES):
        _check_inputs(0, 0, log_n, blowup_bits)
        import torch

        self.log_n, self.blowup_bits, self.n_queries = log_n, blowup_bits, n_queries
        self.log_eval_size = log_n + blowup_bits
        self._p = C.c_void_p()
        _lib.check(_lib.lib().vx_prover_create(log_n, blowup_bits, n_queries, C.byref(self._p)))
        self.size = proof_size(log_n, blowup_bits, n_queries)
        self.host = torch.empty(self.size, dtype=torch.uint8, pin_memory=True)

    def prove_async(self, a: int, b: int, stream=None) -> None:
        """Enqueue a proof and the copy of its bytes into the pinned buffer."""
        _check_inputs(a, b, self.log_n, self.blowup_bits)
        s = C.c_void_p(stream) if stream else None
        L = _lib.lib()
        _lib.check(L.vx_prover_prove_async(self._p, a, b, s))
        _lib.check(L.vx_prover_fetch_async(self._p, self.host.data_ptr(), s))

    def result_bytes(self) -> bytes:
        """Proof bytes of the last proof (call after its stream has drained)."""
        _lib.check(_lib.lib().vx_prover_check(self._p))
        return self.host.numpy().tobytes()

    def slot_bytes(self) -> int:
        return int(_lib.lib().vx_prover_slot_bytes(self._p))

    def table_bytes(self) -> int:
        return int(_lib.lib().vx_prover_table_bytes(self._p))

    def close(self) -> None:
        if self._p:
            _lib.lib().vx_prover_destroy(self._p)
            self._p = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def prove_cached_bytes(a: int, b: int, cache: ProverCache, stream=None) -> bytes:
    import torch

    cache.prove_async(a, b, stream)
    if stream:
        torch.cuda.ExternalStream(stream).synchronize()
    else:
        torch.cuda.synchronize()
    return cache.result_bytes()


def prove_cached(a: int, b: int, cache: ProverCache) -> StarkProof:
    """prover.rs:231 — prove with pre-computed, device-resident state."""
    return deserialize_proof(prove_cached_bytes(a, b, cache))


class ProverPipeline:
    """prover.rs:2278-2319 — sequential batch over one cache."""

    def __init__(self, log_n: int):
        self.cache = ProverCache(log_n)

    def prove_batch(self, inputs) -> list:
        return [prove_cached(a, b, self.cache) for a, b in inputs]
