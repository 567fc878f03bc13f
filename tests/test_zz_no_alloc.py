"""vx_prove_fib_noalloc: the whole proof with no device allocation.

Some callers cannot call cudaMalloc — hosts whose device memory belongs to
another allocator, sandboxes that forbid allocation after start-up.  This
entry point keeps all its device scratch in one static array of the library
(and, being synchronous on the legacy stream, is never called under a stream
capture).  Its proofs must equal those of
the allocating entry point (vx_prove_fib) byte for byte, on consecutive calls
that reuse the shared array.  This file is collected last on purpose.
"""
import ctypes as C

import pytest

from vortexstark_b200 import _lib

pytestmark = pytest.mark.gpu


def _prove(fn, a, b, log_n, blowup=2, nq=80):
    L = _lib.lib()
    size = int(L.vx_proof_size(log_n, blowup, nq))
    buf = (C.c_uint8 * size)()
    n = C.c_size_t()
    rc = getattr(L, fn)(a, b, log_n, blowup, nq, C.addressof(buf), size, C.byref(n))
    return rc, bytes(buf[: n.value])


def test_noalloc_matches_allocating_entry_point_twice():
    cases = [(123456789, 987654321, 12), (5, 8, 10), (0x7FFFFFFE, 1, 12)]
    for a, b, log_n in cases:  # consecutive calls share the static scratch
        rc, got = _prove("vx_prove_fib_noalloc", a, b, log_n)
        assert rc == 0, _lib.last_error()
        rc2, want = _prove("vx_prove_fib", a, b, log_n)
        assert rc2 == 0, _lib.last_error()
        assert got == want, (a, b, log_n)
    rc, got = _prove("vx_prove_fib_noalloc", 3, 4, 13, blowup=1, nq=40)
    rc2, want = _prove("vx_prove_fib", 3, 4, 13, blowup=1, nq=40)
    assert rc == 0 and rc2 == 0 and got == want


def test_noalloc_rejects_sizes_beyond_its_limit():
    L = _lib.lib()
    buf = (C.c_uint8 * 16)()
    n = C.c_size_t()
    rc = L.vx_prove_fib_noalloc(1, 1, 13, 2, 80, C.addressof(buf), 16, C.byref(n))
    assert rc == _lib.VX_ERR_ARG
    assert "log_n + blowup_bits <= 14" in _lib.last_error()
