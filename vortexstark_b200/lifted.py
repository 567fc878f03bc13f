"""Batched lifted commitment of uneven-size M31 columns ("LIFT" v1).

The multi-column stwo commitment on the B200: every column is extended in the
stwo format (``PolyOps::evaluate_polynomials``, crates/cuda-backend/src/
poly_ops.rs:676-770), all rows go into one lifted Blake2s tree
(``MerkleOpsLifted::build_leaves``, merkle_ops.rs:47-160), a random QM31
combination of the lifted columns (the lift map of accumulate_lift.cu:26-31)
is folded by FRI with the stwo twiddles (fri_ops.rs:44-255), and every tree
is opened at queries from ``draw_query_indices`` (channel.rs:102-116).

``LiftedCommitter`` keeps one shape's buffers and tables on the device
(columns uploaded or written in place, the schedule optionally replayed as
one CUDA graph); ``commit_lifted`` is the one-call form.  ``parse_lifted`` and
``verify_lifted`` read the words back and check them on the host: transcript
replay, every authentication path, and every fold equation.
"""
from __future__ import annotations

import ctypes as C
import hashlib
import struct
from dataclasses import dataclass, field

from . import _lib
from .channel import Channel
from .circle import Coset
from .field import P, m31_inv, qm31_add, qm31_mul, qm31_mul_m31, qm31_sub
from .merkle import hash_leaf, verify_auth_path

MAGIC = 0x5446494C  # "LIFT"


def _u32s(vals):
    return (C.c_uint32 * len(vals))(*vals)


def lifted_size(log_sizes, blowup_bits: int = 2, n_queries: int = 80) -> int:
    """Bytes of the commitment words (0 if the shape is unsupported)."""
    logs = list(log_sizes)
    return int(_lib.lib().vx_lifted_size(len(logs), _u32s(logs), blowup_bits, n_queries))


class LiftedCommitter:
    """Device state of one shape: input columns, LDEs, trees, FRI layers,
    transcript and the commitment words."""

    def __init__(self, log_sizes, blowup_bits: int = 2, n_queries: int = 80):
        import torch

        self.log_sizes = list(log_sizes)
        self.blowup_bits, self.n_queries = blowup_bits, n_queries
        self.size = lifted_size(self.log_sizes, blowup_bits, n_queries)
        if not self.size:
            raise _lib.VortexError(_lib.VX_ERR_ARG, "unsupported lifted-commitment shape")
        self._h = C.c_void_p()
        _lib.check(_lib.lib().vx_lifted_create(len(self.log_sizes), _u32s(self.log_sizes), blowup_bits, n_queries,
                                               C.byref(self._h)))
        self.host = torch.empty(self.size, dtype=torch.uint8, pin_memory=True)

    def column_ptr(self, c: int) -> int:
        """Device address of input column c (2^L_c words)."""
        p = C.c_void_p()
        _lib.check(_lib.lib().vx_lifted_column(self._h, c, C.byref(p)))
        return int(p.value)

    def upload_async(self, host_ptrs, stream=None) -> None:
        """Copy host columns (addresses of 2^L_c words each) to the device."""
        arr = (C.c_void_p * len(host_ptrs))(*host_ptrs)
        _lib.check(_lib.lib().vx_lifted_upload_async(self._h, arr, C.c_void_p(stream) if stream else None))

    def commit_async(self, stream=None, graph: bool = False) -> None:
        s = C.c_void_p(stream) if stream else None
        fn = _lib.lib().vx_lifted_commit_graph if graph else _lib.lib().vx_lifted_commit_async
        _lib.check(fn(self._h, s))

    def stage_async(self, stage: int, stream=None) -> None:
        _lib.check(_lib.lib().vx_lifted_stage_async(self._h, stage, C.c_void_p(stream) if stream else None))

    def fetch_async(self, stream=None) -> None:
        _lib.check(_lib.lib().vx_lifted_fetch_async(self._h, self.host.data_ptr(), C.c_void_p(stream) if stream else None))

    def result_bytes(self) -> bytes:
        _lib.check(_lib.lib().vx_lifted_check(self._h))
        return self.host.numpy().tobytes()

    def launches(self) -> int:
        return int(_lib.lib().vx_lifted_launches(self._h))

    def device_bytes(self) -> int:
        return int(_lib.lib().vx_lifted_device_bytes(self._h))

    def close(self) -> None:
        if self._h:
            _lib.lib().vx_lifted_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def commit_lifted(columns, blowup_bits: int = 2, n_queries: int = 80) -> bytes:
    """One call: host columns (numpy u32 arrays of 2^L_c values, ascending
    size) in, commitment words out (vx_commit_lifted)."""
    import numpy as np

    cols = [np.ascontiguousarray(c, dtype=np.uint32) for c in columns]
    logs = [int(len(c)).bit_length() - 1 for c in cols]
    size = lifted_size(logs, blowup_bits, n_queries)
    if not size:
        raise _lib.VortexError(_lib.VX_ERR_ARG, "unsupported lifted-commitment shape")
    ptrs = (C.c_void_p * len(cols))(*[c.ctypes.data for c in cols])
    buf = bytearray(size)
    n = C.c_size_t()
    _lib.check(_lib.lib().vx_commit_lifted(ptrs, _u32s(logs), len(cols), blowup_bits, n_queries,
                                           C.addressof((C.c_uint8 * size).from_buffer(buf)), size, C.byref(n)))
    return bytes(memoryview(buf)[: n.value])


@dataclass
class Opening:
    values: list = field(default_factory=list)    # per query: tuple of words at q
    svalues: list = field(default_factory=list)   # at q ^ 1
    paths: list = field(default_factory=list)     # per query: list of 8-word siblings
    spaths: list = field(default_factory=list)


@dataclass
class LiftedCommitment:
    n_cols: int
    blowup_bits: int
    lifting_log: int
    log_sizes: list
    lifted_root: tuple
    comb_root: tuple
    fri_roots: list
    last_layer: list
    queries: list
    lifted: Opening
    comb: Opening
    fri: list


def parse_lifted(data: bytes) -> LiftedCommitment:
    w = struct.unpack(f"<{len(data) // 4}I", data)
    pos = 0

    def take(k):
        nonlocal pos
        if pos + k > len(w):
            raise ValueError("LIFT words truncated")
        out = w[pos:pos + k]
        pos += k
        return out

    magic, ver, n_cols, B, S = take(5)
    if magic != MAGIC or ver != 1:
        raise ValueError("not a LIFT v1 commitment")
    logs = list(take(n_cols))
    r0, r1 = tuple(take(8)), tuple(take(8))
    (nfri,) = take(1)
    froots = [tuple(take(8)) for _ in range(nfri)]
    (nlast,) = take(1)
    last = [tuple(take(4)) for _ in range(nlast)]
    (nq,) = take(1)
    qs = list(take(nq))

    def opening(width, depth):
        (n,) = take(1)
        o = Opening()
        o.values = [tuple(take(width)) for _ in range(n)]
        o.svalues = [tuple(take(width)) for _ in range(n)]
        for dst in (o.paths, o.spaths):
            for _ in range(n):
                (d,) = take(1)
                if d != depth:
                    raise ValueError("path depth mismatch")
                dst.append([tuple(take(8)) for _ in range(depth)])
        return o

    lifted = opening(n_cols, S)
    comb = opening(4, S)
    (nfd,) = take(1)
    fri = [opening(4, S - 1 - k) for k in range(nfd)]
    if pos != len(w):
        raise ValueError("trailing words")
    return LiftedCommitment(n_cols, B, S, logs, r0, r1, froots, last, qs, lifted, comb, fri)


def _lifted_leaf(row) -> tuple:
    """merkle_leaves_lifted.cu:25-98: Blake2s of every column's word, in order."""
    return struct.unpack("<8I", hashlib.blake2s(struct.pack(f"<{len(row)}I", *row)).digest())


def _brev(x: int, bits: int) -> int:
    r = 0
    for _ in range(bits):
        r = (r << 1) | (x & 1)
        x >>= 1
    return r


def _circle_fold_tw(log: int, j: int) -> int:
    """fri_ops.rs:44-66: 1 / y(CircleDomain(half_odds(log-1)).at(brev(2j, log)))."""
    k = _brev(j << 1, log)
    hc = Coset.half_odds(log - 1)
    half = 1 << (log - 1)
    p = hc.at(k) if k < half else hc.at(k - half).conjugate()
    return m31_inv(p.y)


def _line_fold_tw(log: int, j: int) -> int:
    """fri_ops.rs:68-92: 1 / x(half_odds(log).at(brev(2j, log)))."""
    return m31_inv(Coset.half_odds(log).at(_brev(j << 1, log)).x)


def _fold(f0, f1, alpha, tw):
    return qm31_add(qm31_add(f0, f1), qm31_mul(alpha, qm31_mul_m31(qm31_sub(f0, f1), tw)))


class LiftedVerificationError(ValueError):
    pass


def verify_lifted(data: bytes, n_queries: int | None = None) -> LiftedCommitment:
    """Replay the transcript, check every path and every fold equation at the
    queries (C is checked against the lifted rows through the combination)."""
    c = parse_lifted(data)
    S, B = c.lifting_log, c.blowup_bits
    if any(c.log_sizes[i] > c.log_sizes[i + 1] for i in range(c.n_cols - 1)):
        raise LiftedVerificationError("log sizes not ascending")
    if S != c.log_sizes[-1] + B or len(c.fri_roots) != S - 3 or len(c.last_layer) != 8:
        raise LiftedVerificationError("shape mismatch")
    nq = len(c.queries)
    if n_queries is not None and nq != n_queries:
        raise LiftedVerificationError("query count mismatch")
    ch = Channel()
    ch.mix_digest(c.lifted_root)
    alpha = ch.draw_felt()
    ch.mix_digest(c.comb_root)
    alphas = [ch.draw_felt()]
    for k, r in enumerate(c.fri_roots):
        ch.mix_digest(r)
        if k + 1 < len(c.fri_roots):
            alphas.append(ch.draw_felt())
    ch.mix_felts(c.last_layer)
    qs = ch.draw_query_indices(S, nq)
    if qs != c.queries:
        raise LiftedVerificationError("query indices differ from the transcript")
    # authentication paths
    for label, root, op, leaf, shift in (
            ("lifted", c.lifted_root, c.lifted, _lifted_leaf, 0),
            ("combination", c.comb_root, c.comb, hash_leaf, 0)):
        for j, q in enumerate(qs):
            if not verify_auth_path(root, leaf(op.values[j]), q >> shift, op.paths[j]):
                raise LiftedVerificationError(f"{label} path at query {j}")
            if not verify_auth_path(root, leaf(op.svalues[j]), (q >> shift) ^ 1, op.spaths[j]):
                raise LiftedVerificationError(f"{label} sibling path at query {j}")
    for k, (root, op) in enumerate(zip(c.fri_roots, c.fri)):
        for j, q in enumerate(qs):
            i = q >> (k + 1)
            if not verify_auth_path(root, hash_leaf(op.values[j]), i, op.paths[j]):
                raise LiftedVerificationError(f"FRI layer {k} path at query {j}")
            if not verify_auth_path(root, hash_leaf(op.svalues[j]), i ^ 1, op.spaths[j]):
                raise LiftedVerificationError(f"FRI layer {k} sibling path at query {j}")
    # the combination at q and q ^ 1 from the opened rows
    pw = [(1, 0, 0, 0)]
    for _ in range(1, c.n_cols):
        pw.append(qm31_mul(pw[-1], alpha))
    for j in range(nq):
        for row, val in ((c.lifted.values[j], c.comb.values[j]), (c.lifted.svalues[j], c.comb.svalues[j])):
            acc = (0, 0, 0, 0)
            for ci, v in enumerate(row):
                acc = qm31_add(acc, qm31_mul_m31(pw[ci], v))
            if acc != tuple(val):
                raise LiftedVerificationError(f"combination mismatch at query {j}")
    # fold equations: circle fold C -> F0, line folds F(k-1) -> F(k), last layer
    for j, q in enumerate(qs):
        i = q >> 1
        f0, f1 = (c.comb.values[j], c.comb.svalues[j]) if q % 2 == 0 else (c.comb.svalues[j], c.comb.values[j])
        want = _fold(f0, f1, alphas[0], _circle_fold_tw(S, i))
        if want != (c.fri[0].values[j]):
            raise LiftedVerificationError(f"circle fold at query {j}")
        for k in range(1, len(c.fri)):
            i_prev = q >> k
            f0, f1 = ((c.fri[k - 1].values[j], c.fri[k - 1].svalues[j]) if i_prev % 2 == 0
                      else (c.fri[k - 1].svalues[j], c.fri[k - 1].values[j]))
            want = _fold(f0, f1, alphas[k], _line_fold_tw(S - k, i_prev >> 1))
            if want != c.fri[k].values[j]:
                raise LiftedVerificationError(f"line fold {k} at query {j}")
        kl = len(c.fri) - 1
        il = q >> (kl + 1)
        if c.fri[kl].values[j] != c.last_layer[il] or c.fri[kl].svalues[j] != c.last_layer[il ^ 1]:
            raise LiftedVerificationError(f"last layer at query {j}")
    return c
