"""StarkProof and its "KRAK" v1 byte layout.

Mirrors ``StarkProof`` / ``QueryDecommitment`` (src/prover.rs:127-166) and
``serialize_proof`` / ``deserialize_proof`` (src/bin/stark_cli.rs:1051-1233):
a little-endian u32 stream of magic 0x4B52414B, version 1, log_n, a, b, the
trace and quotient roots, the FRI roots, the last layer (8 QM31), the query
indices, then the trace, quotient and FRI decommitments.
"""
from __future__ import annotations

import struct
from dataclasses import dataclass, field

MAGIC = 0x4B52414B
VERSION = 1

# Protocol constants of the Fibonacci prover (src/prover.rs:104-125).
BLOWUP_BITS = 2
N_QUERIES = 80
LOG_LAST_LAYER_DEGREE_BOUND = 3  # src/fri.rs:265


@dataclass
class QueryDecommitment:
    values: list
    sibling_values: list
    auth_paths: list  # list of paths, each a list of 8-word tuples (leaf -> root)
    sibling_auth_paths: list


@dataclass
class StarkProof:
    trace_commitment: tuple
    quotient_commitment: tuple
    fri_commitments: list
    fri_last_layer: list  # 8 QM31 as 4-tuples
    log_trace_size: int
    public_inputs: tuple
    query_indices: list
    trace_decommitment: QueryDecommitment
    quotient_decommitment: QueryDecommitment
    fri_decommitments: list = field(default_factory=list)


class _Reader:
    def __init__(self, data: bytes):
        self.w = struct.unpack(f"<{len(data) // 4}I", data[: len(data) // 4 * 4])
        self.i = 0
        self.nbytes = len(data)

    def u32(self) -> int:
        if self.i >= len(self.w):
            raise ValueError("truncated proof")
        v = self.w[self.i]
        self.i += 1
        return v

    def arr(self, n: int) -> tuple:
        if self.i + n > len(self.w):
            raise ValueError("truncated proof")
        v = self.w[self.i:self.i + n]
        self.i += n
        return tuple(v)


def _read_decom(r: _Reader, width: int) -> QueryDecommitment:
    n = r.u32()
    if width == 1:
        vals = list(r.arr(n))
        svals = list(r.arr(n))
    else:
        vals = [r.arr(width) for _ in range(n)]
        svals = [r.arr(width) for _ in range(n)]

    def paths():
        out = []
        for _ in range(n):
            d = r.u32()
            out.append([r.arr(8) for _ in range(d)])
        return out

    p = paths()
    sp = paths()
    return QueryDecommitment(vals, svals, p, sp)


def deserialize_proof(data: bytes) -> StarkProof:
    """stark_cli.rs:1189-1233"""
    if len(data) % 4:
        raise ValueError("proof length is not a multiple of 4")
    r = _Reader(data)
    if r.u32() != MAGIC:
        raise ValueError("invalid proof file (bad magic)")
    v = r.u32()
    if v != VERSION:
        raise ValueError(f"unsupported proof version {v}")
    log_n, a, b = r.u32(), r.u32(), r.u32()
    tc, qc = r.arr(8), r.arr(8)
    nf = r.u32()
    frs = [r.arr(8) for _ in range(nf)]
    nl = r.u32()
    last = [r.arr(4) for _ in range(nl)]
    nq = r.u32()
    qi = list(r.arr(nq))
    td = _read_decom(r, 1)
    qd = _read_decom(r, 4)
    nfd = r.u32()
    fds = [_read_decom(r, 4) for _ in range(nfd)]
    if r.i != len(r.w):
        raise ValueError("trailing bytes after proof")
    return StarkProof(tc, qc, frs, last, log_n, (a, b), qi, td, qd, fds)


def _write_decom(w: list, d: QueryDecommitment, width: int) -> None:
    w.append(len(d.values))
    for v in d.values:
        w.extend([v] if width == 1 else v)
    for v in d.sibling_values:
        w.extend([v] if width == 1 else v)
    for paths in (d.auth_paths, d.sibling_auth_paths):
        for p in paths:
            w.append(len(p))
            for h in p:
                w.extend(h)


def serialize_proof(p: StarkProof) -> bytes:
    """stark_cli.rs:1092-1123"""
    w = [MAGIC, VERSION, p.log_trace_size, p.public_inputs[0], p.public_inputs[1]]
    w += list(p.trace_commitment) + list(p.quotient_commitment)
    w.append(len(p.fri_commitments))
    for c in p.fri_commitments:
        w += list(c)
    w.append(len(p.fri_last_layer))
    for v in p.fri_last_layer:
        w += list(v)
    w.append(len(p.query_indices))
    w += list(p.query_indices)
    _write_decom(w, p.trace_decommitment, 1)
    _write_decom(w, p.quotient_decommitment, 4)
    w.append(len(p.fri_decommitments))
    for d in p.fri_decommitments:
        _write_decom(w, d, 4)
    return struct.pack(f"<{len(w)}I", *w)
