"""Blake2s Merkle commitments on the B200.

Mirrors src/merkle.rs: ``MerkleTree.commit`` (28-130, full tree),
``commit_root_only`` (142-231), ``commit_root_soa4`` (236-312), the
``*_with_subtrees`` forms that also return the 1024-leaf tile roots
(317-451), ``auth_path`` / ``batch_auth_paths`` (455-497) and the host
helpers ``hash_leaf`` / ``hash_pair`` / ``verify_auth_path`` (520-593, 864-884).
Leaf = Blake2s(LE words of the row), node = Blake2s(left || right).
"""
from __future__ import annotations

import hashlib
import struct

from . import _lib

HASH_WORDS = 8
TILE_SIZE = 1024


def _empty(n):
    import torch

    return torch.empty(max(int(n), 1), dtype=torch.int32, device="cuda")


def _words(t):
    import numpy as np

    return t.detach().cpu().numpy().view(np.uint32)


def _ptrs(cols):
    import torch

    return torch.tensor([c.data_ptr() for c in cols], dtype=torch.int64, device="cuda")


def hash_leaf(values) -> tuple:
    """merkle.rs:570-593"""
    vals = list(values)[:16]
    return struct.unpack("<8I", hashlib.blake2s(struct.pack(f"<{len(vals)}I", *vals)).digest())


def hash_pair(left, right) -> tuple:
    """merkle.rs:864-884"""
    return struct.unpack("<8I", hashlib.blake2s(struct.pack("<16I", *left, *right)).digest())


def verify_auth_path(expected_root, leaf_hash, index: int, path) -> bool:
    """merkle.rs:520-566"""
    cur = tuple(leaf_hash)
    for sib in path:
        cur = hash_pair(cur, sib) if index % 2 == 0 else hash_pair(sib, cur)
        index //= 2
    return cur == tuple(expected_root)


class MerkleTree:
    """Full tree with every layer kept on the device (layers[0] = root)."""

    def __init__(self, layers, log_n_leaves):
        self.layers = layers
        self.log_n_leaves = log_n_leaves

    @staticmethod
    def _leaf_hashes(columns, n):
        L = _lib.lib()
        out = _empty(n * 8)
        if len(columns) == 1:
            L.cuda_merkle_hash_leaves_forge_single(columns[0].data_ptr(), out.data_ptr(), n)
        elif len(columns) == 4:
            L.cuda_merkle_hash_leaves_forge_quad(*[c.data_ptr() for c in columns], out.data_ptr(), n)
        else:
            ptrs = _ptrs(columns)
            L.cuda_merkle_hash_leaves(ptrs.data_ptr(), out.data_ptr(), len(columns), n)
        return out

    @classmethod
    def commit(cls, columns, log_n_leaves: int) -> "MerkleTree":
        """merkle.rs:28-130"""
        L = _lib.lib()
        n = 1 << log_n_leaves
        cur = cls._leaf_hashes(columns, n)
        layers = [cur]
        size = n
        while size > 1:
            size //= 2
            par = _empty(size * 8)
            L.cuda_merkle_hash_nodes(cur.data_ptr(), par.data_ptr(), size)
            layers.append(par)
            cur = par
        return cls(list(reversed(layers)), log_n_leaves)

    @classmethod
    def commit_soa4(cls, c0, c1, c2, c3, log_n_leaves: int) -> "MerkleTree":
        """merkle.rs:907-973"""
        return cls.commit([c0, c1, c2, c3], log_n_leaves)

    def root(self) -> tuple:
        return tuple(int(x) for x in _words(self.layers[0][:8]))

    def auth_path(self, index: int) -> list:
        return self.batch_auth_paths([index])[0]

    def batch_auth_paths(self, indices) -> list:
        """merkle.rs:473-497 — siblings from the leaf level up to below the root."""
        paths = [[] for _ in indices]
        cur = list(indices)
        for layer_idx in range(self.log_n_leaves, 0, -1):
            host = _words(self.layers[layer_idx]).reshape(-1, 8)
            for q, idx in enumerate(cur):
                paths[q].append(tuple(int(x) for x in host[idx ^ 1]))
                cur[q] = idx // 2
        return paths

    @staticmethod
    def commit_root_only_with_subtrees(columns, log_n_leaves: int):
        """merkle.rs:386-451 — root and the 1024-leaf tile roots."""
        L = _lib.lib()
        n = 1 << log_n_leaves
        if n < TILE_SIZE:
            t = MerkleTree.commit(columns, log_n_leaves)
            return t.root(), []
        ptrs = _ptrs(columns)
        tiles = n // TILE_SIZE
        sub = _empty(tiles * 8)
        L.cuda_merkle_tiled_generic(ptrs.data_ptr(), sub.data_ptr(), len(columns), n)
        return MerkleTree._reduce(sub, tiles), [tuple(int(x) for x in r) for r in _words(sub).reshape(-1, 8)]

    @staticmethod
    def commit_root_soa4_with_subtrees(c0, c1, c2, c3, log_n_leaves: int):
        """merkle.rs:317-383"""
        L = _lib.lib()
        n = 1 << log_n_leaves
        if n < TILE_SIZE:
            t = MerkleTree.commit([c0, c1, c2, c3], log_n_leaves)
            return t.root(), []
        tiles = n // TILE_SIZE
        sub = _empty(tiles * 8)
        L.cuda_merkle_tiled_soa4(c0.data_ptr(), c1.data_ptr(), c2.data_ptr(), c3.data_ptr(), sub.data_ptr(), n)
        return MerkleTree._reduce(sub, tiles), [tuple(int(x) for x in r) for r in _words(sub).reshape(-1, 8)]

    @staticmethod
    def commit_root_only(columns, log_n_leaves: int) -> tuple:
        return MerkleTree.commit_root_only_with_subtrees(columns, log_n_leaves)[0]

    @staticmethod
    def _reduce(cur, size: int) -> tuple:
        """prover.rs:1170-1210 — hash_nodes down to <= 1024, then one block."""
        L = _lib.lib()
        while size > 1024:
            size //= 2
            par = _empty(size * 8)
            L.cuda_merkle_hash_nodes(cur.data_ptr(), par.data_ptr(), size)
            cur = par
        if size > 1:
            root = _empty(8)
            L.cuda_merkle_reduce_to_root(cur.data_ptr(), root.data_ptr(), size)
            cur = root
        return tuple(int(x) for x in _words(cur[:8]))


class FusedRoot:
    """Root-only commitment through the fused tree kernels
    (vx_merkle_root_cols): the drop-in for ``commit_root_only`` /
    ``commit_root_soa4`` with a reusable device workspace."""

    def __init__(self, log_n_leaves: int):
        import torch

        self.log_n_leaves = log_n_leaves
        self.words = int(_lib.lib().vx_merkle_workspace_words(log_n_leaves))
        if not self.words:
            raise _lib.VortexError(_lib.VX_ERR_ARG, f"unsupported tree size 2^{log_n_leaves}")
        self.workspace = torch.empty(self.words, dtype=torch.int32, device="cuda")
        self.root_dev = torch.empty(8, dtype=torch.int32, device="cuda")

    def commit_async(self, columns, stream=None) -> None:
        import ctypes as C

        ptrs = (C.c_void_p * len(columns))(*[c.data_ptr() for c in columns])
        _lib.check(_lib.lib().vx_merkle_root_cols(ptrs, len(columns), self.log_n_leaves, self.workspace.data_ptr(),
                                                  self.words, self.root_dev.data_ptr(),
                                                  C.c_void_p(stream) if stream else None))

    def commit(self, columns) -> tuple:
        self.commit_async(columns)
        return tuple(int(x) for x in _words(self.root_dev))


def build_leaves_lifted(columns, lifting_log_size: int):
    """crates/cuda-backend/src/merkle_ops.rs:48-173 — one lifted leaf hash per
    row of the largest column; columns must be sorted by ascending size."""
    import torch

    L = _lib.lib()
    sched = []
    i = 0
    while i < len(columns):
        ls = int(columns[i].numel()).bit_length() - 1
        j = i
        while j < len(columns) and int(columns[j].numel()).bit_length() - 1 == ls:
            j += 1
        for s in range(i, j, 16):
            e = min(s + 16, j)
            idx = list(range(s, e)) + [0] * (16 - (e - s))
            sched += idx + [e - s, ls]
        i = j
    d_sched = torch.tensor(sched, dtype=torch.int64, device="cuda").to(torch.int32)
    ptrs = _ptrs(columns)
    n = 1 << lifting_log_size
    out = _empty(n * 8)
    L.cuda_build_leaves_lifted(ptrs.data_ptr(), d_sched.data_ptr(), len(sched) // 18, lifting_log_size,
                               out.data_ptr(), n)
    return out
