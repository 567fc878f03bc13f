"""ctypes bindings for the CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()``
and by the CPU-baseline leg of ``bench.py``.  The product package
(``vortexstark_b200``) never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

P = 0x7FFFFFFF
U32P = C.POINTER(C.c_uint32)


def build() -> str:
    """Compile liboracle.so with the committed Makefile (gcc + OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True, env={**os.environ, "CC": "gcc"})
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        L.vxo_prove.argtypes = [C.c_uint32] * 5 + [C.POINTER(C.POINTER(C.c_uint8)), C.POINTER(C.c_size_t)]
        L.vxo_prove.restype = C.c_int
        L.vxo_prove_lean.argtypes = [C.c_uint32] * 5 + [C.POINTER(C.POINTER(C.c_uint8)), C.POINTER(C.c_size_t)]
        L.vxo_prove_lean.restype = C.c_int
        L.vxo_verify.argtypes = [C.POINTER(C.c_uint8), C.c_size_t, C.c_uint32, C.c_uint32, C.c_char_p, C.c_size_t]
        L.vxo_verify.restype = C.c_int
        L.vxo_proof_size.argtypes = [C.c_uint32] * 3
        L.vxo_proof_size.restype = C.c_size_t
        L.vxo_prove_roots.argtypes = [C.c_uint32] * 4 + [U32P] * 3
        L.vxo_free.argtypes = [C.c_void_p]
        L.vxo_set_threads.argtypes = [C.c_int]
        L.vxo_get_threads.restype = C.c_int
        L.vxo_blake2s.argtypes = [C.c_char_p, C.c_size_t, C.POINTER(C.c_uint8)]
        L.vxo_twiddles.argtypes = [C.c_void_p, C.c_int, U32P, U32P, U32P]
        L.vxo_ntt_evaluate.argtypes = [U32P, U32P, U32P, U32P, C.c_uint32]
        L.vxo_ntt_interpolate.argtypes = [U32P, U32P, U32P, U32P, C.c_uint32]
        L.vxo_ntt_layer.argtypes = [U32P, U32P, C.c_uint32, C.c_uint64, C.c_int]
        L.vxo_bit_reverse.argtypes = [U32P, C.c_uint32]
        L.vxo_permute_hc_to_canonic_brt.argtypes = [U32P, U32P, C.c_uint32]
        L.vxo_permute_canonic_brt_to_hc.argtypes = [U32P, U32P, C.c_uint32]
        L.vxo_fibonacci_trace.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, U32P]
        L.vxo_fibonacci_quotient.argtypes = [U32P, C.c_uint64, U32P, U32P, U32P, U32P, U32P]
        L.vxo_merkle_root.argtypes = [C.POINTER(U32P), C.c_uint32, C.c_uint32, U32P]
        L.vxo_lifted_leaves.argtypes = [C.POINTER(U32P), U32P, C.c_uint32, C.c_uint32, U32P]
        L.vxo_fold_twiddles.argtypes = [C.c_void_p, C.c_int, U32P]
        L.vxo_fold_line.argtypes = [C.POINTER(U32P), U32P, U32P, C.POINTER(U32P), C.c_uint64]
        L.vxo_fold_circle_into_line.argtypes = [C.POINTER(U32P), C.POINTER(U32P), U32P, U32P, U32P, C.c_uint64]
        L.vxo_batch_inverse.argtypes = [U32P, U32P, C.c_size_t]
        L.vxo_qm31_mul.argtypes = [U32P, U32P, U32P]
        L.vxo_hash_leaf.argtypes = [U32P, C.c_uint32, U32P]
        L.vxo_hash_pair.argtypes = [U32P, U32P, U32P]
        L.vxo_stwo_twiddles.argtypes = [C.c_uint32, C.c_int, U32P]
        L.vxo_stwo_ntt_evaluate.argtypes = [U32P, U32P, C.c_uint32]
        L.vxo_stwo_ntt_interpolate.argtypes = [U32P, U32P, C.c_uint32]
        L.vxo_bit_reverse_qm31.argtypes = [U32P, U32P, C.c_uint32]
        L.vxo_accumulate_lift.argtypes = [U32P, U32P, C.c_uint64, C.c_uint32]
        L.vxo_pack_leaves.argtypes = [C.POINTER(U32P), C.POINTER(U32P), C.c_uint64]
        L.vxo_fri_chain.argtypes = [C.POINTER(U32P), C.c_uint32, U32P, U32P, U32P, U32P]
        L.vxo_eval_at_point.argtypes = [U32P, U32P, C.c_uint32, U32P]
        L.vxo_barycentric_partials.argtypes = [U32P, U32P, C.c_uint32, C.c_uint32, U32P]
        L.vxo_stwo_fold_circle_twiddles.argtypes = [C.c_uint32, U32P]
        L.vxo_lifted_size.argtypes = [C.c_uint32, U32P, C.c_uint32, C.c_uint32]
        L.vxo_lifted_size.restype = C.c_size_t
        L.vxo_commit_lifted.argtypes = [C.POINTER(U32P), U32P, C.c_uint32, C.c_uint32, C.c_uint32,
                                        C.POINTER(C.POINTER(C.c_uint8)), C.POINTER(C.c_size_t)]
        L.vxo_commit_lifted.restype = C.c_int
        L.vxo_lifted_lde.argtypes = [C.POINTER(U32P), U32P, C.c_uint32, C.c_uint32, C.POINTER(U32P)]
        L.vxo_lifted_lde.restype = C.c_int
        L.vxo_pow_prefix.argtypes = [U32P, C.c_uint32, U32P]
        L.vxo_verify_pow_nonce.argtypes = [U32P, C.c_uint32, C.c_uint64, C.c_int]
        L.vxo_verify_pow_nonce.restype = C.c_int
        L.vxo_grind_pow.argtypes = [U32P, C.c_uint32, C.c_int, C.c_uint32, C.POINTER(C.c_uint64)]
        L.vxo_grind_pow.restype = C.c_int
        for name in ("subgroup", "half_coset", "half_odds"):
            f = getattr(L, f"vxo_coset_{name}")
            f.argtypes = [C.c_uint32]
            f.restype = Coset
        L.vxo_coset_at.argtypes = [C.POINTER(Coset), C.c_uint64]
        L.vxo_coset_at.restype = Point
        L.vxo_point_pow.argtypes = [Point, C.c_uint64]
        L.vxo_point_pow.restype = Point
        L.vxo_point_mul.argtypes = [Point, Point]
        L.vxo_point_mul.restype = Point
        _lib = L
    return _lib


class Point(C.Structure):
    _fields_ = [("x", C.c_uint32), ("y", C.c_uint32)]


class Coset(C.Structure):
    _fields_ = [("initial", Point), ("step", Point), ("log_size", C.c_uint32)]


def _p(a: np.ndarray):
    assert a.dtype == np.uint32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(U32P)


def coset(kind: str, log_size: int) -> Coset:
    return getattr(lib(), f"vxo_coset_{kind}")(log_size)


def set_threads(n: int) -> None:
    lib().vxo_set_threads(int(n))


def get_threads() -> int:
    return int(lib().vxo_get_threads())


def prove(a: int, b: int, log_n: int, blowup_bits: int = 2, n_queries: int = 80) -> bytes:
    L = lib()
    out = C.POINTER(C.c_uint8)()
    n = C.c_size_t()
    rc = L.vxo_prove(a, b, log_n, blowup_bits, n_queries, C.byref(out), C.byref(n))
    if rc:
        raise ValueError(f"oracle prove rejected its arguments (rc={rc})")
    try:
        return C.string_at(out, n.value)
    finally:
        L.vxo_free(out)


def prove_lean(a: int, b: int, log_n: int, blowup_bits: int = 2, n_queries: int = 80) -> bytes:
    """The same bytes as ``prove`` in bounded host memory (for 2^30- and
    2^31-point proofs): the quotient is recomputed where it is read and
    trees keep their levels from height 8 up."""
    L = lib()
    out = C.POINTER(C.c_uint8)()
    n = C.c_size_t()
    rc = L.vxo_prove_lean(a, b, log_n, blowup_bits, n_queries, C.byref(out), C.byref(n))
    if rc:
        raise ValueError(f"oracle prove_lean failed (rc={rc})")
    try:
        return C.string_at(out, n.value)
    finally:
        L.vxo_free(out)


def verify(proof: bytes, blowup_bits: int = 2, n_queries: int = 80) -> tuple[int, str]:
    buf = (C.c_uint8 * len(proof)).from_buffer_copy(proof)
    msg = C.create_string_buffer(256)
    rc = lib().vxo_verify(buf, len(proof), blowup_bits, n_queries, msg, 256)
    return rc, msg.value.decode()


def proof_size(log_n: int, blowup_bits: int = 2, n_queries: int = 80) -> int:
    return int(lib().vxo_proof_size(log_n, blowup_bits, n_queries))


def prove_roots(a: int, b: int, log_n: int, blowup_bits: int = 2):
    le = log_n + blowup_bits
    tr = np.zeros(8, np.uint32)
    qr = np.zeros(8, np.uint32)
    fr = np.zeros(8 * (le - 3), np.uint32)
    rc = lib().vxo_prove_roots(a, b, log_n, blowup_bits, _p(tr), _p(qr), _p(fr))
    if rc:
        raise ValueError("bad arguments")
    return tr, qr, fr.reshape(-1, 8)


def blake2s(data: bytes) -> bytes:
    out = (C.c_uint8 * 32)()
    lib().vxo_blake2s(data, len(data), out)
    return bytes(out)


def twiddles(cs: Coset, inverse: bool):
    m = 1 << cs.log_size
    line = np.zeros(max(m - 1, 1), np.uint32)
    circ = np.zeros(max(m // 2, 1), np.uint32)
    offs = np.zeros(32, np.uint32)
    lib().vxo_twiddles(C.byref(cs), int(inverse), _p(line), _p(circ), _p(offs))
    n_line = max(cs.log_size - 1, 0)
    return line[: m - 1], circ[: m // 2], offs[:n_line]


def ntt_evaluate(data: np.ndarray, cs: Coset) -> np.ndarray:
    d = np.ascontiguousarray(data, dtype=np.uint32).copy()
    line, circ, offs = twiddles(cs, False)
    offs32 = np.zeros(32, np.uint32)
    offs32[: len(offs)] = offs
    lib().vxo_ntt_evaluate(_p(d), _p(line), _p(circ), _p(offs32), cs.log_size)
    return d


def ntt_interpolate(data: np.ndarray, cs: Coset) -> np.ndarray:
    d = np.ascontiguousarray(data, dtype=np.uint32).copy()
    line, circ, offs = twiddles(cs, True)
    offs32 = np.zeros(32, np.uint32)
    offs32[: len(offs)] = offs
    lib().vxo_ntt_interpolate(_p(d), _p(line), _p(circ), _p(offs32), cs.log_size)
    return d


def ntt_layer(data: np.ndarray, tw: np.ndarray, layer_idx: int, forward: bool) -> np.ndarray:
    d = np.ascontiguousarray(data, dtype=np.uint32).copy()
    t = np.ascontiguousarray(tw, dtype=np.uint32)
    lib().vxo_ntt_layer(_p(d), _p(t), layer_idx, len(d), int(forward))
    return d


def bit_reverse(data: np.ndarray) -> np.ndarray:
    d = np.ascontiguousarray(data, dtype=np.uint32).copy()
    lib().vxo_bit_reverse(_p(d), int(len(d)).bit_length() - 1)
    return d


def permute_hc_to_canonic_brt(data: np.ndarray) -> np.ndarray:
    s = np.ascontiguousarray(data, dtype=np.uint32)
    d = np.zeros_like(s)
    lib().vxo_permute_hc_to_canonic_brt(_p(s), _p(d), int(len(s)).bit_length() - 1)
    return d


def permute_canonic_brt_to_hc(data: np.ndarray) -> np.ndarray:
    s = np.ascontiguousarray(data, dtype=np.uint32)
    d = np.zeros_like(s)
    lib().vxo_permute_canonic_brt_to_hc(_p(s), _p(d), int(len(s)).bit_length() - 1)
    return d


def fibonacci_trace(a: int, b: int, log_n: int) -> np.ndarray:
    out = np.zeros(1 << log_n, np.uint32)
    lib().vxo_fibonacci_trace(a, b, log_n, _p(out))
    return out


def fibonacci_quotient(ev: np.ndarray, alpha) -> np.ndarray:
    ev = np.ascontiguousarray(ev, dtype=np.uint32)
    q = np.zeros((4, len(ev)), np.uint32)
    al = np.array(alpha, np.uint32)
    lib().vxo_fibonacci_quotient(_p(ev), len(ev), _p(al), _p(q[0]), _p(q[1]), _p(q[2]), _p(q[3]))
    return q


def merkle_root(cols) -> np.ndarray:
    cols = [np.ascontiguousarray(c, dtype=np.uint32) for c in cols]
    arr = (U32P * len(cols))(*[_p(c) for c in cols])
    out = np.zeros(8, np.uint32)
    lib().vxo_merkle_root(arr, len(cols), int(len(cols[0])).bit_length() - 1, _p(out))
    return out


def lifted_leaves(cols, lifting_log: int) -> np.ndarray:
    cols = [np.ascontiguousarray(c, dtype=np.uint32) for c in cols]
    logs = np.array([int(len(c)).bit_length() - 1 for c in cols], np.uint32)
    arr = (U32P * len(cols))(*[_p(c) for c in cols])
    out = np.zeros((1 << lifting_log) * 8, np.uint32)
    lib().vxo_lifted_leaves(arr, _p(logs), len(cols), lifting_log, _p(out))
    return out.reshape(-1, 8)


def fold_twiddles(cs: Coset, extract_y: bool) -> np.ndarray:
    out = np.zeros(1 << (cs.log_size - 1), np.uint32)
    lib().vxo_fold_twiddles(C.byref(cs), int(extract_y), _p(out))
    return out


def fold_line(src: np.ndarray, tw: np.ndarray, alpha) -> np.ndarray:
    src = np.ascontiguousarray(src, dtype=np.uint32)
    half = src.shape[1] // 2
    out = np.zeros((4, half), np.uint32)
    ins = (U32P * 4)(*[_p(src[c]) for c in range(4)])
    outs = (U32P * 4)(*[_p(out[c]) for c in range(4)])
    al = np.array(alpha, np.uint32)
    lib().vxo_fold_line(ins, _p(np.ascontiguousarray(tw, dtype=np.uint32)), _p(al), outs, half)
    return out


def fold_circle_into_line(dst: np.ndarray, src: np.ndarray, tw: np.ndarray, alpha) -> np.ndarray:
    src = np.ascontiguousarray(src, dtype=np.uint32)
    dst = np.ascontiguousarray(dst, dtype=np.uint32).copy()
    half = src.shape[1] // 2
    al = np.array(alpha, np.uint32)
    al2 = qm31_mul(al, al)
    ins = (U32P * 4)(*[_p(src[c]) for c in range(4)])
    outs = (U32P * 4)(*[_p(dst[c]) for c in range(4)])
    lib().vxo_fold_circle_into_line(outs, ins, _p(np.ascontiguousarray(tw, dtype=np.uint32)), _p(al), _p(al2), half)
    return dst


def fri_chain(src: np.ndarray, state_words):
    """FRI chain with per-layer commitments of a QM31 codeword (4 x 2^L
    words, SoA) on half_coset(L), transcript started from `state_words`
    (8 words): (roots [L-1, 8], alphas [L-1, 4], last [2, 4])."""
    src = np.ascontiguousarray(src, dtype=np.uint32)
    L = int(src.shape[1]).bit_length() - 1
    ins = (U32P * 4)(*[_p(src[c]) for c in range(4)])
    st = np.ascontiguousarray(state_words, dtype=np.uint32)
    roots = np.zeros((L - 1, 8), np.uint32)
    alphas = np.zeros((L - 1, 4), np.uint32)
    last = np.zeros((2, 4), np.uint32)
    lib().vxo_fri_chain(ins, L, _p(st), _p(roots), _p(alphas), _p(last))
    return roots, alphas, last


def eval_at_point(coeffs: np.ndarray, factors: np.ndarray) -> np.ndarray:
    """Fold 2^k M31 coefficients with k QM31 factors (shape [k, 4])."""
    c = np.ascontiguousarray(coeffs, dtype=np.uint32)
    f = np.ascontiguousarray(factors, dtype=np.uint32).reshape(-1)
    k = int(len(c)).bit_length() - 1
    out = np.zeros(4, np.uint32)
    lib().vxo_eval_at_point(_p(c), _p(f), k, _p(out))
    return out


def barycentric_partials(evals: np.ndarray, weights: np.ndarray, n_blocks: int) -> np.ndarray:
    e = np.ascontiguousarray(evals, dtype=np.uint32)
    w = np.ascontiguousarray(weights, dtype=np.uint32).reshape(-1)
    out = np.zeros((n_blocks, 4), np.uint32)
    lib().vxo_barycentric_partials(_p(e), _p(w), len(e), n_blocks, _p(out))
    return out


def batch_inverse(x: np.ndarray) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.uint32)
    out = np.zeros_like(x)
    lib().vxo_batch_inverse(_p(x), _p(out), len(x))
    return out


def qm31_mul(a, b) -> np.ndarray:
    a = np.array(a, np.uint32)
    b = np.array(b, np.uint32)
    out = np.zeros(4, np.uint32)
    lib().vxo_qm31_mul(_p(a), _p(b), _p(out))
    return out


# ---- stwo-format NTT and the batched lifted commitment ----
def stwo_twiddles(log_n: int, inverse: bool = False) -> np.ndarray:
    out = np.zeros(1 << (log_n - 1), np.uint32)
    lib().vxo_stwo_twiddles(log_n, int(inverse), _p(out))
    return out


def stwo_ntt_evaluate(data: np.ndarray, tw: np.ndarray | None = None) -> np.ndarray:
    d = np.ascontiguousarray(data, dtype=np.uint32).copy()
    k = int(len(d)).bit_length() - 1
    t = stwo_twiddles(k) if tw is None else np.ascontiguousarray(tw, dtype=np.uint32)
    lib().vxo_stwo_ntt_evaluate(_p(d), _p(t), k)
    return d


def stwo_ntt_interpolate(data: np.ndarray, itw: np.ndarray | None = None) -> np.ndarray:
    d = np.ascontiguousarray(data, dtype=np.uint32).copy()
    k = int(len(d)).bit_length() - 1
    t = stwo_twiddles(k, True) if itw is None else np.ascontiguousarray(itw, dtype=np.uint32)
    lib().vxo_stwo_ntt_interpolate(_p(d), _p(t), k)
    return d


def bit_reverse_qm31(data: np.ndarray) -> np.ndarray:
    s = np.ascontiguousarray(data, dtype=np.uint32).reshape(-1)
    d = np.zeros_like(s)
    lib().vxo_bit_reverse_qm31(_p(s), _p(d), int(len(s) // 4).bit_length() - 1)
    return d


def accumulate_lift(col: np.ndarray, curr: np.ndarray) -> np.ndarray:
    c = np.ascontiguousarray(col, dtype=np.uint32).copy()
    s = np.ascontiguousarray(curr, dtype=np.uint32)
    ratio = (int(len(c)).bit_length() - 1) - (int(len(s)).bit_length() - 1)
    lib().vxo_accumulate_lift(_p(c), _p(s), len(c), ratio)
    return c


def pack_leaves(cols) -> np.ndarray:
    cols = [np.ascontiguousarray(c, dtype=np.uint32) for c in cols]
    n = len(cols[0])
    out = np.zeros((64, n // 16), np.uint32)
    ins = (U32P * 4)(*[_p(c) for c in cols])
    outs = (U32P * 64)(*[_p(out[i]) for i in range(64)])
    lib().vxo_pack_leaves(ins, outs, n)
    return out


def stwo_fold_circle_twiddles(log: int) -> np.ndarray:
    out = np.zeros(1 << (log - 1), np.uint32)
    lib().vxo_stwo_fold_circle_twiddles(log, _p(out))
    return out


def lifted_size(log_sizes, blowup_bits: int = 2, n_queries: int = 80) -> int:
    logs = np.array(log_sizes, np.uint32)
    return int(lib().vxo_lifted_size(len(logs), _p(logs), blowup_bits, n_queries))


def commit_lifted(cols, blowup_bits: int = 2, n_queries: int = 80) -> bytes:
    """The "LIFT" v1 words of the batched lifted commitment of `cols`
    (sorted by ascending size)."""
    cols = [np.ascontiguousarray(c, dtype=np.uint32) for c in cols]
    logs = np.array([int(len(c)).bit_length() - 1 for c in cols], np.uint32)
    arr = (U32P * len(cols))(*[_p(c) for c in cols])
    out = C.POINTER(C.c_uint8)()
    n = C.c_size_t()
    L = lib()
    rc = L.vxo_commit_lifted(arr, _p(logs), len(cols), blowup_bits, n_queries, C.byref(out), C.byref(n))
    if rc:
        raise ValueError(f"oracle commit_lifted rejected its arguments (rc={rc})")
    try:
        return C.string_at(out, n.value)
    finally:
        L.vxo_free(out)


def lifted_lde(cols, blowup_bits: int = 2):
    cols = [np.ascontiguousarray(c, dtype=np.uint32) for c in cols]
    logs = np.array([int(len(c)).bit_length() - 1 for c in cols], np.uint32)
    arr = (U32P * len(cols))(*[_p(c) for c in cols])
    outs = (U32P * len(cols))()
    L = lib()
    if L.vxo_lifted_lde(arr, _p(logs), len(cols), blowup_bits, outs):
        raise ValueError("oracle lifted_lde rejected its arguments")
    res = []
    for c, lg in enumerate(logs):
        m = 1 << (int(lg) + blowup_bits)
        res.append(np.ctypeslib.as_array(outs[c], shape=(m,)).copy())
        L.vxo_free(outs[c])
    return res


# ---- proof of work ----
def pow_prefix(state_words, pow_bits: int) -> np.ndarray:
    st = np.array(state_words, np.uint32)
    out = np.zeros(8, np.uint32)
    lib().vxo_pow_prefix(_p(st), pow_bits, _p(out))
    return out


def verify_pow_nonce(prefix, pow_bits: int, nonce: int, m31: bool = False) -> bool:
    return bool(lib().vxo_verify_pow_nonce(_p(np.array(prefix, np.uint32)), pow_bits, nonce, int(m31)))


def grind_pow(prefix, pow_bits: int, m31: bool = False, max_batches: int = 1 << 12) -> int:
    n = C.c_uint64()
    if lib().vxo_grind_pow(_p(np.array(prefix, np.uint32)), pow_bits, int(m31), max_batches, C.byref(n)):
        raise ValueError("no nonce found")
    return int(n.value)


# ---- the reference's own CUDA kernels (oracle/_ref/libvxref.so) ----
_REF_PATH = os.path.join(_HERE, "_ref", "libvxref.so")
_ref = None


def ref_available() -> bool:
    return os.path.exists(_REF_PATH)


def ref_lib():
    """libvxref.so: the reference's hot-path .cu files compiled for sm_100a plus
    ref_driver.cu (built by oracle/build_ref.sh).  Needs a GPU to run."""
    global _ref
    if _ref is None:
        R = C.CDLL(_REF_PATH)
        R.vxref_prove.argtypes = [C.c_uint32] * 5 + [C.c_void_p, C.c_size_t, C.POINTER(C.c_size_t)]
        R.vxref_prove.restype = C.c_int
        R.vxref_ntt_time.argtypes = [C.c_uint32, C.c_uint32, C.POINTER(C.c_float), C.POINTER(C.c_float)]
        R.vxref_ntt_time.restype = C.c_int
        _ref = R
    return _ref


def ref_prove(a: int, b: int, log_n: int, blowup_bits: int = 2, n_queries: int = 80) -> bytes:
    """Proof produced by the reference's CUDA kernels (prove_lean_inner order)."""
    size = proof_size(log_n, blowup_bits, n_queries)
    buf = (C.c_uint8 * size)()
    n = C.c_size_t()
    rc = ref_lib().vxref_prove(a, b, log_n, blowup_bits, n_queries, C.addressof(buf), size, C.byref(n))
    if rc:
        raise RuntimeError(f"reference-kernel prover failed (rc={rc})")
    return bytes(buf[: n.value])


def ref_ntt_time(log_n: int, reps: int = 5):
    """(evaluate ms, interpolate ms) of the reference's circle NTT on this GPU."""
    e, i = C.c_float(), C.c_float()
    rc = ref_lib().vxref_ntt_time(log_n, reps, C.byref(e), C.byref(i))
    if rc:
        raise RuntimeError("reference NTT timing failed")
    return e.value, i.value
