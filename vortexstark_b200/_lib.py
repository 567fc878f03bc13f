"""ctypes binding of libvortex_b200.so (the C ABI declared in include/vortex_b200.h).

The library is built in-tree by ``vortexstark_b200/build.py``.  There is no
fallback: every entry point of this package calls into the CUDA library, and
loading fails loudly if it is missing.
"""
from __future__ import annotations

import ctypes as C
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB_PATH = os.path.join(HERE, "libvortex_b200.so")
HEADER = os.path.join(ROOT, "include", "vortex_b200.h")

VX_OK, VX_ERR_ARG, VX_ERR_CUDA, VX_ERR_OOM, VX_ERR_DEVICE = 0, 1, 2, 3, 4

u32 = C.c_uint32
u32p = C.c_void_p  # device or host pointers are passed as raw addresses
vp = C.c_void_p

_SIGS = {
    # NTT
    "cuda_circle_ntt_evaluate": [vp, vp, vp, vp, vp, u32, u32],
    "cuda_circle_ntt_interpolate": [vp, vp, vp, vp, vp, u32, u32],
    "cuda_circle_ntt_evaluate_batch": [vp, vp, vp, vp, vp, u32, u32, u32],
    "cuda_circle_ntt_interpolate_batch": [vp, vp, vp, vp, vp, u32, u32, u32],
    "cuda_circle_ntt_evaluate_batch_forge": [vp, vp, vp, vp, vp, u32, u32, u32],
    "cuda_circle_ntt_interpolate_batch_forge": [vp, vp, vp, vp, vp, u32, u32, u32],
    "cuda_circle_ntt_layer_forge": [vp, vp, u32, u32, C.c_int],
    "cuda_batch_inverse_m31_forge": [vp, vp, u32],
    "cuda_circle_ntt_layer": [vp, vp, u32, u32, C.c_int],
    "cuda_bit_reverse_m31": [vp, u32],
    "cuda_permute_hc_to_canonic_brt": [vp, vp, u32, u32],
    "cuda_permute_canonic_brt_to_hc_natural": [vp, vp, u32, u32],
    # twiddles
    "cuda_compute_coset_points": [u32, u32, u32, u32, vp, vp, u32],
    "cuda_squash_x": [vp, vp, u32],
    "cuda_extract_and_squash": [vp, vp, vp, u32],
    "cuda_batch_inverse_m31": [vp, vp, u32],
    "cuda_batch_inverse_m31_stream": [vp, vp, u32, vp],
    "cuda_compute_fold_twiddle_sources": [u32, u32, u32, u32, vp, u32, u32, C.c_int],
    "cuda_compute_fold_twiddle_sources_stream": [u32, u32, u32, u32, vp, u32, u32, C.c_int, vp],
    # glue
    "cuda_zero_pad": [vp, vp, u32, u32],
    "cuda_fibonacci_quotient": [vp, vp, vp, vp, vp, vp, u32],
    "cuda_fibonacci_quotient_chunk": [vp, vp, vp, vp, vp, vp, u32, u32, u32],
    "cuda_fibonacci_quotient_chunk_stream": [vp, vp, vp, vp, vp, vp, u32, u32, u32, vp],
    # Merkle
    "cuda_merkle_hash_leaves": [vp, vp, u32, u32],
    "cuda_merkle_hash_leaves_forge_single": [vp, vp, u32],
    "cuda_merkle_hash_leaves_forge_quad": [vp, vp, vp, vp, vp, u32],
    "cuda_merkle_hash_nodes": [vp, vp, u32],
    "cuda_merkle_reduce_to_root": [vp, vp, u32],
    "cuda_merkle_commit_small_soa4": [vp, vp, vp, vp, vp, u32],
    "cuda_merkle_hash_leaves_merge_soa4": [vp, vp, vp, vp, vp, u32],
    "cuda_merkle_tiled_soa4": [vp, vp, vp, vp, vp, u32],
    "cuda_merkle_tiled_soa4_stream": [vp, vp, vp, vp, vp, u32, vp],
    "cuda_merkle_tiled_generic": [vp, vp, u32, u32],
    "cuda_build_leaves_lifted": [vp, vp, u32, u32, vp, u32],
    # FRI
    "cuda_fold_line_soa": [vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, u32],
    "cuda_fold_circle_into_line_soa": [vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, u32],
    "cuda_fold_line_soa_forge": [vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, u32],
    "cuda_fold_circle_into_line_soa_forge": [vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, u32],
    "cuda_device_sync": [],
    # proof of work
    "cuda_grind_pow": [vp, vp, u32, C.c_uint64, u32],
    "cuda_grind_pow_m31_output": [vp, vp, u32, C.c_uint64, u32],
    "vx_grind_pow": ([vp, u32, C.c_int, u32, C.POINTER(C.c_uint64), vp], C.c_int),
    # stwo-format path
    "cuda_stwo_ntt_evaluate": [vp, vp, u32],
    "cuda_stwo_ntt_interpolate": [vp, vp, u32],
    "cuda_stwo_ntt_batch_evaluate": [vp, vp, u32, u32],
    "cuda_stwo_ntt_batch_interpolate": [vp, vp, u32, u32],
    "cuda_bit_reverse_qm31": [vp, vp, u32, u32],
    "cuda_accumulate_lift": [vp, vp, u32, u32],
    "cuda_pack_leaves": [vp, vp, u32],
    "cuda_bit_reverse_qm31_forge": [vp, vp, u32, u32],
    "cuda_gather_u32": [vp, vp, vp, u32],
    "cuda_gather_u256": [vp, vp, vp, u32],
    "cuda_gather_u32_forge": [vp, vp, vp, u32, u32],
    "cuda_gather_u256_forge": [vp, vp, vp, u32, u32],
    "cuda_barycentric_eval": [vp, vp, u32, vp, u32],
    "cuda_eval_at_point": [vp, vp, vp, u32, vp, vp],
    # vx_ API
    "vx_last_error": ([], C.c_char_p),
    "vx_version": ([], C.c_int),
    "vx_proof_size": ([u32, u32, u32], C.c_size_t),
    "vx_prover_create": ([u32, u32, u32, C.POINTER(vp)], C.c_int),
    "vx_prover_destroy": [vp],
    "vx_prover_slot_bytes": ([vp], C.c_size_t),
    "vx_prover_table_bytes": ([vp], C.c_size_t),
    "vx_prover_prove_async": ([vp, u32, u32, vp], C.c_int),
    "vx_prover_fetch_async": ([vp, vp, vp], C.c_int),
    "vx_prover_stage_async": ([vp, u32, u32, u32, vp], C.c_int),
    "vx_prover_launches": ([vp], C.c_uint32),
    "vx_probe_blake2s": ([u32, u32, u32, vp, vp], C.c_int),
    "vx_tree_plan": ([u32, C.POINTER(u32), C.POINTER(u32), C.POINTER(u32), C.POINTER(u32),
                      C.POINTER(C.c_uint64)], C.c_int),
    "vx_autotune": ([u32, C.c_char_p, C.c_size_t], C.c_int),
    "vx_merkle_workspace_words": ([u32], C.c_uint64),
    "vx_fri_chain_create": ([u32, C.POINTER(vp)], C.c_int),
    "vx_fri_chain_destroy": [vp],
    "vx_fri_chain_layers": ([vp], u32),
    "vx_fri_chain_commit_async": ([vp, vp, vp, vp], C.c_int),
    "vx_fri_chain_launches": ([vp], u32),
    "vx_fri_chain_fetch": ([vp, vp, vp, vp, vp], C.c_int),
    "vx_merkle_root_cols": ([vp, u32, u32, vp, C.c_uint64, vp, vp], C.c_int),
    "vx_tune_set": ([u32, u32, u32, u32], C.c_int),
    "vx_tune_get": ([u32, u32, C.POINTER(u32), C.POINTER(u32)], C.c_int),
    "vx_ntt_plan": ([u32, u32, u32, C.POINTER(u32), C.POINTER(u32), C.POINTER(u32), C.POINTER(u32)], C.c_int),
    "vx_prover_proof_device": ([vp, C.POINTER(vp), C.POINTER(C.c_size_t)], C.c_int),
    "vx_prover_check": ([vp], C.c_int),
    "vx_prove_fib": ([u32, u32, u32, u32, u32, vp, C.c_size_t, C.POINTER(C.c_size_t)], C.c_int),
    "vx_prove_fib_noalloc": ([u32, u32, u32, u32, u32, vp, C.c_size_t, C.POINTER(C.c_size_t)], C.c_int),
    "vx_prove_fib_batch": ([vp, vp, u32, u32, u32, u32, vp, C.c_size_t, C.POINTER(C.c_size_t)], C.c_int),
    "vx_server_create": ([C.c_size_t, u32, u32, u32, C.c_int, C.POINTER(vp)], C.c_int),
    "vx_server_submit": ([vp, C.c_uint64, u32, u32, u32], C.c_int),
    "vx_server_set_policy": ([vp, u32, u32, C.c_int, u32, C.c_int, C.c_int], C.c_int),
    "vx_server_set_queue_order": ([vp, C.c_int, u32], C.c_int),
    "vx_server_prewarm": ([vp, u32, u32], C.c_int),
    "vx_server_poll": ([vp, vp, u32, C.POINTER(u32), C.c_int], C.c_int),
    "vx_server_result": ([vp, C.c_uint64, vp, C.c_size_t, C.POINTER(C.c_size_t)], C.c_int),
    "vx_server_stats": ([vp, C.POINTER(u32), C.POINTER(u32), C.POINTER(u32), C.POINTER(C.c_size_t)], C.c_int),
    "vx_server_destroy": [vp],
    "vx_release_all": [],
    "vx_clear_error": [],
    "vx_stwo_twiddles": ([u32, C.c_int, vp, vp], C.c_int),
    "vx_stwo_fold_circle_twiddles": ([u32, vp, vp], C.c_int),
    "vx_lifted_size": ([u32, vp, u32, u32], C.c_size_t),
    "vx_lifted_create": ([u32, vp, u32, u32, C.POINTER(vp)], C.c_int),
    "vx_lifted_destroy": [vp],
    "vx_lifted_column": ([vp, u32, C.POINTER(vp)], C.c_int),
    "vx_lifted_upload_async": ([vp, vp, vp], C.c_int),
    "vx_lifted_stage_async": ([vp, u32, vp], C.c_int),
    "vx_lifted_commit_async": ([vp, vp], C.c_int),
    "vx_lifted_commit_graph": ([vp, vp], C.c_int),
    "vx_lifted_fetch_async": ([vp, vp, vp], C.c_int),
    "vx_lifted_check": ([vp], C.c_int),
    "vx_lifted_launches": ([vp], C.c_uint32),
    "vx_lifted_device_bytes": ([vp], C.c_size_t),
    "vx_commit_lifted": ([vp, vp, u32, u32, u32, vp, C.c_size_t, C.POINTER(C.c_size_t)], C.c_int),
    "vx_lifted_release_all": [],
}

_lib = None


class VortexError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"vortex_b200 error {code}: {msg}")
        self.code = code


def header_symbols() -> list[str]:
    """Every function declared in include/vortex_b200.h."""
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    names = re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", txt)
    decl = [n for n in names if n.startswith(("cuda_", "vx_")) and n not in ("vx_prover",)]
    out = []
    for n in decl:
        if n not in out:
            out.append(n)
    return out


def lib() -> C.CDLL:
    """Load libvortex_b200.so, raising if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing; build it with `python -m vortexstark_b200.build` "
                "(there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, sig in _SIGS.items():
            f = getattr(L, name)
            if isinstance(sig, tuple):
                f.argtypes, f.restype = sig
            else:
                f.argtypes, f.restype = sig, None
        _lib = L
    return _lib


def clear_error() -> None:
    lib().vx_clear_error()


def raise_if_error() -> None:
    """After a void (reference-style) launcher: raise what it recorded."""
    msg = (lib().vx_last_error() or b"").decode()
    if msg:
        lib().vx_clear_error()
        raise VortexError(VX_ERR_CUDA, msg)


def check(rc: int) -> None:
    if rc != VX_OK:
        raise VortexError(rc, (lib().vx_last_error() or b"").decode())


def last_error() -> str:
    return (lib().vx_last_error() or b"").decode()
