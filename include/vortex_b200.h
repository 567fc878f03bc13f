/*
 * vortex_b200.h — C ABI of libvortex_b200.so, the B200 (sm_100a) commitment
 * path of the VortexSTARK Circle-STARK prover.
 *
 * Two groups of entry points:
 *
 *  1. Drop-in replacements for the launchers that the reference's Rust FFI
 *     layer binds (src/cuda/ffi.rs).  Same symbol names, argument order and
 *     meaning: device pointers for data, host pointers for the small
 *     parameter arrays (alpha[4], layer offsets), void return, legacy
 *     default stream unless a `_stream` variant says otherwise.  As in the
 *     reference, the NTT evaluate/interpolate launchers synchronise the
 *     device before returning; the others are asynchronous.  A launch
 *     failure is recorded and can be read with vx_last_error().
 *
 *  2. New entry points (prefix vx_) for the device-resident whole-proof
 *     path: explicit streams, int status codes (VX_OK on success).
 *
 * All field data are canonical M31 words (< 2^31 - 1).  QM31 columns are
 * SoA: four M31 columns.
 */
#ifndef VORTEX_B200_H
#define VORTEX_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes of the vx_ API ---- */
#define VX_OK 0
#define VX_ERR_ARG 1    /* invalid argument (size, range, null pointer)      */
#define VX_ERR_CUDA 2   /* a CUDA runtime call failed                        */
#define VX_ERR_OOM 3    /* device allocation failed                          */
#define VX_ERR_DEVICE 4 /* a kernel reported an error through its status word */

/* ======================================================================
 * 1. Reference-compatible launchers (src/cuda/ffi.rs)
 * ====================================================================== */

/* -- circle NTT, natural order (ffi.rs:260-311; circle_ntt.cu:248-404) -- */
/* replaces cuda_circle_ntt_evaluate, circle_ntt.cu:248-275 */
void cuda_circle_ntt_evaluate(uint32_t *d_data, const uint32_t *d_twiddles, const uint32_t *d_circle_twids,
                              const uint32_t *h_layer_offsets, const uint32_t *h_layer_sizes,
                              uint32_t n_line_layers, uint32_t n);
/* replaces cuda_circle_ntt_interpolate, circle_ntt.cu:277-312 */
void cuda_circle_ntt_interpolate(uint32_t *d_data, const uint32_t *d_itwiddles, const uint32_t *d_circle_itwids,
                                 const uint32_t *h_layer_offsets, const uint32_t *h_layer_sizes,
                                 uint32_t n_line_layers, uint32_t n);
/* replaces cuda_circle_ntt_evaluate_batch, circle_ntt.cu:314-357 (d_columns: device array) */
void cuda_circle_ntt_evaluate_batch(uint32_t **d_columns, const uint32_t *d_twiddles, const uint32_t *d_circle_twids,
                                    const uint32_t *h_layer_offsets, const uint32_t *h_layer_sizes,
                                    uint32_t n_line_layers, uint32_t n, uint32_t n_cols);
/* replaces cuda_circle_ntt_interpolate_batch, circle_ntt.cu:359-404 */
void cuda_circle_ntt_interpolate_batch(uint32_t **d_columns, const uint32_t *d_itwiddles,
                                       const uint32_t *d_circle_itwids, const uint32_t *h_layer_offsets,
                                       const uint32_t *h_layer_sizes, uint32_t n_line_layers, uint32_t n,
                                       uint32_t n_cols);
/* replaces cuda_circle_ntt_evaluate_batch_forge / _interpolate_batch_forge, circle_ntt_batch_forge.cu:26-185
 * (ntt.rs:191-281 with the default `forge-ntt-batch` feature): the same transforms with col_ptrs a HOST
 * array of device column pointers; synchronous */
void cuda_circle_ntt_evaluate_batch_forge(uint32_t *const *col_ptrs, const uint32_t *d_twiddles,
                                          const uint32_t *d_circle_twids, const uint32_t *h_layer_offsets,
                                          const uint32_t *h_layer_sizes, uint32_t n_line_layers, uint32_t n,
                                          uint32_t n_cols);
void cuda_circle_ntt_interpolate_batch_forge(uint32_t *const *col_ptrs, const uint32_t *d_itwiddles,
                                             const uint32_t *d_circle_itwids, const uint32_t *h_layer_offsets,
                                             const uint32_t *h_layer_sizes, uint32_t n_line_layers, uint32_t n,
                                             uint32_t n_cols);
/* replaces cuda_circle_ntt_layer_forge (ffi.rs:395-398): the layer of cuda_circle_ntt_layer */
void cuda_circle_ntt_layer_forge(uint32_t *d_data, const uint32_t *d_twiddles, uint32_t layer_idx, uint32_t n,
                                 int forward);
/* replaces cuda_batch_inverse_m31_forge, batch_inverse_forge.cu:1-20: the chunk-of-64 batch inverse */
void cuda_batch_inverse_m31_forge(const uint32_t *input, uint32_t *output, uint32_t n);
/* replaces cuda_circle_ntt_layer, circle_ntt.cu:408-420 */
void cuda_circle_ntt_layer(uint32_t *d_data, const uint32_t *d_twiddles, uint32_t layer_idx, uint32_t n, int forward);
/* replaces cuda_bit_reverse_m31, circle_ntt.cu:422-427 */
void cuda_bit_reverse_m31(uint32_t *data, uint32_t log_n);
/* replaces cuda_permute_hc_to_canonic_brt, permute.cu:30-44 (ffi.rs:317-322) */
void cuda_permute_hc_to_canonic_brt(const uint32_t *src, uint32_t *dst, uint32_t n, uint32_t log_n);
/* replaces cuda_permute_canonic_brt_to_hc_natural, permute.cu:46-58 (ffi.rs:328-333) */
void cuda_permute_canonic_brt_to_hc_natural(const uint32_t *src, uint32_t *dst, uint32_t n, uint32_t log_n);

/* -- twiddles (ffi.rs:431-469; twiddles.cu:147-213; batch_inverse.cu:43-57) -- */
/* replaces cuda_compute_coset_points, twiddles.cu:177-190 */
void cuda_compute_coset_points(uint32_t initial_x, uint32_t initial_y, uint32_t step_x, uint32_t step_y,
                               uint32_t *output_x, uint32_t *output_y, uint32_t n);
/* replaces cuda_squash_x, twiddles.cu:192-198 */
void cuda_squash_x(const uint32_t *input, uint32_t *output, uint32_t out_n);
/* replaces cuda_extract_and_squash, twiddles.cu:200-210 */
void cuda_extract_and_squash(const uint32_t *input, uint32_t *twiddle_out, uint32_t *squash_out, uint32_t half_n);
/* replaces cuda_batch_inverse_m31, batch_inverse.cu:45-50 */
void cuda_batch_inverse_m31(const uint32_t *input, uint32_t *output, uint32_t n);
/* replaces cuda_batch_inverse_m31_stream, batch_inverse.cu:52-57 */
void cuda_batch_inverse_m31_stream(const uint32_t *input, uint32_t *output, uint32_t n, void *stream);
/* replaces cuda_compute_fold_twiddle_sources, twiddles.cu:147-160 */
void cuda_compute_fold_twiddle_sources(uint32_t initial_x, uint32_t initial_y, uint32_t step_x, uint32_t step_y,
                                       uint32_t *output, uint32_t n, uint32_t log_n, int extract_y);
/* replaces cuda_compute_fold_twiddle_sources_stream, twiddles.cu:162-175 */
void cuda_compute_fold_twiddle_sources_stream(uint32_t initial_x, uint32_t initial_y, uint32_t step_x,
                                              uint32_t step_y, uint32_t *output, uint32_t n, uint32_t log_n,
                                              int extract_y, void *stream);

/* -- glue (ffi.rs:471-503; constraint.cu:94-153) -- */
/* replaces cuda_zero_pad, constraint.cu:108-117 */
void cuda_zero_pad(const uint32_t *src, uint32_t *dst, uint32_t src_n, uint32_t dst_n);
/* replaces cuda_fibonacci_quotient, constraint.cu:94-106 (alpha: host [4]) */
void cuda_fibonacci_quotient(const uint32_t *trace, uint32_t *out0, uint32_t *out1, uint32_t *out2, uint32_t *out3,
                             const uint32_t *alpha, uint32_t n);
/* replaces cuda_fibonacci_quotient_chunk, constraint.cu:121-136 */
void cuda_fibonacci_quotient_chunk(const uint32_t *trace, uint32_t *out0, uint32_t *out1, uint32_t *out2,
                                   uint32_t *out3, const uint32_t *alpha, uint32_t offset, uint32_t chunk_n,
                                   uint32_t global_n);
/* replaces cuda_fibonacci_quotient_chunk_stream, constraint.cu:139-153 */
void cuda_fibonacci_quotient_chunk_stream(const uint32_t *trace, uint32_t *out0, uint32_t *out1, uint32_t *out2,
                                          uint32_t *out3, const uint32_t *alpha, uint32_t offset, uint32_t chunk_n,
                                          uint32_t global_n, void *stream);

/* -- Blake2s Merkle (ffi.rs:776-866, 937-944; blake2s.cu:537-646) -- */
/* replaces cuda_merkle_hash_leaves, blake2s.cu:539-548 (columns: device array) */
void cuda_merkle_hash_leaves(const uint32_t *const *columns, uint32_t *hashes, uint32_t n_cols, uint32_t n_leaves);
/* replaces cuda_merkle_hash_leaves_forge_single, merkle_hash_leaves_forge.cu:20-33 */
void cuda_merkle_hash_leaves_forge_single(const uint32_t *column, uint32_t *hashes, uint32_t n_leaves);
/* replaces cuda_merkle_hash_leaves_forge_quad, merkle_hash_leaves_forge.cu:35-51 */
void cuda_merkle_hash_leaves_forge_quad(const uint32_t *c0, const uint32_t *c1, const uint32_t *c2,
                                        const uint32_t *c3, uint32_t *hashes, uint32_t n_leaves);
/* replaces cuda_merkle_hash_nodes, blake2s.cu:550-559 */
void cuda_merkle_hash_nodes(const uint32_t *children, uint32_t *parents, uint32_t n_parents);
/* replaces cuda_merkle_reduce_to_root, blake2s.cu:562-569 (n_nodes <= 1024, power of two) */
void cuda_merkle_reduce_to_root(const uint32_t *nodes, uint32_t *root_out, uint32_t n_nodes);
/* replaces cuda_merkle_commit_small_soa4, blake2s.cu:573-584 (n_leaves <= 2048) */
void cuda_merkle_commit_small_soa4(const uint32_t *col0, const uint32_t *col1, const uint32_t *col2,
                                   const uint32_t *col3, uint32_t *root_out, uint32_t n_leaves);
/* replaces cuda_merkle_hash_leaves_merge_soa4, blake2s.cu:588-600 */
void cuda_merkle_hash_leaves_merge_soa4(const uint32_t *col0, const uint32_t *col1, const uint32_t *col2,
                                        const uint32_t *col3, uint32_t *parents, uint32_t n_leaves);
/* replaces cuda_merkle_tiled_soa4, blake2s.cu:604-615 (one root per 1024 leaves) */
void cuda_merkle_tiled_soa4(const uint32_t *col0, const uint32_t *col1, const uint32_t *col2, const uint32_t *col3,
                            uint32_t *subtree_roots, uint32_t n_leaves);
/* replaces cuda_merkle_tiled_soa4_stream, blake2s.cu:618-630 */
void cuda_merkle_tiled_soa4_stream(const uint32_t *col0, const uint32_t *col1, const uint32_t *col2,
                                   const uint32_t *col3, uint32_t *subtree_roots, uint32_t n_leaves, void *stream);
/* replaces cuda_merkle_tiled_generic, blake2s.cu:634-644 (columns: device array) */
void cuda_merkle_tiled_generic(const uint32_t *const *columns, uint32_t *subtree_roots, uint32_t n_cols,
                               uint32_t n_leaves);
/* replaces cuda_build_leaves_lifted, merkle_leaves_lifted.cu:104-120.
 * schedule: device array of {uint32 col_indices[16]; uint32 n_cols; uint32 log_size} */
void cuda_build_leaves_lifted(const uint32_t *const *col_ptrs, const void *schedule, uint32_t n_chunks,
                              uint32_t lifting_log_size, uint32_t *output_hashes, uint32_t n_leaves);

/* -- FRI folds (ffi.rs:345-425; fri.cu:128-163) -- */
/* replaces cuda_fold_line_soa, fri.cu:130-145 (alpha: host [4]) */
void cuda_fold_line_soa(const uint32_t *in0, const uint32_t *in1, const uint32_t *in2, const uint32_t *in3,
                        const uint32_t *twiddles, uint32_t *out0, uint32_t *out1, uint32_t *out2, uint32_t *out3,
                        const uint32_t *alpha, uint32_t half_n);
/* replaces cuda_fold_circle_into_line_soa, fri.cu:147-161 (alpha, alpha_sq: host [4]) */
void cuda_fold_circle_into_line_soa(uint32_t *dst0, uint32_t *dst1, uint32_t *dst2, uint32_t *dst3,
                                    const uint32_t *src0, const uint32_t *src1, const uint32_t *src2,
                                    const uint32_t *src3, const uint32_t *twiddles, const uint32_t *alpha,
                                    const uint32_t *alpha_sq, uint32_t half_n);
/* replaces cuda_fold_line_soa_forge, fri_fold_line_forge.cu (same semantics as cuda_fold_line_soa) */
void cuda_fold_line_soa_forge(const uint32_t *in0, const uint32_t *in1, const uint32_t *in2, const uint32_t *in3,
                              const uint32_t *twiddles, uint32_t *out0, uint32_t *out1, uint32_t *out2,
                              uint32_t *out3, const uint32_t *alpha, uint32_t half_n);
/* replaces cuda_fold_circle_into_line_soa_forge, fri_fold_circle_forge.cu */
void cuda_fold_circle_into_line_soa_forge(uint32_t *dst0, uint32_t *dst1, uint32_t *dst2, uint32_t *dst3,
                                          const uint32_t *src0, const uint32_t *src1, const uint32_t *src2,
                                          const uint32_t *src3, const uint32_t *twiddles, const uint32_t *alpha,
                                          const uint32_t *alpha_sq, uint32_t half_n);

/* replaces cuda_device_sync, fields.cu:44 */
void cuda_device_sync(void);

/* -- proof-of-work grinding (ffi.rs:761-772, 1195-1204) -- */
/* replaces cuda_grind_pow, grind.cu:92-118: nonces batch_offset + i for
 * i < n_threads; *result (device, set to UINT64_MAX by the caller) receives the
 * smallest nonce whose Blake2s(prefixed_digest || nonce_le) has >= pow_bits
 * trailing zeros in its first 16 bytes (LE u128).  prefixed_digest: 8 device
 * words.  Asynchronous on the legacy stream, as the reference's. */
void cuda_grind_pow(const uint32_t *prefixed_digest, uint64_t *result, uint32_t pow_bits, uint64_t batch_offset,
                    uint32_t n_threads);
/* replaces cuda_grind_pow_m31_output, grind_m31_output.cu: the same with the
 * four output words reduced mod P before the trailing-zero count */
void cuda_grind_pow_m31_output(const uint32_t *prefixed_digest, uint64_t *result, uint32_t pow_bits,
                               uint64_t batch_offset, uint32_t n_threads);

/* -- stwo-format path (crates/cuda-backend; ffi.rs:1182-1194) -- */
/* replaces cuda_stwo_ntt_evaluate, circle_ntt_stwo.cu:268-330: bit-reversed
 * circle FFT of n = 2^k (k >= 2) words in place with the stwo twiddle table
 * (2^(k-1) words, StwoNttCache / CpuBackend::precompute_twiddles layout);
 * synchronises the device before returning.  n = 2 (which the reference
 * serves by reading past its 1-word table) is rejected. */
void cuda_stwo_ntt_evaluate(uint32_t *data, const uint32_t *twiddles, uint32_t n);
/* replaces cuda_stwo_ntt_interpolate, circle_ntt_stwo.cu:333-402 (inverse
 * table; scales by 2^((30 k) mod 31) = 1/n) */
void cuda_stwo_ntt_interpolate(uint32_t *data, const uint32_t *itwiddles, uint32_t n);
/* replaces cuda_stwo_ntt_batch_evaluate, circle_ntt_stwo_batch.cu:239-306:
 * n_cols columns of n words; col_ptrs is a HOST array of device pointers */
void cuda_stwo_ntt_batch_evaluate(uint32_t *const *col_ptrs, const uint32_t *twiddles, uint32_t n,
                                  uint32_t n_cols);
/* replaces cuda_stwo_ntt_batch_interpolate, circle_ntt_stwo_batch.cu:308-374 */
void cuda_stwo_ntt_batch_interpolate(uint32_t *const *col_ptrs, const uint32_t *itwiddles, uint32_t n,
                                     uint32_t n_cols);
/* replaces cuda_bit_reverse_qm31, bit_reverse_wide.cu:41-50: out[brev(i)] =
 * in[i] for n = 2^log_n QM31 elements of 4 words, out of place (n must be
 * 2^log_n; the reference writes out of bounds otherwise) */
void cuda_bit_reverse_qm31(const uint32_t *in, uint32_t *out, uint32_t n, uint32_t log_n);
/* replaces cuda_accumulate_lift, accumulate_lift.cu:35-44: col[i] +=
 * curr[((i >> (log_ratio + 1)) << 1) | (i & 1)] for i < col_n */
void cuda_accumulate_lift(uint32_t *col, const uint32_t *curr, uint32_t col_n, uint32_t log_ratio);
/* replaces cuda_bit_reverse_qm31_forge (ffi.rs:1004-1019): the same as
 * cuda_bit_reverse_qm31 */
void cuda_bit_reverse_qm31_forge(const uint32_t *in, uint32_t *out, uint32_t n, uint32_t log_n);
/* replaces cuda_gather_u32, gather.cu:44-53: dst[i] = src[idx[i]], i < n
 * (ColumnOps decommitment, column.rs) */
void cuda_gather_u32(const uint32_t *src, const uint32_t *idx, uint32_t *dst, uint32_t n);
/* replaces cuda_gather_u256, gather.cu:55-64: dst[8i .. 8i+8) = src[8 idx[i] .. +8) */
void cuda_gather_u256(const uint32_t *src, const uint32_t *idx, uint32_t *dst, uint32_t n);
/* replace cuda_gather_u32_forge / cuda_gather_u256_forge (ffi.rs:986-1002,
 * gather_forge.cu): the same with src_len words of source; an element whose
 * source lies outside it is not written */
void cuda_gather_u32_forge(const uint32_t *src, const uint32_t *idx, uint32_t *dst, uint32_t n, uint32_t src_len);
void cuda_gather_u256_forge(const uint32_t *src, const uint32_t *idx, uint32_t *dst, uint32_t n, uint32_t src_len);
/* replaces cuda_barycentric_eval, barycentric_eval.cu:44-110: out[4b .. 4b+4)
 * = sum of evals[i] * weights[i] (M31 times QM31, weights AoS) over the i
 * of block b of a grid-stride loop of n_blocks x 256 threads (the caller
 * adds the n_blocks partial sums); synchronises the device. */
void cuda_barycentric_eval(const uint32_t *evals, const uint32_t *weights, uint32_t n, uint32_t *out,
                           uint32_t n_blocks);
/* replaces cuda_eval_at_point, circle_ntt.cu:429-468 (PolyOps::eval_at_point,
 * poly_ops.rs:382-443): folds n = 2^k M31 coefficients with the k QM31
 * folding factors (AoS, factor l for level l, level 0 splitting the top
 * index bit: v[t] + f_l v[t + n/2^(l+1)]) into one QM31, written to the
 * HOST array h_result[4].  d_scratch1 and d_scratch2 hold 2n words each
 * (the reference's n/2 QM31) and must not overlap.  For n >= 2^12 with a
 * 16-byte-aligned d_scratch1 and a non-null d_scratch2: 2^13 words of
 * d_scratch1 and at most 12 n / 2^11 + 8 words of d_scratch2 are used;
 * otherwise at most 4 n / 2^11 + 4 words of d_scratch1.  Synchronous.
 * n = 1 gives the coefficient; n not a power of two is rejected. */
void cuda_eval_at_point(const uint32_t *d_coeffs, const uint32_t *d_folding_factors, uint32_t *h_result, uint32_t n,
                        uint32_t *d_scratch1, uint32_t *d_scratch2);
/* replaces cuda_pack_leaves, pack_leaves.cu:44-52: output[c*16 + p][i] =
 * input[c][16 i + p]; both pointer arrays are DEVICE arrays (4 and 64
 * entries), N a multiple of 16 */
void cuda_pack_leaves(const uint32_t *const *input_col_ptrs, uint32_t *const *output_col_ptrs, uint32_t n);

/* ======================================================================
 * 2. Device-resident whole-proof path (new; no counterpart symbol in the
 *    reference — it replaces the body of prover.rs:264-619 / 627-1167)
 * ====================================================================== */

/* Message describing the last failure on the calling host thread (empty
 * if none since the last vx_clear_error). */
const char *vx_last_error(void);
/* Forget the calling thread's recorded failure (before a void launcher). */
void vx_clear_error(void);
/* Library version, major * 10000 + minor * 100 + patch. */
int vx_version(void);

/* Bytes of a proof in the reference's "KRAK" v1 layout
 * (stark_cli.rs:1092-1123) for (log_n, blowup_bits, n_queries). */
size_t vx_proof_size(uint32_t log_n, uint32_t blowup_bits, uint32_t n_queries);

/* One proof slot: device buffers for one in-flight proof of 2^log_n trace
 * rows with a 2^(log_n+blowup_bits) evaluation domain, plus shared,
 * device-resident twiddle tables for that size.  4 <= log_n,
 * log_n + blowup_bits <= 31, blowup_bits >= 1. */
typedef struct vx_prover vx_prover;
int vx_prover_create(uint32_t log_n, uint32_t blowup_bits, uint32_t n_queries, vx_prover **out);
void vx_prover_destroy(vx_prover *p);
/* Device bytes held by the slot (not counting the shared tables). */
size_t vx_prover_slot_bytes(const vx_prover *p);
/* Device bytes of the shared tables for this size. */
size_t vx_prover_table_bytes(const vx_prover *p);
/* Enqueue a whole proof of the Fibonacci AIR with public inputs (a, b) on
 * `stream` (a cudaStream_t; NULL = legacy default).  No host
 * synchronisation inside; the proof stays in the slot's device buffer. */
int vx_prover_prove_async(vx_prover *p, uint32_t a, uint32_t b, void *stream);
/* The proof's stages in order: 0 trace, 1 interpolate, 2 LDE evaluate,
 * 3 trace commitment, 4 quotient commitment, 5 circle fold + FRI layer 0,
 * 6 line folds + commitments, 7 last layer + query sampling,
 * 8 decommitment.  vx_prover_prove_async enqueues all of them; this enqueues
 * one (each stage reads what the earlier ones left in the slot), for
 * per-stage timing. */
#define VX_N_STAGES 9
int vx_prover_stage_async(vx_prover *p, uint32_t stage, uint32_t a, uint32_t b, void *stream);
/* Kernels enqueued by the last vx_prover_prove_async of this slot. */
uint32_t vx_prover_launches(const vx_prover *p);
/* Enqueue the copy of the slot's proof bytes to host memory `dst`
 * (vx_proof_size bytes; pinned memory makes it asynchronous). */
int vx_prover_fetch_async(vx_prover *p, void *dst, void *stream);
/* Device address and size of the slot's proof bytes. */
int vx_prover_proof_device(vx_prover *p, const void **dptr, size_t *bytes);
/* Check the slot's device status word after the stream has drained. */
int vx_prover_check(vx_prover *p);

/* Synchronous convenience: prove (a, b) at log_n into the host buffer
 * `out` (capacity `cap`), writing the proof length to *out_len.  Slots and
 * tables are cached per size and reused by later calls. */
int vx_prove_fib(uint32_t a, uint32_t b, uint32_t log_n, uint32_t blowup_bits, uint32_t n_queries, uint8_t *out,
                 size_t cap, size_t *out_len);

/* ---- proof-of-work search on the device (new) ----
 * Replaces the host loop of GrindOps::grind (crates/cuda-backend/src/
 * grind_ops.rs:20-134): nonces (hi << 32) | low, low < 2^20, hi = 0 ..
 * max_batches - 1 (stwo's search order), the smallest accepted one to
 * *nonce_out; launches of 2^26 candidates with one 8-byte read-back between
 * them.  prefixed_digest: 8 HOST words (Blake2s(0x12345678_le || 0^12 ||
 * channel state || pow_bits_le), reduced mod P by the caller for the M31
 * channel).  pow_bits = 0 gives nonce 0 without work.  VX_ERR_DEVICE if no
 * nonce exists in the range.  Synchronous. */
int vx_grind_pow(const uint32_t prefixed_digest[8], uint32_t pow_bits, int m31_output, uint32_t max_batches,
                 uint64_t *nonce_out, void *stream);

/* ---- stwo twiddles built on the device (new) ----
 * Replaces the CPU loops of StwoNttCache::new (ntt.rs:300-362) and the
 * host-built uploads of CudaBackend's twiddle cache (poly_ops.rs:102-127):
 * the 2^(log_n-1)-word table of CanonicCoset(log_n)'s circle domain
 * (inverse != 0: elementwise inverses), 2 <= log_n <= 29, into device
 * memory `out`, enqueued on `stream`. */
int vx_stwo_twiddles(uint32_t log_n, int inverse, uint32_t *out, void *stream);
/* Replaces get_or_compute_circle_fold_twiddles (fri_ops.rs:44-66): 2^(log-1)
 * words 1 / y(CanonicCoset(log).circle_domain().at(brev(2i, log))). */
int vx_stwo_fold_circle_twiddles(uint32_t log, uint32_t *out, void *stream);

/* ---- batched lifted commitment of uneven-size columns (new) ----
 * The workload of a multi-column stwo commitment on B200: columns sorted by
 * ascending log size L_c (1..64 columns, 2 <= L_c, L_c + blowup <= 28), each
 * given as 2^L_c M31 values in stwo's bit-reversed circle-domain order.
 *  1. LDE_c = stwo evaluate at 2^(L_c + blowup) of the zero-padded stwo
 *     interpolation (PolyOps::evaluate_polynomials, poly_ops.rs:676-770);
 *  2. one lifted Blake2s tree over all LDE rows, S = max L_c + blowup
 *     (MerkleOpsLifted::build_leaves, merkle_ops.rs:47-160); mix its root,
 *     draw alpha;
 *  3. C[i] = sum_c alpha^c * LDE_c[lift_row(i)] (accumulate_lift.cu:26-31),
 *     committed as a 4-word-leaf tree; mix, draw the first fold challenge;
 *  4. FRI: circle fold with the stwo twiddles, line folds down to 8 values,
 *     each layer committed and mixed, a fresh challenge per fold
 *     (fri_ops.rs:143-255, the Fibonacci FRI of prover.rs:860-926);
 *  5. mix_felts(last layer); draw_query_indices(S, n_queries)
 *     (channel.rs:102-116); open every tree at the queries.
 * The result is "LIFT" v1 words: "LIFT", 1, n_cols, blowup, S, log sizes;
 * the lifted root; C's root; nfri = S - 3, the FRI roots; 8, the last layer;
 * n_queries, the query indices; then for the lifted tree (a row = n_cols
 * words), for C and for every FRI layer k (at q >> (k + 1)): n, values at q,
 * values at q ^ 1, paths of q, paths of q ^ 1 (each path: depth, 8 words per
 * height), as the KRAK layout orders them.  The transcript is this
 * library's own (the reference has no such proof); tests check it against a
 * CPU restatement. */
typedef struct vx_lifted vx_lifted;
/* Bytes of the commitment for this shape, 0 if unsupported. */
size_t vx_lifted_size(uint32_t n_cols, const uint32_t *log_sizes, uint32_t blowup_bits, uint32_t n_queries);
/* Device buffers and tables for one shape. */
int vx_lifted_create(uint32_t n_cols, const uint32_t *log_sizes, uint32_t blowup_bits, uint32_t n_queries,
                     vx_lifted **out);
void vx_lifted_destroy(vx_lifted *h);
/* Device address of input column c (2^L_c words); write the column there,
 * or use vx_lifted_upload_async. */
int vx_lifted_column(vx_lifted *h, uint32_t c, uint32_t **dev_ptr);
/* Copy host columns (host_cols[c] of 2^L_c words) to the device on `stream`. */
int vx_lifted_upload_async(vx_lifted *h, const uint32_t *const *host_cols, void *stream);
/* Stages: 0 LDE, 1 lifted tree, 2 combination + its tree, 3 circle fold,
 * 4 line folds, 5 last layer + queries, 6 openings.  For per-stage timing. */
#define VX_LIFT_STAGES 7
int vx_lifted_stage_async(vx_lifted *h, uint32_t stage, void *stream);
/* All stages on the device-resident columns, no host synchronisation. */
int vx_lifted_commit_async(vx_lifted *h, void *stream);
/* The same schedule as one CUDA graph, captured on the first call. */
int vx_lifted_commit_graph(vx_lifted *h, void *stream);
/* Copy the commitment words to host memory `dst` (vx_lifted_size bytes). */
int vx_lifted_fetch_async(vx_lifted *h, void *dst, void *stream);
/* Device status word, after the stream has drained. */
int vx_lifted_check(vx_lifted *h);
/* Kernels of the last whole commitment; device bytes held. */
uint32_t vx_lifted_launches(const vx_lifted *h);
size_t vx_lifted_device_bytes(const vx_lifted *h);
/* Synchronous convenience: host columns in, commitment words out; one
 * instance per shape is cached (vx_lifted_release_all frees them). */
int vx_commit_lifted(const uint32_t *const *host_cols, const uint32_t *log_sizes, uint32_t n_cols,
                     uint32_t blowup_bits, uint32_t n_queries, uint8_t *out, size_t cap, size_t *out_len);
void vx_lifted_release_all(void);

/* ---- serving: continuous batching of mixed-size proof requests (new) ----
 * A dispatcher thread admits queued requests as proof slots of their size
 * free up or can be created inside the device-memory budget, up to
 * max_inflight proofs on the GPU at once, each on its own stream as one CUDA
 * graph (use_graphs != 0) or as plain launches.  A request's proof bytes do
 * not depend on what else is in flight. */
typedef struct vx_server vx_server;
typedef struct {
    uint64_t tag;         /* as submitted */
    int32_t status;       /* VX_OK or an error code */
    uint32_t log_n;
    uint64_t submit_ns;   /* host steady-clock times */
    uint64_t start_ns;
    uint64_t done_ns;
    uint64_t proof_bytes;
} vx_completion;
int vx_server_create(size_t budget_bytes, uint32_t max_inflight, uint32_t blowup_bits, uint32_t n_queries,
                     int use_graphs, vx_server **out);
/* Scheduling policy, before the first prewarm or submit (a slot's stream
 * priority is fixed when the slot is created; VX_ERR_ARG afterwards).
 * Proofs with at least 2^large_log_eval evaluation points are "large"; at
 * most max_large of them are in flight at once (per size when
 * large_per_size != 0).  priority: 0 puts small proofs on the
 * highest-priority streams, 1 gives every slot the same priority, 2 puts
 * large proofs on the highest-priority streams, 3 grades by size
 * (2^(large_log_eval-2) .. 2^(large_log_eval-1) points in between, smaller
 * ones highest, large ones lowest).  small_cap bounds the small proofs in
 * flight while a large one is (0: no bound).  split_large != 0 runs a large
 * proof as two graphs: its head (LDE, trace and quotient commitments, the
 * FRI layers whose trees are deeper than 16) counts against max_large, its
 * tail (the smaller FRI layers, queries, decommitment) runs on a
 * highest-priority stream after it and does not, so the next large proof's
 * head overlaps it.  Defaults: 24, 1, 0, 0, 0, 1.
 * Proof bytes never depend on the policy. */
int vx_server_set_policy(vx_server *s, uint32_t large_log_eval, uint32_t max_large, int priority,
                         uint32_t small_cap, int large_per_size, int split_large);
/* Order in which waiting large proofs take a free large place (any time;
 * ignored when large_per_size is set).  smallest_first == 0: oldest first
 * (the default).  smallest_first != 0: the smallest log_n first, oldest
 * within a size, except that once the oldest waiting large proof has waited
 * max_wait_us (0: never) it goes first.  Small proofs are not affected.
 * Proof bytes never depend on the order. */
int vx_server_set_queue_order(vx_server *s, int smallest_first, uint32_t max_wait_us);
/* Queue one request (non-blocking). */
int vx_server_submit(vx_server *s, uint64_t tag, uint32_t log_n, uint32_t a, uint32_t b);
/* Create up to `count` slots of this size ahead of time (counts against the budget). */
int vx_server_prewarm(vx_server *s, uint32_t log_n, uint32_t count);
/* Take up to `max` completions, waiting up to wait_ms for the first one. */
int vx_server_poll(vx_server *s, vx_completion *out, uint32_t max, uint32_t *n_out, int wait_ms);
/* Copy (out != NULL) and release the proof bytes of a completed request. */
int vx_server_result(vx_server *s, uint64_t tag, uint8_t *out, size_t cap, size_t *len);
int vx_server_stats(vx_server *s, uint32_t *n_slots, uint32_t *inflight, uint32_t *pending, size_t *bytes_used);
/* Waits for in-flight proofs, then frees every slot. */
void vx_server_destroy(vx_server *s);

/* Blake2s throughput probe: `blocks` x `threads` threads each run `iters`
 * chained compressions on registers only (no memory traffic) and write one
 * word to out[thread].  Gives the achievable compressions/s, the ALU
 * roofline of the Merkle kernels. */
int vx_probe_blake2s(uint32_t blocks, uint32_t threads, uint32_t iters, uint32_t *out, void *stream);

/* Host-only description of the Merkle build plan for a tree of 2^depth
 * leaves (1 <= depth <= 31); no device work.  heights[0..*n_levels) are the
 * stored levels' heights (heights[0] = 0 is the leaf level, the last is
 * depth); the reduce kernel starts from stored level *top (0: the leaves);
 * *n_counters group counters, *pool_words device words for the stored levels
 * and counters. */
int vx_tree_plan(uint32_t depth, uint32_t heights[12], uint32_t *n_levels, uint32_t *top, uint32_t *n_counters,
                 uint64_t *pool_words);

/* Root-only Merkle commitment through the fused tree kernels (leaf
 * subtrees, 16 -> 1 node kernels, one reduce launch) — replaces
 * MerkleTree::commit_root_only (merkle.rs:142-231) and commit_root_soa4
 * (merkle.rs:236-312), whose reference form is a launch per tree level.
 * Leaf i = Blake2s of the LE words col[0][i] .. col[n_cols-1][i]
 * (1 <= n_cols <= 16), node = Blake2s(left || right), 2^log_n_leaves leaves
 * (1..31).  host_col_ptrs: HOST array of device column pointers.
 * workspace: device memory of workspace_words words (at least
 * vx_merkle_workspace_words(log_n_leaves); it holds the stored levels and
 * is reused across calls).  root_out: 8 device words.  Enqueued on
 * `stream`, no host synchronisation. */
uint64_t vx_merkle_workspace_words(uint32_t log_n_leaves);
int vx_merkle_root_cols(const uint32_t *const *host_col_ptrs, uint32_t n_cols, uint32_t log_n_leaves,
                        uint32_t *workspace, uint64_t workspace_words, uint32_t *root_out, void *stream);

/* FRI chain of a QM31 codeword with a commitment per layer — the proof's
 * FRI (prover.rs:860-926; folds fri.rs:163-224) run down to 2 values, as
 * one call.  The codeword is 4 SoA device columns of 2^log_size words
 * (3 <= log_size <= 30), its evaluation on half_coset(log_size).  With the
 * transcript started from `state` (8 host words): alpha_0 = draw_felt;
 * layer 0 = circle fold of the codeword (into zero); for k >= 1 layer k =
 * line fold of layer k-1 with the half_odds twiddles and alpha_k; every
 * layer committed as a tree of 4-word leaves, its root mixed, then the
 * next challenge drawn.  log_size - 1 layers; the last holds 2 values.
 * Folds run inside the hashing kernels, transcript steps in the kernel
 * that finishes each tree; no host synchronisation until fetch. */
typedef struct vx_fri_chain vx_fri_chain;
int vx_fri_chain_create(uint32_t log_size, vx_fri_chain **out);
void vx_fri_chain_destroy(vx_fri_chain *h);
uint32_t vx_fri_chain_layers(const vx_fri_chain *h);
/* host_cols: HOST array of 4 device pointers (8-byte aligned). */
int vx_fri_chain_commit_async(vx_fri_chain *h, const uint32_t *const *host_cols, const uint32_t state[8],
                              void *stream);
/* Kernels enqueued by the last commit. */
uint32_t vx_fri_chain_launches(const vx_fri_chain *h);
/* Waits for `stream`, then: roots (8 words per layer), alphas (4 per layer),
 * last = the 2 values of the last layer, 4 words each.  VX_ERR_DEVICE if a
 * challenge draw gave up. */
int vx_fri_chain_fetch(vx_fri_chain *h, uint32_t *roots, uint32_t *alphas, uint32_t last[8], void *stream);

/* Autotuner — no counterpart in the reference, whose kernels have fixed
 * shapes (circle_ntt.cu: one launch per layer; blake2s.cu: one leaf per
 * thread).  On the current device, times every distinct NTT pass plan
 * on 4096-element tiles (bottom pass of 10..12 layers, upper passes of at
 * most 6..9; the larger tiles are set with vx_tune_set) of each
 * transform length 13..max_log (shorter ones are a single pass), and the
 * Merkle leaf kernel's subtree size (2^1..2^4 leaves per thread) of each tree
 * depth 17..max_log, separately for narrow leaves (M31 columns) and for wide
 * leaves (FRI folds, lifted rows; timed with fold leaves, depths up to 25),
 * on scratch buffers of that size
 * (about 16 * 2^max_log + 52 * 2^min(max_log, 25) bytes, freed before return),
 * and keeps the fastest for later launches on this device.  Every choice
 * computes identical values, so proofs do not change.  Plans are read when
 * a transform is launched and when a tree is carved (prover slot or lifted
 * context creation), so tune before creating those.  Writes a JSON report
 * ({"ntt":{"log":[bottom,upper,ms]},"leaf_k":{"depth":[k,ms]},
 * "fold_leaf_k":{"depth":[k,ms]}}) to `report`
 * (cap bytes, NUL-terminated, truncated).  12 <= max_log <= 28.  Not safe
 * to run while other host threads launch on the same device. */
int vx_autotune(uint32_t max_log, char *report, size_t cap);
/* Set one knob on the current device.  kind 0: NTT plan of transforms over
 * 2^`layers` elements (applied to the layers such a transform runs; an LDE
 * of 2^26 points from 2^24 coefficients runs 24 layers under the 2^26
 * plan), a = bottom pass maximum (9..14), b = upper pass maximum (3..12),
 * a = 0 restores the default (11, 8).  kind 1: leaf kernel subtree
 * log for narrow-leaf trees of depth `layers`, a in 1..4, 0 restores the
 * default; kind 2: the same for wide-leaf trees (FRI layers, lifted rows,
 * their combinations). */
int vx_tune_set(uint32_t kind, uint32_t layers, uint32_t a, uint32_t b);
/* Read the knob that launches on the current device use (b = 0 for kinds 1, 2). */
int vx_tune_get(uint32_t kind, uint32_t layers, uint32_t *a, uint32_t *b);
/* Host-only: the pass plan of a `total`-layer transform (4..31) for a bottom
 * pass of at most bottom_max (9..14) layers and upper passes of at most
 * upper_max (3..12); transforms of at most max(12, bottom_max) layers are one
 * pass.  Pass i applies layers [starts[i], starts[i] + layers[i]) on tiles of
 * 2^tile_cols_log[i] contiguous columns (0 for the bottom pass). */
int vx_ntt_plan(uint32_t total, uint32_t bottom_max, uint32_t upper_max, uint32_t starts[32], uint32_t layers[32],
                uint32_t tile_cols_log[32], uint32_t *n_passes);

/* Whole proof without any device allocation — no counterpart in the
 * reference.  For callers that cannot call cudaMalloc: hosts whose device
 * memory is owned by another allocator (a Rust arena, a framework's caching
 * pool) and sandboxes that forbid cudaMalloc after start-up.  Same result as
 * vx_prove_fib, with every byte of device scratch in one fixed 8 MiB static
 * device array of this library (held on every GPU that loads it until the
 * process exits), so the size is limited to log_n + blowup_bits <= 14 and
 * n_queries <= 80; larger sizes are rejected with VX_ERR_ARG.  The first call
 * on a device looks up the array's device address and uploads constant
 * tables.  Every call is synchronous: it copies with cudaMemcpy, launches on
 * the legacy default stream and returns when the proof is in `out`, so it
 * must not be called while any stream capture is active in the process.
 * All calls share the array and it keeps the last call's contents; calls
 * that overlapped on the GPU would race on it, so a process-wide lock
 * serialises them (each call blocks the others until its proof is back). */
int vx_prove_fib_noalloc(uint32_t a, uint32_t b, uint32_t log_n, uint32_t blowup_bits, uint32_t n_queries,
                         uint8_t *out, size_t cap, size_t *out_len);

/* Many proofs of one size — replaces ProverPipeline::prove_batch
 * (prover.rs:2278-2311), which proves its inputs one after another with a
 * shared cache.  Proves (a[i], b[i]) for i < count into out + i *
 * *proof_size (cap >= count * vx_proof_size bytes), each proof
 * byte-identical to vx_prove_fib's.  Up to four cached slots on their own
 * streams keep that many proofs in flight, so one proof's latency-bound FRI
 * tail overlaps the next ones' hashing; a slot after the first is added only
 * while it fits in half of the free device memory.  Returns when all proofs
 * are in `out`. */
int vx_prove_fib_batch(const uint32_t *a, const uint32_t *b, uint32_t count, uint32_t log_n, uint32_t blowup_bits,
                       uint32_t n_queries, uint8_t *out, size_t cap, size_t *proof_size);

/* Free the slots cached by vx_prove_fib and vx_prove_fib_batch on every
 * device (a size's shared tables are freed with the last slot, of any
 * owner, that uses them) and the column-pointer arrays the forge batch
 * launchers keep per device.  After a cudaDeviceReset call this before the
 * next call into the library. */
void vx_release_all(void);

#ifdef __cplusplus
}
#endif
#endif /* VORTEX_B200_H */
