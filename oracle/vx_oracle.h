/*
 * vx_oracle.h — CPU restatement of the VortexSTARK Fibonacci commitment path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the oracle: the tests, the
 * smoke entry and the CPU-baseline leg of the benchmark load it to produce
 * expected outputs.  The product path (vortexstark_b200) never calls it.
 *
 * Every function restates the reference's arithmetic bit-exactly; the
 * reference file:line it follows is cited beside each declaration.
 * Pinning: Blake2s is checked against Python hashlib.blake2s, the group
 * facts against src/circle.rs:586-622, the last-layer polynomial KAT
 * against src/fri.rs:513-580, and the whole path against an independent
 * pure-Python restatement (oracle/pyoracle.py) and against the reference's
 * own CUDA kernels compiled from source (oracle/_ref, run on a B200).
 */
#ifndef VX_ORACLE_H
#define VX_ORACLE_H
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VXO_P 0x7FFFFFFFu

/* ---- field (src/field/m31.rs:24-35, qm31.rs:110-133) ---- */
uint32_t vxo_m31_mul(uint32_t a, uint32_t b);
uint32_t vxo_m31_inv(uint32_t a);
void vxo_qm31_mul(const uint32_t a[4], const uint32_t b[4], uint32_t out[4]);

/* ---- circle group (src/circle.rs:10-268) ---- */
typedef struct { uint32_t x, y; } vxo_point;
typedef struct { vxo_point initial, step; uint32_t log_size; } vxo_coset;
vxo_point vxo_point_mul(vxo_point a, vxo_point b);
vxo_point vxo_point_pow(vxo_point a, uint64_t k);
vxo_coset vxo_coset_subgroup(uint32_t log_size);   /* circle.rs:101-109 */
vxo_coset vxo_coset_half_coset(uint32_t log_size); /* circle.rs:113-122 */
vxo_coset vxo_coset_half_odds(uint32_t log_size);  /* circle.rs:132-143 */
vxo_point vxo_coset_at(const vxo_coset *c, uint64_t i); /* circle.rs:183-185 */

/* ---- twiddles (circle.rs:357-550, twiddles.cu:80-142, batch_inverse.cu) ----
 * line: m-1 words, layer l at offset offsets[l] with m>>(l+1) words;
 * circle: m/2 words.  inverse != 0 gives elementwise inverses (0 -> 0). */
void vxo_twiddles(const vxo_coset *c, int inverse, uint32_t *line, uint32_t *circle,
                  uint32_t *offsets);
void vxo_batch_inverse(const uint32_t *in, uint32_t *out, size_t n);

/* ---- circle NTT (circle_ntt.cu:74-117, 248-312) ---- */
void vxo_ntt_layer(uint32_t *d, const uint32_t *tw, uint32_t layer_idx, uint64_t n, int forward);
void vxo_ntt_evaluate(uint32_t *d, const uint32_t *line, const uint32_t *circle,
                      const uint32_t *offsets, uint32_t log_n);
void vxo_ntt_interpolate(uint32_t *d, const uint32_t *iline, const uint32_t *icircle,
                         const uint32_t *offsets, uint32_t log_n);
/* whole-coset helpers that build their own tables */
void vxo_evaluate_on(uint32_t *d, const vxo_coset *c);
void vxo_interpolate_on(uint32_t *d, const vxo_coset *c);

/* ---- bit reverse / permute (circle_ntt.cu:234-244, circle.rs:192-226) ---- */
void vxo_bit_reverse(uint32_t *d, uint32_t log_n);
void vxo_permute_hc_to_canonic_brt(const uint32_t *src, uint32_t *dst, uint32_t log_n);
void vxo_permute_canonic_brt_to_hc(const uint32_t *src, uint32_t *dst, uint32_t log_n);

/* ---- glue (constraint.cu:10-90) ---- */
void vxo_fibonacci_trace(uint32_t a, uint32_t b, uint32_t log_n, uint32_t *out); /* air.rs:136-189 */
void vxo_fibonacci_quotient(const uint32_t *eval, uint64_t n, const uint32_t alpha[4],
                            uint32_t *q0, uint32_t *q1, uint32_t *q2, uint32_t *q3);

/* ---- Blake2s (channel.rs:216-298, blake2s.cuh:70-136) ---- */
void vxo_blake2s(const uint8_t *in, size_t len, uint8_t out[32]);
void vxo_hash_leaf(const uint32_t *words, uint32_t n_words, uint32_t out[8]); /* merkle.rs:570-593 */
void vxo_hash_pair(const uint32_t l[8], const uint32_t r[8], uint32_t out[8]); /* merkle.rs:864-884 */
void vxo_blake2s_compress_words(uint32_t h[8], const uint32_t m[16], uint32_t t, uint32_t f);

/* ---- Merkle (merkle.rs:28-130, 455-497, 841-851) ----
 * Full tree as an array of levels: level 0 = leaves (n*8 words), top = root.
 * cols: n_cols pointers to n-word columns; leaf = hash of the first
 * min(n_cols,16) words of the row (blake2s.cu:25-53). */
typedef struct { uint32_t log_n; uint32_t **levels; } vxo_tree;
void vxo_tree_build(vxo_tree *t, const uint32_t *const *cols, uint32_t n_cols, uint32_t log_n);
void vxo_tree_free(vxo_tree *t);
void vxo_tree_root(const vxo_tree *t, uint32_t out[8]);
void vxo_tree_path(const vxo_tree *t, uint64_t idx, uint32_t *out /* log_n*8 */);
void vxo_merkle_root(const uint32_t *const *cols, uint32_t n_cols, uint32_t log_n, uint32_t out[8]);
int vxo_verify_path(const uint32_t root[8], const uint32_t leaf[8], uint64_t idx,
                    const uint32_t *path, uint32_t depth); /* merkle.rs:520-566 */
/* Lifted multi-size leaves (merkle_leaves_lifted.cu:25-98): columns sorted by
 * ascending log size; leaf idx reads row ((idx >> (S-L+1)) << 1) | (idx & 1). */
void vxo_lifted_leaves(const uint32_t *const *cols, const uint32_t *log_sizes, uint32_t n_cols,
                       uint32_t lifting_log, uint32_t *out /* 2^S * 8 */);

/* ---- FRI (fri.rs:73-224, 411-427; fri.cu:58-126) ---- */
void vxo_fold_twiddles(const vxo_coset *domain, int extract_y, uint32_t *out /* size/2 */);
void vxo_fold_line(const uint32_t *const in[4], const uint32_t *tw, const uint32_t alpha[4],
                   uint32_t *const out[4], uint64_t half_n);
void vxo_fold_circle_into_line(uint32_t *const dst[4], const uint32_t *const src[4],
                               const uint32_t *tw, const uint32_t alpha[4],
                               const uint32_t alpha_sq[4], uint64_t half_n);

/* FRI chain with per-layer commitments of a 2^log_size QM31 codeword (SoA4)
 * on half_coset(log_size): log_size - 1 layers down to 2 values; roots
 * (8 words per layer), the challenges (4 words per layer), the last layer
 * (2 QM31, 4 words each). */
void vxo_fri_chain(const uint32_t *const src[4], uint32_t log_size, const uint32_t state[8], uint32_t *roots,
                   uint32_t *alphas, uint32_t last[8]);

/* PolyOps::eval_at_point by folding (circle_ntt.cu:429-468) and the
 * barycentric evaluation's per-block partial sums (barycentric_eval.cu). */
void vxo_eval_at_point(const uint32_t *coeffs, const uint32_t *factors, uint32_t log_n, uint32_t out[4]);
void vxo_barycentric_partials(const uint32_t *evals, const uint32_t *weights, uint32_t n, uint32_t n_blocks,
                              uint32_t *out);

/* ---- channel (channel.rs:15-185) ---- */
typedef struct { uint8_t state[32]; uint32_t n_draws; } vxo_channel;
void vxo_channel_init(vxo_channel *ch);
void vxo_channel_mix_digest(vxo_channel *ch, const uint32_t d[8]);
void vxo_channel_mix_felts(vxo_channel *ch, const uint32_t *felts, size_t n_felts);
void vxo_channel_draw_felt(vxo_channel *ch, uint32_t out[4]);
uint64_t vxo_channel_draw_number(vxo_channel *ch, uint64_t bound);
void vxo_channel_draw_query_indices(vxo_channel *ch, uint32_t log_domain, uint32_t n, uint32_t *out);

/* ---- whole proof (prover.rs:264-619; stark_cli.rs:1051-1123) ----
 * Returns the proof in the reference's "KRAK" v1 byte layout.  The caller
 * frees *out with vxo_free.  Returns 0 on success. */
int vxo_prove(uint32_t a, uint32_t b, uint32_t log_n, uint32_t blowup_bits, uint32_t n_queries,
              uint8_t **out, size_t *out_len);
/* The same proof bytes as vxo_prove in bounded host memory: the quotient is
 * recomputed where it is read, trees keep levels from height 8 up and
 * re-hash a 256-leaf subtree per authentication path.  For the 2^30- and
 * 2^31-point proofs (log_n = 28 / blowup 2, log_n = 30 / blowup 1). */
int vxo_prove_lean(uint32_t a, uint32_t b, uint32_t log_n, uint32_t blowup_bits, uint32_t n_queries,
                   uint8_t **out, size_t *out_len);
/* Proof size in bytes for (log_n, blowup_bits, n_queries). */
size_t vxo_proof_size(uint32_t log_n, uint32_t blowup_bits, uint32_t n_queries);
/* verifier.rs:39-310 on the byte layout; returns 0 if accepted, else a
 * positive code; msg (if non-NULL) receives a short reason. */
int vxo_verify(const uint8_t *proof, size_t len, uint32_t blowup_bits, uint32_t n_queries,
               char *msg, size_t msg_len);
/* Commitment values of a proof, for diagnostics: trace root, quotient
 * root, fri roots (count = log_eval-3). */
int vxo_prove_roots(uint32_t a, uint32_t b, uint32_t log_n, uint32_t blowup_bits,
                    uint32_t *trace_root, uint32_t *quotient_root, uint32_t *fri_roots);
/* ---- stwo-format circle NTT (ntt.rs:300-379, circle_ntt_stwo.cu:15-404) ----
 * Twiddles of CanonicCoset(log_n).circle_domain() as StwoNttCache::new builds
 * them (ntt.rs:300-341): 2^(log_n-1) words, level j = x-coordinates of the
 * first half of half_odds(log_n-1) doubled j times in bit-reversed order,
 * then a 1.  inverse != 0: elementwise inverses.  log_n >= 2. */
void vxo_stwo_twiddles(uint32_t log_n, int inverse, uint32_t *out);
/* line layers k = log_n-2 .. 0 (table at 2^(log_n-1) - 2^(log_n-1-k)), then
 * the circle layer [y, -y, -x, x] from the pairs of level 0 */
void vxo_stwo_ntt_evaluate(uint32_t *d, const uint32_t *tw, uint32_t log_n);
/* circle layer, line layers 0 .. log_n-2, then x 2^((30 log_n) mod 31) */
void vxo_stwo_ntt_interpolate(uint32_t *d, const uint32_t *itw, uint32_t log_n);
void vxo_bit_reverse_qm31(const uint32_t *in, uint32_t *out, uint32_t log_n);          /* bit_reverse_wide.cu:21-52 */
void vxo_accumulate_lift(uint32_t *col, const uint32_t *curr, uint64_t col_n, uint32_t log_ratio); /* accumulate_lift.cu:16-31 */
void vxo_pack_leaves(const uint32_t *const in[4], uint32_t *const out[64], uint64_t n); /* pack_leaves.cu:22-38 */
/* circle-fold twiddles of CanonicCoset(log).circle_domain(), 2^(log-1)
 * words: 1 / y(domain.at(bit_reverse_index(i << 1, log))) (fri_ops.rs:44-66).
 * Line folds use vxo_fold_twiddles(half_odds(l), 0) (fri_ops.rs:68-92). */
void vxo_stwo_fold_circle_twiddles(uint32_t log, uint32_t *out);

/* ---- batched lifted commitment ("LIFT" v1, a synthetic transcript) ----
 * Columns sorted by ascending log size L_c (2 <= L_c, L_c + blowup <= 28,
 * 1..64 columns), values in stwo's bit-reversed circle-domain order.
 *  1. LDE_c = stwo evaluate at 2^(L_c+B) of the zero-padded stwo interpolation;
 *  2. one lifted Blake2s tree over all LDE_c (S = max L_c + B), root R0;
 *  3. channel: mix(R0), alpha = draw_felt;
 *  4. C[i] = sum_c alpha^c * LDE_c[lift_row(i)] (accumulate_lift.cu:26-31), QM31[2^S];
 *  5. SoA4 tree over C, mix(R1), alpha_0; circle fold with the stwo twiddles,
 *     then line folds down to 8 values, each layer committed and mixed, a
 *     fresh alpha before every fold (the Fibonacci FRI of prover.rs:860-926);
 *  6. mix_felts(last 8), draw_query_indices(S, n_queries) (channel.rs:102-116).
 * Words: "LIFT", 1, n_cols, B, S, log sizes; R0; R1; nfri, FRI roots; 8, last
 * layer; nq, queries; decommitments (n, values at q, values at q^1, paths of
 * q, paths of q^1) of the lifted tree (a row = n_cols words), of C and of
 * every FRI layer (at q >> (k+1)), as the KRAK layout orders them. */
size_t vxo_lifted_size(uint32_t n_cols, const uint32_t *log_sizes, uint32_t blowup, uint32_t n_queries);
int vxo_commit_lifted(const uint32_t *const *cols, const uint32_t *log_sizes, uint32_t n_cols, uint32_t blowup,
                      uint32_t n_queries, uint8_t **out, size_t *out_len);
/* The LDE columns of step 1 (malloc'd, free each with vxo_free). */
int vxo_lifted_lde(const uint32_t *const *cols, const uint32_t *log_sizes, uint32_t n_cols, uint32_t blowup,
                   uint32_t **lde_out);

/* ---- proof of work (channel.rs:140-168, grind.cu:26-90, grind_ops.rs) ----
 * prefix = Blake2s(0x12345678_le || 0^12 || state || pow_bits_le); a nonce is
 * accepted when Blake2s(prefix || nonce_le) has >= pow_bits trailing zeros in
 * its first 16 bytes as a LE u128 (m31 != 0: those 4 words reduced mod P
 * first, grind_m31_output.cu).  The search visits (hi << 32) | low, low <
 * 2^20, hi = 0 .. max_batches-1, and returns the smallest accepted nonce
 * (0 when pow_bits = 0); 1 if none. */
void vxo_pow_prefix(const uint32_t state[8], uint32_t pow_bits, uint32_t out[8]);
int vxo_verify_pow_nonce(const uint32_t prefix[8], uint32_t pow_bits, uint64_t nonce, int m31);
int vxo_grind_pow(const uint32_t prefix[8], uint32_t pow_bits, int m31, uint32_t max_batches, uint64_t *nonce);

void vxo_free(void *p);
void vxo_set_threads(int n);
int vxo_get_threads(void);

#ifdef __cplusplus
}
#endif
#endif
