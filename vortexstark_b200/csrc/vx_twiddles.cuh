// Twiddle tables for the circle NTT and the FRI folds.
//
// Every point of every coset used on this path is a power of the circle
// generator G = (2, 1268011823) of order 2^31, so each twiddle is a
// coordinate of G^E for an exponent E computed from its index:
//   coset (e0, k): p_j = G^(e0 + j * 2^(31-k))          (circle.rs:183-185)
//   line layer l:  T_l[h] = x(G^(2^l (e0 + 2^(l+1) h 2^(31-k))))
//                  (extract-and-squash of circle.rs:493-518 in closed form)
//   circle:        C[h]   = y(G^(e0 + h 2^(31-k)))
//   fold:          tw[i]  = 1 / coord(G^(e0 + brev(2i, k) 2^(31-k)))
//                  (twiddles.cu:23-52 then batch_inverse.cu)
// G^E is one circle multiply of two table entries: G^(E & 0xFFFF) and
// G^((E >> 16) << 16), built once per device.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "vx_field.cuh"

namespace vx {

struct GenTables {
    const cpoint *lo;  // G^i, i < 2^16
    const cpoint *hi;  // G^(i << 16), i < 2^15
};

// Lazily builds and uploads the generator tables for the current device.
cudaError_t gen_tables_get(GenTables *out);

__device__ __forceinline__ cpoint gpow(const GenTables &t, uint32_t e) {
    e &= 0x7FFFFFFFu;
    return pmul(t.hi[e >> 16], t.lo[e & 0xFFFFu]);
}

// A coset as exponents: initial = G^e0, step = G^(2^(31-k)).
struct ecoset { uint32_t e0, k; };
inline ecoset ecoset_half_coset(uint32_t k) { return {k <= 30 ? (1u << (30 - k)) : 0u, k}; }
inline ecoset ecoset_subgroup(uint32_t k) { return {0u, k}; }
__host__ __device__ inline uint32_t ecoset_half_odds_e0(uint32_t k) { return k >= 29 ? 1u : (1u << (29 - k)); }
inline ecoset ecoset_half_odds(uint32_t k) { return {ecoset_half_odds_e0(k), k}; }
inline ecoset ecoset_eval_domain(uint32_t k) { return k <= 30 ? ecoset_half_coset(k) : ecoset_subgroup(k); }

// NTT tables in the reference layout (line: 2^k - 1 words, circle: 2^(k-1)).
// inverse: elementwise inverses with the reference's chunked batch inverse.
cudaError_t build_ntt_tables(ecoset c, bool inverse, uint32_t *line, uint32_t *circle, cudaStream_t stream);

// FRI fold twiddles of a domain of 2^k points: 2^(k-1) words.
cudaError_t build_fold_twiddles(ecoset c, bool extract_y, uint32_t *out, cudaStream_t stream);

// Same as build_ntt_tables / build_fold_twiddles with caller-provided
// generator tables (no lazy allocation inside).
cudaError_t build_ntt_tables_with(const GenTables &g, ecoset c, bool inverse, uint32_t *line, uint32_t *circle,
                                  cudaStream_t stream);
cudaError_t build_fold_twiddles_with(const GenTables &g, ecoset c, bool extract_y, uint32_t *out,
                                     cudaStream_t stream);
// Host computation of the generator tables: lo[i] = G^i (i < 2^16) followed
// by hi[i] = G^(i << 16) (i < 2^15), as (x, y) word pairs: 196608 words.
constexpr uint32_t kGenTableWords = 2u * ((1u << 16) + (1u << 15));
void gen_tables_host(uint32_t *words);

// stwo NTT table of CanonicCoset(log_n)'s circle domain (ntt.rs:300-341):
// 2^(log_n-1) words; level j (j <= log_n-2) at 2^(log_n-1) - 2^(log_n-1-j)
// holds x(half_odds(L).at(brev(p, L-1))) for p < 2^(L-1), L = log_n-1-j
// (half_odds(L) doubled is half_odds(L-1)); the last word is 1.  inverse:
// elementwise inverses.  log_n in [2, 29].
cudaError_t build_stwo_table_with(const GenTables &g, uint32_t log_n, bool inverse, uint32_t *out,
                                  cudaStream_t stream);
// stwo circle-fold twiddles of CanonicCoset(log)'s circle domain
// (fri_ops.rs:44-66): out[i] = 1 / y(half_odds(log-1).at(brev(2i, log))),
// 2^(log-1) words (brev(2i, log) < 2^(log-1), so the conjugate half of the
// domain is never reached).
cudaError_t build_stwo_fold_circle_with(const GenTables &g, uint32_t log, uint32_t *out, cudaStream_t stream);

// Reference batch inverse: aligned chunks of 64, 0 -> 0, and a zero in a
// chunk's first slot zeroes that whole chunk (batch_inverse.cu:8-41).
cudaError_t batch_inverse(const uint32_t *in, uint32_t *out, uint64_t n, cudaStream_t stream);

}  // namespace vx
