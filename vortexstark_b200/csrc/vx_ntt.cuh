// Circle NTT in the reference's natural-order layout, as multi-layer passes.
//
// Layer L (stride 2^L) pairs i0 and i0 + 2^L and uses the twiddle indexed by
// h = i0 >> (L + 1): line table l = L - 1 for L >= 1, the circle table for
// L = 0 (circle_ntt.cu:89-117).  Forward runs L = k-1 .. 0 with
// v0' = v0 + v1 t, v1' = v0 - v1 t; inverse runs L = 0 .. k-1 with
// v0' = v0 + v1, v1' = (v0 - v1) t, then scales by 2^-k (circle_ntt.cu:248-312).
//
// A pass applies the layers of one bit range [s, s + r) to tiles of
// 2^r rows x 2^w columns held in shared memory; every element of a tile has
// the same bits outside [s, s + r) except the w low column bits, so each
// global row segment is 2^w contiguous words (w = min(s, 3) keeps segments at
// one 32-byte sector).  A transform of 2^k points runs in ceil(k / 11) passes.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace vx {

struct NttTables {
    const uint32_t *line;     // flat line twiddles, layer l at line + off[l]
    const uint32_t *circle;   // circle twiddles (n/2), or the stwo pair table
    uint32_t off[32];
    uint32_t circle_mode;     // 0: circle[h]; 1: stwo, [y, -y, -x, x][h & 3] of the
                              // pair (circle[2 (h >> 2)], circle[2 (h >> 2) + 1])
};

// Enqueue a full forward (evaluate) or inverse (interpolate, with 1/n scale)
// transform of `n_cols` columns of 2^log_n points.  Columns are either
// `dev_cols[c]` (device array of pointers) or `data + c * col_stride`.
// For the LDE, `src` (coefficients, 2^src_log words) replaces the first pass's
// input: element g reads src[g & (2^src_log - 1)], and the top
// (log_n - src_log) layers, which only replicate zero-padded coefficients,
// are skipped.  An inverse transform may read `src` (src_log = log_n) to
// run out of place.  src == nullptr means in place.
cudaError_t ntt_transform(uint32_t *data, uint32_t *const *dev_cols, uint64_t col_stride, uint32_t n_cols,
                          uint32_t log_n, const NttTables &tw, bool forward, const uint32_t *src,
                          uint32_t src_log, cudaStream_t stream);

// ntt_transform with an explicit pass plan (ntt_plan's bottom_max / upper_max;
// 0 = the device's current choice).
cudaError_t ntt_transform_planned(uint32_t *data, uint32_t *const *dev_cols, uint64_t col_stride, uint32_t n_cols,
                                  uint32_t log_n, const NttTables &tw, bool forward, const uint32_t *src,
                                  uint32_t src_log, uint32_t bottom_max, uint32_t upper_max, cudaStream_t stream);

// Transforms of several column groups of different lengths, for the same
// direction: group g is n_cols columns of 2^log_n words at data + c *
// col_stride, with its own tables and optional source (as ntt_transform).
// Groups of 15..21 applied layers share one launch per pass (a 12-layer
// bottom pass and one upper pass); the others run as their own transforms.
// `launches` (if non-null) is increased by the kernels enqueued.
struct NttGroup {
    uint32_t *data;
    uint64_t col_stride;
    uint32_t n_cols, log_n;
    NttTables tw;
    const uint32_t *src;
    uint32_t src_log;
};
cudaError_t ntt_transform_groups(const NttGroup *groups, uint32_t n_groups, bool forward, cudaStream_t stream,
                                 uint32_t *launches);

// Kernel launches of a transform that applies `layers` layers to 2^log_n
// elements (log_n = 0: as many elements as layers).
uint32_t ntt_pass_count(uint32_t layers, uint32_t log_n = 0);

// Pass plan of a `total`-layer transform for a bottom pass of at most
// bottom_max (9..12) layers and upper passes of at most upper_max (3..9):
// pass i covers layers [ps[i], ps[i] + pr[i]) on tiles with 2^pw[i] columns.
// Transforms of at most 12 layers are one pass.
uint32_t ntt_plan(uint32_t total, uint32_t bottom_max, uint32_t upper_max, uint32_t ps[32], uint32_t pr[32],
                  uint32_t pw[32]);
// Per-device plan choice for transforms over 2^log_n elements (default 11 /
// 8), applied to the layers such a transform runs; every choice computes
// the same values.
void ntt_knobs_set(int dev, uint32_t log_n, uint32_t bottom_max, uint32_t upper_max);
void ntt_knobs_get(uint32_t log_n, uint32_t *bottom_max, uint32_t *upper_max);

// One butterfly layer over the whole array (reference cuda_circle_ntt_layer).
cudaError_t ntt_single_layer(uint32_t *data, const uint32_t *tw, uint32_t layer_idx, uint32_t log_n, bool forward,
                             cudaStream_t stream);
// The same layer over n_cols columns given as a device array of pointers.
cudaError_t ntt_single_layer_cols(uint32_t *const *dev_cols, uint32_t n_cols, const uint32_t *tw, uint32_t layer_idx,
                                  uint32_t log_n, bool forward, cudaStream_t stream);

// Reference table layout for a coset of 2^log_n points: line twiddles
// (2^log_n - 1 words) and circle twiddles (2^(log_n-1) words); offsets of
// line layer l are  sum_{j<l} 2^(log_n-1-j).
void ntt_table_offsets(uint32_t log_n, uint32_t off[32]);

// stwo layout (ntt.rs:300-341, circle_ntt_stwo.cu:268-404): one table of
// 2^(log_n-1) words, line layer l at 2^(log_n-1) - 2^(log_n-1-l), and the
// circle layer derived from layer 0's pairs.  Tables for ntt_transform.
NttTables stwo_tables(const uint32_t *tw, uint32_t log_n);

}  // namespace vx
