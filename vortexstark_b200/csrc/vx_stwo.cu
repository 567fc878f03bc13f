// stwo-format launchers (the crates/cuda-backend symbols of src/cuda/ffi.rs):
// the bit-reversed-order circle NTT of circle_ntt_stwo.cu and its batched
// form, the QM31 bit reverse of bit_reverse_wide.cu, lift-and-accumulate
// (accumulate_lift.cu) and the leaf packing of pack_leaves.cu.  Same
// signatures, arguments and synchronisation as the reference; the kernels
// are this library's own: the NTT runs on the register-radix passes of
// vx_ntt.cu with the stwo table layout, the permutations go through
// shared-memory tiles so both their reads and their writes are coalesced.
#include <mutex>

#include "vx_common.cuh"
#include "vx_field.cuh"
#include "vx_ntt.cuh"
#include "vx_twiddles.cuh"

namespace vx {
namespace {

inline uint32_t log2_of(uint64_t n) {
    uint32_t l = 0;
    while ((1ull << l) < n) l++;
    return l;
}

// ---- host pointer lists of the batched NTT, uploaded once per call into a
// per-device buffer that only grows (the reference mallocs one per call) ----
std::mutex g_ptr_mu;
uint32_t **g_ptr_buf[64] = {nullptr};
uint32_t g_ptr_cap[64] = {0};

cudaError_t upload_ptrs(uint32_t *const *host, uint32_t n, uint32_t ***dev_out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (g_ptr_cap[dev] < n) {
        if (g_ptr_buf[dev]) cudaFree(g_ptr_buf[dev]);
        g_ptr_buf[dev] = nullptr;
        g_ptr_cap[dev] = 0;
        uint32_t cap = n < 64u ? 64u : n;
        e = cudaMalloc(&g_ptr_buf[dev], cap * sizeof(uint32_t *));
        if (e != cudaSuccess) return e;
        g_ptr_cap[dev] = cap;
    }
    e = cudaMemcpy(g_ptr_buf[dev], host, n * sizeof(uint32_t *), cudaMemcpyHostToDevice);
    *dev_out = g_ptr_buf[dev];
    return e;
}

bool stwo_size_ok(uint32_t n, const char *who) {
    uint32_t l = log2_of(n);
    if (n < 4 || (1ull << l) != n || l > 30) {
        set_last_error(VX_ERR_ARG, "%s: n = %u must be a power of two >= 4", who, n);
        return false;
    }
    return true;
}

// ---- QM31 bit reverse (bit_reverse_wide.cu:21-36), out of place ----
// Tiled: index bits [lo: 5][mid: L-10][hi: 5] go to [brev hi][brev mid][brev lo];
// a block moves the 32 x 32 (hi, lo) tile of one mid value through shared
// memory, reading rows of 32 consecutive elements and writing rows of 32.
constexpr uint32_t kBrT = 5;                 // tile side 2^5
constexpr uint32_t kBrS = 1u << kBrT;
__global__ void __launch_bounds__(256) brev_qm31_tiled_kernel(const uint4 *__restrict__ in, uint4 *__restrict__ out,
                                                               uint32_t log_n) {
    __shared__ uint4 tile[kBrS][kBrS + 1];
    const uint32_t mid_bits = log_n - 2 * kBrT;
    const uint64_t mid = blockIdx.x;
    const uint64_t bmid = mid_bits ? brev_bits((uint32_t)mid, mid_bits) : 0u;
    const uint32_t tx = threadIdx.x & (kBrS - 1u), ty = threadIdx.x >> kBrT;  // 32 x 8
#pragma unroll
    for (uint32_t r = 0; r < kBrS; r += 8) {
        const uint32_t hi = ty + r, lo = tx;
        const uint64_t i = lo | (mid << kBrT) | ((uint64_t)hi << (log_n - kBrT));
        tile[hi][lo] = in[i];
    }
    __syncthreads();
#pragma unroll
    for (uint32_t r = 0; r < kBrS; r += 8) {
        const uint32_t row = ty + r, col = tx;  // row = brev(lo), col = brev(hi)
        const uint32_t lo = brev_bits(row, kBrT), hi = brev_bits(col, kBrT);
        const uint64_t j = col | (bmid << kBrT) | ((uint64_t)row << (log_n - kBrT));
        out[j] = tile[hi][lo];
    }
}

__global__ void brev_qm31_kernel(const uint32_t *__restrict__ in, uint32_t *__restrict__ out, uint64_t n,
                                 uint32_t log_n) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint64_t j = brev_bits((uint32_t)i, log_n);
#pragma unroll
    for (int c = 0; c < 4; c++) out[4 * j + c] = in[4 * i + c];
}

// ---- lift_and_accumulate pass (accumulate_lift.cu:16-31): col[i] +=
// curr[((i >> (r + 1)) << 1) | (i & 1)], four elements per thread ----
__global__ void accumulate_lift4_kernel(uint4 *__restrict__ col, const uint32_t *__restrict__ curr, uint64_t n4,
                                        uint32_t r) {
    uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n4) return;
    const uint64_t i = 4 * t;
    uint4 v = col[t];
    uint32_t s0, s1, s2, s3;
    if (r == 0) {
        uint4 c = __ldg((const uint4 *)curr + t);
        s0 = c.x; s1 = c.y; s2 = c.z; s3 = c.w;
    } else {
        // 2^(r+1) >= 4: the four indices share i >> (r + 1)
        uint2 c = __ldg((const uint2 *)(curr + ((i >> (r + 1)) << 1)));
        s0 = c.x; s1 = c.y; s2 = c.x; s3 = c.y;
    }
    v.x = madd(v.x, s0); v.y = madd(v.y, s1); v.z = madd(v.z, s2); v.w = madd(v.w, s3);
    col[t] = v;
}

__global__ void accumulate_lift_kernel(uint32_t *__restrict__ col, const uint32_t *__restrict__ curr, uint64_t n,
                                       uint32_t r) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    col[i] = madd(col[i], curr[((i >> (r + 1)) << 1) | (i & 1)]);
}

// ---- pack_leaves (pack_leaves.cu:22-38): out[c*16 + p][i] = in[c][16 i + p].
// A block reads 16 x 32 consecutive words of one input column and writes 32
// consecutive words to each of the 16 output columns. ----
__global__ void __launch_bounds__(256) pack_leaves_kernel(const uint32_t *const *__restrict__ in,
                                                          uint32_t *const *__restrict__ out, uint64_t n_out) {
    __shared__ uint32_t tile[16][33];
    const uint32_t c = blockIdx.y;
    const uint64_t base = (uint64_t)blockIdx.x * 32u;  // output position of the tile
    const uint32_t *src = in[c];
    for (uint32_t k = threadIdx.x; k < 512u; k += blockDim.x) {
        const uint64_t pos = base + (k >> 4);
        if (pos < n_out) tile[k & 15u][k >> 4] = src[16ull * base + k];
    }
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < 512u; k += blockDim.x) {
        const uint32_t p = k >> 5, q = k & 31u;
        if (base + q < n_out) out[c * 16u + p][base + q] = tile[p][q];
    }
}

// ---- evaluation of a circle polynomial at a QM31 point by folding ----
// The reference folds level by level (circle_ntt.cu:186-231, 429-468):
// level l combines v[t] + f_l v[t + half], l = 0 at the top index bit.  The
// result is linear in the coefficients: sum_i c[i] w(i), w(i) the product of
// f_(log_n - 1 - b) over the set bits b of i, so any grouping gives the same
// field value.  For n = 2^11 (and when the first scratch buffer is not
// 16-byte aligned) a block folds a contiguous chunk of 2^11 coefficients
// (8 per thread in registers, then 8 levels in shared memory), scales the
// chunk's value by the factors of its high index bits, and a second kernel
// adds the chunk values.  Larger n take the table-driven form below.
constexpr uint32_t kEvalChunkLog = 11, kEvalThreads = 256;
__device__ __forceinline__ qm31 qscale(qm31 f, uint32_t m) { return qmulm(f, m); }

template <bool VEC>  // VEC: coeffs 16-byte aligned, two 16-byte loads per thread
__global__ void __launch_bounds__(kEvalThreads) eval_chunk_kernel(const uint32_t *__restrict__ coeffs,
                                                                  const uint32_t *__restrict__ factors,
                                                                  uint32_t log_n, uint32_t *__restrict__ partial) {
    __shared__ uint32_t fs[4 * 32];
    __shared__ qm31 s[kEvalThreads];
    const uint32_t t = threadIdx.x;
    if (t < 4 * log_n) fs[t] = factors[t];
    __syncthreads();
    auto fac = [&](uint32_t bit) {  // factor of index bit `bit`
        const uint32_t l = log_n - 1 - bit;
        return qm31{{fs[4 * l], fs[4 * l + 1], fs[4 * l + 2], fs[4 * l + 3]}};
    };
    const uint64_t base = ((uint64_t)blockIdx.x << kEvalChunkLog) + 8ull * t;
    uint32_t c[8];
    if (VEC) {
        const uint4 q0 = __ldg((const uint4 *)(coeffs + base)), q1 = __ldg((const uint4 *)(coeffs + base) + 1);
        c[0] = q0.x; c[1] = q0.y; c[2] = q0.z; c[3] = q0.w; c[4] = q1.x; c[5] = q1.y; c[6] = q1.z; c[7] = q1.w;
    } else {
#pragma unroll
        for (int j = 0; j < 8; j++) c[j] = __ldg(coeffs + base + j);
    }
    // index bits 2, 1, 0 of the thread's 8 coefficients
    const qm31 f2 = fac(2), f1 = fac(1), f0 = fac(0);
    qm31 u[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const qm31 b = qscale(f2, c[j + 4]);
        u[j] = {{madd(c[j], b.v[0]), b.v[1], b.v[2], b.v[3]}};
    }
    const qmat m1 = qmat_of(f1), m0 = qmat_of(f0);
    const qm31 w0 = qadd(u[0], qmul_mat(m1, u[2])), w1 = qadd(u[1], qmul_mat(m1, u[3]));
    s[t] = qadd(w0, qmul_mat(m0, w1));
    __syncthreads();
    // index bits 3 .. 10: thread bits 0 .. 7, highest first
    for (uint32_t k = 8; k-- > 0;) {
        const uint32_t half = 1u << k;
        if (t < half) s[t] = qadd(s[t], qmul_mat(qmat_of(fac(k + 3)), s[t + half]));
        __syncthreads();
    }
    if (t == 0) {
        qm31 r = s[0];
        const uint64_t chunk = blockIdx.x;
        for (uint32_t b = kEvalChunkLog; b < log_n; b++)
            if ((chunk >> (b - kEvalChunkLog)) & 1ull) r = qmul(r, fac(b));
#pragma unroll
        for (int w = 0; w < 4; w++) partial[4ull * blockIdx.x + w] = r.v[w];
    }
}

// Table-driven form for log_n >= 12.  With i = hi 2^11 + lo,
//   value = sum_hi W(hi) sum_lo c[i] w(lo),
// w(lo) the product of the factors of lo's set bits (bits 0..10) and W(hi)
// that of hi's (bits 11..), W(hi) = T1[hi mod 2^m1] T2[hi >> m1].  One block
// builds w, T1 and T2 by doubling and a second launch multiplies them into
// W(hi) for every chunk; persistent blocks hold w in shared memory, take
// 2048-coefficient chunks, multiply-accumulate in 64 bits and scale each
// thread's part of a chunk by W(hi); a last launch adds the block sums.
constexpr uint32_t kEvTabLog = 11, kEvTabThreads = 1024, kEvAccThreads = 256;

// Block 0 builds w (index bits 0..10), block 1 T1 (bits 11..11+m1-1),
// block 2 T2 (the rest), each by doubling in shared memory, then writes it.
__global__ void __launch_bounds__(kEvTabThreads) eval_tables_kernel(const uint32_t *__restrict__ factors,
                                                                    uint32_t log_n, uint32_t m1, uint32_t m2,
                                                                    uint32_t *wlo, uint32_t *t1, uint32_t *t2) {
    __shared__ qm31 tab[1u << kEvTabLog];
    const uint32_t t = threadIdx.x;
    const uint32_t b0 = blockIdx.x == 0 ? 0u : blockIdx.x == 1 ? kEvTabLog : kEvTabLog + m1;
    const uint32_t k = blockIdx.x == 0 ? kEvTabLog : blockIdx.x == 1 ? m1 : m2;
    uint32_t *out = blockIdx.x == 0 ? wlo : blockIdx.x == 1 ? t1 : t2;
    if (t == 0) tab[0] = qm31{{1u, 0u, 0u, 0u}};
    __syncthreads();
    for (uint32_t j = 0; j < k; j++) {
        const uint32_t l = log_n - 1 - (b0 + j);  // the factor of index bit b0 + j
        const qm31 f{{factors[4 * l], factors[4 * l + 1], factors[4 * l + 2], factors[4 * l + 3]}};
        for (uint32_t x = t; x < (1u << j); x += kEvTabThreads) tab[x + (1u << j)] = qmul(tab[x], f);
        __syncthreads();
    }
    for (uint32_t x = t; x < (1u << k); x += kEvTabThreads)
        for (int c = 0; c < 4; c++) out[4 * x + c] = tab[x].v[c];
}

// W(hi) = T1[hi mod 2^m1] T2[hi >> m1] for every chunk.
__global__ void eval_wtab_kernel(const uint32_t *__restrict__ t1, const uint32_t *__restrict__ t2, uint32_t m1,
                                 uint64_t chunks, uint32_t *__restrict__ wtab) {
    const uint64_t hi = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (hi >= chunks) return;
    const uint64_t i1 = hi & ((1ull << m1) - 1ull), i2 = hi >> m1;
    const qm31 r = qmul(qm31{{t1[4 * i1], t1[4 * i1 + 1], t1[4 * i1 + 2], t1[4 * i1 + 3]}},
                        qm31{{t2[4 * i2], t2[4 * i2 + 1], t2[4 * i2 + 2], t2[4 * i2 + 3]}});
#pragma unroll
    for (int k = 0; k < 4; k++) wtab[4 * hi + k] = r.v[k];
}

// Persistent blocks hold w in shared memory and take 2048-coefficient
// chunks; each thread multiply-accumulates its 8 coefficients of a chunk in
// 64 bits, scales that partial sum by the chunk's W(hi) and keeps its own
// running sum, so chunks need no block-wide step; the block adds its
// threads' sums once at the end.
__global__ void __launch_bounds__(kEvAccThreads) eval_accum_kernel(const uint32_t *__restrict__ coeffs,
                                                                   const uint32_t *__restrict__ wlo,
                                                                   const uint32_t *__restrict__ wtab,
                                                                   uint64_t chunks, uint32_t *__restrict__ partial) {
    __shared__ uint4 w[1u << kEvTabLog];
    __shared__ qm31 red[kEvAccThreads / 32];
    const uint32_t t = threadIdx.x, lane = t & 31u, warp = t >> 5;
    for (uint32_t x = t; x < (1u << kEvTabLog); x += kEvAccThreads) w[x] = __ldg((const uint4 *)wlo + x);
    __syncthreads();
    qm31 acc{{0u, 0u, 0u, 0u}};
    for (uint64_t hi = blockIdx.x; hi < chunks; hi += gridDim.x) {
        const uint32_t *cp = coeffs + (hi << kEvTabLog);
        uint32_t c[8];
#pragma unroll
        for (int j = 0; j < 8; j++) c[j] = __ldg(cp + t + kEvAccThreads * j);
        const qm31 W{{__ldg(wtab + 4 * hi), __ldg(wtab + 4 * hi + 1), __ldg(wtab + 4 * hi + 2),
                      __ldg(wtab + 4 * hi + 3)}};
        // products < 2^62: four of them, or a reduced value and four, stay below 2^64
        uint64_t a0 = 0, a1 = 0, a2 = 0, a3 = 0;
#pragma unroll
        for (int j = 0; j < 8; j++) {
            if (j == 4) { a0 = reduce64(a0); a1 = reduce64(a1); a2 = reduce64(a2); a3 = reduce64(a3); }
            const uint4 q = w[t + kEvAccThreads * j];
            a0 += (uint64_t)c[j] * q.x; a1 += (uint64_t)c[j] * q.y;
            a2 += (uint64_t)c[j] * q.z; a3 += (uint64_t)c[j] * q.w;
        }
        const qm31 v{{reduce64(a0), reduce64(a1), reduce64(a2), reduce64(a3)}};
        acc = qadd(acc, qmul_mat(qmat_of(W), v));
    }
#pragma unroll
    for (int m = 16; m > 0; m >>= 1) {
        qm31 o;
#pragma unroll
        for (int k = 0; k < 4; k++) o.v[k] = __shfl_xor_sync(0xFFFFFFFFu, acc.v[k], m);
        acc = qadd(acc, o);
    }
    if (lane == 0) red[warp] = acc;
    __syncthreads();
    if (t == 0) {
        qm31 sum = red[0];
        for (uint32_t k = 1; k < kEvAccThreads / 32; k++) sum = qadd(sum, red[k]);
#pragma unroll
        for (int k = 0; k < 4; k++) partial[4ull * blockIdx.x + k] = sum.v[k];
    }
}

__global__ void __launch_bounds__(kEvalThreads) eval_sum_kernel(const uint32_t *__restrict__ vals, uint64_t count,
                                                                const uint32_t *__restrict__ coeffs,
                                                                const uint32_t *__restrict__ factors, uint32_t log_n,
                                                                uint32_t *__restrict__ out) {
    __shared__ qm31 s[kEvalThreads];
    const uint32_t t = threadIdx.x;
    qm31 acc{{0u, 0u, 0u, 0u}};
    if (coeffs) {  // small polynomial: weight each coefficient directly
        for (uint64_t i = t; i < (1ull << log_n); i += kEvalThreads) {
            qm31 w{{1u, 0u, 0u, 0u}};
            for (uint32_t b = 0; b < log_n; b++)
                if ((i >> b) & 1ull) {
                    const uint32_t l = log_n - 1 - b;
                    w = qmul(w, qm31{{factors[4 * l], factors[4 * l + 1], factors[4 * l + 2], factors[4 * l + 3]}});
                }
            acc = qadd(acc, qmulm(w, coeffs[i]));
        }
    } else {
        for (uint64_t i = t; i < count; i += kEvalThreads)
            acc = qadd(acc, qm31{{vals[4 * i], vals[4 * i + 1], vals[4 * i + 2], vals[4 * i + 3]}});
    }
    s[t] = acc;
    __syncthreads();
    for (uint32_t half = kEvalThreads / 2; half > 0; half >>= 1) {
        if (t < half) s[t] = qadd(s[t], s[t + half]);
        __syncthreads();
    }
    if (t < 4) out[t] = s[0].v[t];
}

// ---- barycentric evaluation partial sums (barycentric_eval.cu:52-94) ----
// Block b accumulates evals[i] * weights[i] (M31 times QM31, weights AoS)
// over the i that a grid-stride loop of n_blocks x 256 threads gives it, so
// the partial sums are the reference's.
// Each thread keeps kBaryInFlight of its elements in flight per step (the launch has
// only n_blocks <= 256 blocks of 256 threads); it still accumulates exactly
// the elements i = its index + k * (grid threads), so each block's sum is the
// reference's.  VEC: weights 16-byte aligned, one 16-byte load per weight.
constexpr int kBaryInFlight = 8;
template <bool VEC>
__device__ __forceinline__ qm31 bary_weight(const uint32_t *__restrict__ weights, uint64_t i) {
    if (VEC) {
        const uint4 q = __ldg((const uint4 *)weights + i);
        return qm31{{q.x, q.y, q.z, q.w}};
    }
    const uint64_t b = 4ull * i;
    return qm31{{__ldg(weights + b), __ldg(weights + b + 1), __ldg(weights + b + 2), __ldg(weights + b + 3)}};
}

template <bool VEC>
__global__ void __launch_bounds__(256) barycentric_kernel(const uint32_t *__restrict__ evals,
                                                          const uint32_t *__restrict__ weights, uint32_t n,
                                                          uint32_t *__restrict__ out) {
    __shared__ qm31 s[8];
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    // 64-bit multiply-accumulate per coordinate, folded every 4 products:
    // (x & P) + (x >> 31) < 2^34 plus four products of canonical words
    // (< 2^62 each) stays below 2^64; reduced to canonical M31 once
    uint64_t a0 = 0, a1 = 0, a2 = 0, a3 = 0;
    auto fold = [&]() {
        a0 = (a0 & VX_P) + (a0 >> 31); a1 = (a1 & VX_P) + (a1 >> 31);
        a2 = (a2 & VX_P) + (a2 >> 31); a3 = (a3 & VX_P) + (a3 >> 31);
    };
    auto mac = [&](const qm31 &w, uint32_t e) {
        a0 += (uint64_t)w.v[0] * e; a1 += (uint64_t)w.v[1] * e;
        a2 += (uint64_t)w.v[2] * e; a3 += (uint64_t)w.v[3] * e;
    };
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    for (; i + (kBaryInFlight - 1) * stride < n; i += kBaryInFlight * stride) {
        uint32_t e[kBaryInFlight];
        qm31 w[kBaryInFlight];
#pragma unroll
        for (int k = 0; k < kBaryInFlight; k++) {
            e[k] = __ldg(evals + i + k * stride);
            w[k] = bary_weight<VEC>(weights, i + k * stride);
        }
#pragma unroll
        for (int k = 0; k < kBaryInFlight; k++) {
            mac(w[k], e[k]);
            if ((k & 3) == 3) fold();
        }
    }
    for (; i < n; i += stride) {
        mac(bary_weight<VEC>(weights, i), __ldg(evals + i));
        fold();
    }
    fold();
    qm31 acc{{reduce64(a0), reduce64(a1), reduce64(a2), reduce64(a3)}};
#pragma unroll
    for (int m = 16; m > 0; m >>= 1) {
        qm31 o;
#pragma unroll
        for (int c = 0; c < 4; c++) o.v[c] = __shfl_xor_sync(0xffffffffu, acc.v[c], m);
        acc = qadd(acc, o);
    }
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    if (lane == 0) s[warp] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        qm31 r = s[0];
        for (uint32_t w = 1; w < (blockDim.x + 31) / 32; w++) r = qadd(r, s[w]);
#pragma unroll
        for (int c = 0; c < 4; c++) out[4 * blockIdx.x + c] = r.v[c];
    }
}

// ---- gathers (gather.cu): dst[i] = src[idx[i]], or 8-word elements ----
// The bounded forms skip an element whose source lies outside src_len words.
__global__ void gather_u32_kernel(const uint32_t *__restrict__ src, const uint32_t *__restrict__ idx,
                                  uint32_t *__restrict__ dst, uint32_t n, uint64_t src_len) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t j = idx[i];
    if (j < src_len) dst[i] = src[j];
}
__global__ void gather_u256_kernel(const uint32_t *__restrict__ src, const uint32_t *__restrict__ idx,
                                   uint32_t *__restrict__ dst, uint32_t n, uint64_t src_len) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint64_t j = 8ull * idx[i];
    if (j + 8 > src_len) return;
#pragma unroll
    for (int w = 0; w < 8; w++) dst[8ull * i + w] = src[j + w];
}

}  // namespace
}  // namespace vx

using namespace vx;

extern "C" {

void cuda_stwo_ntt_evaluate(uint32_t *d, const uint32_t *tw, uint32_t n) {
    if (!stwo_size_ok(n, "cuda_stwo_ntt_evaluate")) return;
    const uint32_t log_n = log2_of(n);
    cudaError_t e = ntt_transform(d, nullptr, 0, 1, log_n, stwo_tables(tw, log_n), true, nullptr, 0, 0);
    if (e != cudaSuccess) set_last_error(VX_ERR_CUDA, "cuda_stwo_ntt_evaluate: %s", cudaGetErrorString(e));
    cudaDeviceSynchronize();
}

void cuda_stwo_ntt_interpolate(uint32_t *d, const uint32_t *itw, uint32_t n) {
    if (!stwo_size_ok(n, "cuda_stwo_ntt_interpolate")) return;
    const uint32_t log_n = log2_of(n);
    cudaError_t e = ntt_transform(d, nullptr, 0, 1, log_n, stwo_tables(itw, log_n), false, nullptr, 0, 0);
    if (e != cudaSuccess) set_last_error(VX_ERR_CUDA, "cuda_stwo_ntt_interpolate: %s", cudaGetErrorString(e));
    cudaDeviceSynchronize();
}

static void stwo_batch(uint32_t *const *cols, const uint32_t *tw, uint32_t n, uint32_t n_cols, bool fwd,
                       const char *who) {
    if (n_cols == 0 || n < 2) return;  // the reference returns early for these
    if (!stwo_size_ok(n, who)) return;
    const uint32_t log_n = log2_of(n);
    std::lock_guard<std::mutex> lk(g_ptr_mu);
    uint32_t **dev = nullptr;
    cudaError_t e = upload_ptrs(cols, n_cols, &dev);
    if (e == cudaSuccess) e = ntt_transform(nullptr, dev, 0, n_cols, log_n, stwo_tables(tw, log_n), fwd, nullptr, 0, 0);
    if (e != cudaSuccess) set_last_error(VX_ERR_CUDA, "%s: %s", who, cudaGetErrorString(e));
    cudaDeviceSynchronize();  // the pointer buffer is reused by the next call
}

void cuda_stwo_ntt_batch_evaluate(uint32_t *const *cols, const uint32_t *tw, uint32_t n, uint32_t n_cols) {
    stwo_batch(cols, tw, n, n_cols, true, "cuda_stwo_ntt_batch_evaluate");
}

void cuda_stwo_ntt_batch_interpolate(uint32_t *const *cols, const uint32_t *itw, uint32_t n, uint32_t n_cols) {
    stwo_batch(cols, itw, n, n_cols, false, "cuda_stwo_ntt_batch_interpolate");
}

void cuda_bit_reverse_qm31(const uint32_t *in, uint32_t *out, uint32_t n, uint32_t log_n) {
    if (n == 0) return;
    if (log_n > 31 || (1ull << log_n) != n) {
        set_last_error(VX_ERR_ARG, "cuda_bit_reverse_qm31: n = %u is not 2^log_n (log_n = %u)", n, log_n);
        return;
    }
    const bool aligned = (((uintptr_t)in | (uintptr_t)out) & 15u) == 0;
    if (log_n >= 2 * kBrT && aligned)
        brev_qm31_tiled_kernel<<<(unsigned)(1ull << (log_n - 2 * kBrT)), 256>>>((const uint4 *)in, (uint4 *)out,
                                                                                log_n);
    else
        brev_qm31_kernel<<<blocks_for(n, 256), 256>>>(in, out, n, log_n);
    VX_LAUNCH_CHECK();
}

void cuda_accumulate_lift(uint32_t *col, const uint32_t *curr, uint32_t col_n, uint32_t log_ratio) {
    if (col_n == 0) return;
    const bool vec = (col_n % 4u == 0) && (((uintptr_t)col & 15u) == 0) &&
                     (log_ratio == 0 ? (((uintptr_t)curr & 15u) == 0) : (((uintptr_t)curr & 7u) == 0));
    if (vec)
        accumulate_lift4_kernel<<<blocks_for(col_n / 4u, 256), 256>>>((uint4 *)col, curr, col_n / 4u, log_ratio);
    else
        accumulate_lift_kernel<<<blocks_for(col_n, 256), 256>>>(col, curr, col_n, log_ratio);
    VX_LAUNCH_CHECK();
}

void cuda_pack_leaves(const uint32_t *const *input_col_ptrs, uint32_t *const *output_col_ptrs, uint32_t n) {
    if (n == 0) return;
    if (n % 16u) {
        set_last_error(VX_ERR_ARG, "cuda_pack_leaves: N = %u is not a multiple of 16", n);
        return;
    }
    const uint64_t n_out = n / 16u;
    pack_leaves_kernel<<<dim3(blocks_for(n_out, 32), 4), 256>>>(input_col_ptrs, output_col_ptrs, n_out);
    VX_LAUNCH_CHECK();
}

void cuda_bit_reverse_qm31_forge(const uint32_t *in, uint32_t *out, uint32_t n, uint32_t log_n) {
    cuda_bit_reverse_qm31(in, out, n, log_n);
}

void cuda_gather_u32(const uint32_t *src, const uint32_t *idx, uint32_t *dst, uint32_t n) {
    if (n == 0) return;
    gather_u32_kernel<<<blocks_for(n, 256), 256>>>(src, idx, dst, n, ~0ull);
    VX_LAUNCH_CHECK();
}
void cuda_gather_u32_forge(const uint32_t *src, const uint32_t *idx, uint32_t *dst, uint32_t n, uint32_t src_len) {
    if (n == 0) return;
    gather_u32_kernel<<<blocks_for(n, 256), 256>>>(src, idx, dst, n, src_len);
    VX_LAUNCH_CHECK();
}
void cuda_gather_u256(const uint32_t *src, const uint32_t *idx, uint32_t *dst, uint32_t n) {
    if (n == 0) return;
    gather_u256_kernel<<<blocks_for(n, 256), 256>>>(src, idx, dst, n, ~0ull);
    VX_LAUNCH_CHECK();
}
void cuda_gather_u256_forge(const uint32_t *src, const uint32_t *idx, uint32_t *dst, uint32_t n, uint32_t src_len) {
    if (n == 0) return;
    gather_u256_kernel<<<blocks_for(n, 256), 256>>>(src, idx, dst, n, src_len);
    VX_LAUNCH_CHECK();
}

void cuda_barycentric_eval(const uint32_t *evals, const uint32_t *weights, uint32_t n, uint32_t *out,
                           uint32_t n_blocks) {
    if (n_blocks == 0) return;
    if (((uintptr_t)weights & 15u) == 0)
        barycentric_kernel<true><<<n_blocks, 256>>>(evals, weights, n, out);
    else
        barycentric_kernel<false><<<n_blocks, 256>>>(evals, weights, n, out);
    VX_LAUNCH_CHECK();
    cudaDeviceSynchronize();  // the reference's launcher returns with the sums in place
}

// Scratch as poly_ops.rs allocates it (2n words each).  log_n >= 12 with a
// 16-byte-aligned d_scratch1: the low-bit table (2^13 words) in d_scratch1,
// the high-bit tables, the chunk weights and the block sums (at most
// 12 n / 2^11 + 8 words) in d_scratch2.  Smaller or unaligned: the chunk fold, which uses at most
// 4 n / 2^11 + 4 words of d_scratch1.
void cuda_eval_at_point(const uint32_t *d_coeffs, const uint32_t *d_folding_factors, uint32_t *h_result, uint32_t n,
                        uint32_t *d_scratch1, uint32_t *d_scratch2) {
    if (n == 0 || (n & (n - 1u))) {
        set_last_error(VX_ERR_ARG, "cuda_eval_at_point: n = %u is not a power of two", n);
        return;
    }
    const uint32_t log_n = 31u - __builtin_clz(n);
    if (log_n == 0) {  // a constant: the coefficient itself
        uint32_t c = 0;
        if (cudaMemcpy(&c, d_coeffs, 4, cudaMemcpyDeviceToHost) != cudaSuccess) { VX_LAUNCH_CHECK(); return; }
        h_result[0] = c; h_result[1] = h_result[2] = h_result[3] = 0u;
        return;
    }
    if (log_n < kEvalChunkLog) {
        eval_sum_kernel<<<1, kEvalThreads>>>(nullptr, 0, d_coeffs, d_folding_factors, log_n, d_scratch1);
    } else if (log_n > kEvTabLog && ((uintptr_t)d_scratch1 & 15u) == 0 && d_scratch2 != nullptr) {
        const uint32_t H = log_n - kEvTabLog, m1 = H < 10u ? H : 10u, m2 = H - m1;
        const uint64_t chunks = 1ull << H;
        uint32_t *wlo = d_scratch1, *t1 = d_scratch2, *t2 = t1 + (4u << m1), *wtab = t2 + (4u << m2),
                 *part = wtab + 4 * chunks;
        int dev = 0, sms = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) {
            cudaGetLastError();
            sms = 148;
        }
        const unsigned grid = (unsigned)(chunks < (uint64_t)sms * 6u ? chunks : (uint64_t)sms * 6u);
        eval_tables_kernel<<<3, kEvTabThreads>>>(d_folding_factors, log_n, m1, m2, wlo, t1, t2);
        eval_wtab_kernel<<<blocks_for(chunks, 256), 256>>>(t1, t2, m1, chunks, wtab);
        eval_accum_kernel<<<grid, kEvAccThreads>>>(d_coeffs, wlo, wtab, chunks, part);
        eval_sum_kernel<<<1, kEvalThreads>>>(part, grid, nullptr, nullptr, 0, part + 4ull * grid);
        d_scratch1 = part + 4ull * grid;  // where the value lands
    } else {
        const uint64_t chunks = 1ull << (log_n - kEvalChunkLog);
        if (((uintptr_t)d_coeffs & 15u) == 0)
            eval_chunk_kernel<true><<<(unsigned)chunks, kEvalThreads>>>(d_coeffs, d_folding_factors, log_n, d_scratch1);
        else
            eval_chunk_kernel<false><<<(unsigned)chunks, kEvalThreads>>>(d_coeffs, d_folding_factors, log_n, d_scratch1);
        eval_sum_kernel<<<1, kEvalThreads>>>(d_scratch1, chunks, nullptr, nullptr, 0, d_scratch1 + 4 * chunks);
        d_scratch1 += 4 * chunks;
    }
    VX_LAUNCH_CHECK();
    if (cudaMemcpy(h_result, d_scratch1, 16, cudaMemcpyDeviceToHost) != cudaSuccess) VX_LAUNCH_CHECK();
}

}  // extern "C"

extern "C" int vx_stwo_twiddles(uint32_t log_n, int inverse, uint32_t *out, void *stream) {
    VX_CHECK_ARG(out != nullptr, "vx_stwo_twiddles: out is null");
    VX_CHECK_ARG(log_n >= 2 && log_n <= 29, "vx_stwo_twiddles: log_n %u outside 2..29", log_n);
    GenTables g;
    VX_CUDA_TRY(gen_tables_get(&g));
    VX_CUDA_TRY(build_stwo_table_with(g, log_n, inverse != 0, out, (cudaStream_t)stream));
    return VX_OK;
}

extern "C" int vx_stwo_fold_circle_twiddles(uint32_t log, uint32_t *out, void *stream) {
    VX_CHECK_ARG(out != nullptr, "vx_stwo_fold_circle_twiddles: out is null");
    VX_CHECK_ARG(log >= 2 && log <= 30, "vx_stwo_fold_circle_twiddles: log %u outside 2..30", log);
    GenTables g;
    VX_CUDA_TRY(gen_tables_get(&g));
    VX_CUDA_TRY(build_stwo_fold_circle_with(g, log, out, (cudaStream_t)stream));
    return VX_OK;
}
