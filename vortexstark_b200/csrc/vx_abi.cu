// Reference-compatible launchers (the symbols src/cuda/ffi.rs binds).
//
// Each keeps the reference's signature and semantics: device pointers for
// data, host pointers for alpha[4] and layer offsets, legacy default stream
// unless a stream is passed, and cudaDeviceSynchronize at the end of the NTT
// evaluate / interpolate launchers (circle_ntt.cu:274, 311).  The kernels
// are this library's own.
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>

#include <mutex>

#include "vx_common.cuh"
#include "vx_field.cuh"
#include "vx_merkle.cuh"
#include "vx_ntt.cuh"
#include "vx_twiddles.cuh"

namespace vx {

static thread_local std::string t_err;

void set_last_error(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    t_err = buf;
    (void)code;
}

namespace {

inline uint32_t log2_exact(uint64_t n) {
    uint32_t l = 0;
    while ((1ull << l) < n) l++;
    return l;
}

// ---- twiddle helpers for arbitrary (initial, step) points ----
// p_j = initial * step^j, 16 consecutive points per thread (twiddles.cu:80-105).
// Thread t of T writes points t, t + T, t + 2T, ... (about 16 each), stepping
// by step^T, so a warp's stores are consecutive words.
__global__ void coset_points_kernel(cpoint init, cpoint step, uint32_t *xs, uint32_t *ys, uint64_t n) {
    const uint64_t T = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const cpoint stride_step = ppow(step, T);
    cpoint p = pmul(init, ppow(step, t));
    for (uint64_t j = t; j < n; j += T) {
        xs[j] = p.x;
        ys[j] = p.y;
        p = pmul(p, stride_step);
    }
}

__global__ void extract_squash_kernel(const uint32_t *in, uint32_t *tw_out, uint32_t *sq_out, uint64_t half_n) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= half_n) return;
    uint32_t x = in[2 * i];
    if (tw_out) tw_out[i] = x;
    uint32_t x2 = mmul(x, x);
    sq_out[i] = msub(madd(x2, x2), 1u);
}

// coord(initial * step^brev(2i, log_n)), i < n/2 (twiddles.cu:23-52).
__global__ void fold_sources_generic_kernel(cpoint init, cpoint step, uint32_t *out, uint64_t half, uint32_t log_n,
                                            int extract_y) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= half) return;
    cpoint p = pmul(init, ppow(step, brev_bits((uint32_t)(i << 1), log_n)));
    out[i] = extract_y ? p.y : p.x;
}

// ---- glue (constraint.cu) ----
// VEC: four words per thread with 16-byte accesses (both arrays 16-byte
// aligned); a group that straddles src_n or dst_n goes word by word.
template <bool VEC>
__global__ void zero_pad_kernel(const uint32_t *src, uint32_t *dst, uint64_t src_n, uint64_t dst_n) {
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (!VEC) {
        if (t < dst_n) dst[t] = t < src_n ? src[t] : 0u;
        return;
    }
    const uint64_t i = 4 * t;
    if (i >= dst_n) return;
    if (i + 4 <= dst_n && i + 4 <= src_n) {
        *(uint4 *)(dst + i) = *(const uint4 *)(src + i);
    } else if (i + 4 <= dst_n && i >= src_n) {
        *(uint4 *)(dst + i) = make_uint4(0u, 0u, 0u, 0u);
    } else {
        for (uint64_t j = i; j < i + 4 && j < dst_n; j++) dst[j] = j < src_n ? src[j] : 0u;
    }
}

__device__ __forceinline__ void quotient_one(const uint32_t *tr, uint32_t *o0, uint32_t *o1, uint32_t *o2,
                                             uint32_t *o3, uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                             uint64_t li, uint64_t i, uint64_t global_n) {
    // (i + 1) mod N and (i + 2) mod N for i < N by one conditional subtraction
    // each; N < 3 (where i + 2 can pass 2N) keeps the division
    uint64_t i1 = i + 1, i2 = i + 2;
    if (global_n > 2) {
        if (i1 >= global_n) i1 -= global_n;
        if (i2 >= global_n) i2 -= global_n;
    } else {
        i1 %= global_n;
        i2 %= global_n;
    }
    const uint32_t c = msub(tr[i2], madd(tr[i1], tr[i]));
    o0[li] = mmul(a0, c); o1[li] = mmul(a1, c); o2[li] = mmul(a2, c); o3[li] = mmul(a3, c);
}

// VEC: four consecutive points per thread with 16-byte loads and stores
// (the host checks 16-byte alignment of every array, offset and chunk
// multiples of 4 and N > 2); the last group before the wrap-around takes the
// scalar form.
template <bool VEC>
__global__ void quotient_kernel(const uint32_t *tr, uint32_t *o0, uint32_t *o1, uint32_t *o2, uint32_t *o3,
                                uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint64_t offset, uint64_t chunk,
                                uint64_t global_n) {
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (!VEC) {
        if (t < chunk) quotient_one(tr, o0, o1, o2, o3, a0, a1, a2, a3, t, offset + t, global_n);
        return;
    }
    const uint64_t li = 4 * t;
    if (li >= chunk) return;
    const uint64_t i = offset + li;
    if (i + 5 >= global_n) {
        for (uint32_t k = 0; k < 4; k++) quotient_one(tr, o0, o1, o2, o3, a0, a1, a2, a3, li + k, i + k, global_n);
        return;
    }
    const uint4 x = *(const uint4 *)(tr + i);
    const uint2 y = *(const uint2 *)(tr + i + 4);
    const uint32_t v[6] = {x.x, x.y, x.z, x.w, y.x, y.y};
    uint32_t c[4];
#pragma unroll
    for (int k = 0; k < 4; k++) c[k] = msub(v[k + 2], madd(v[k + 1], v[k]));
    *(uint4 *)(o0 + li) = make_uint4(mmul(a0, c[0]), mmul(a0, c[1]), mmul(a0, c[2]), mmul(a0, c[3]));
    *(uint4 *)(o1 + li) = make_uint4(mmul(a1, c[0]), mmul(a1, c[1]), mmul(a1, c[2]), mmul(a1, c[3]));
    *(uint4 *)(o2 + li) = make_uint4(mmul(a2, c[0]), mmul(a2, c[1]), mmul(a2, c[2]), mmul(a2, c[3]));
    *(uint4 *)(o3 + li) = make_uint4(mmul(a3, c[0]), mmul(a3, c[1]), mmul(a3, c[2]), mmul(a3, c[3]));
}

// ---- bit reverse / permute ----
// In place, tiled (log_n >= 10): write i = hi | mid << 5 | lo << ... as
// (hi: top 5 bits, mid, lo: low 5 bits); brev(i) lies in tile brev(mid) at
// row brev(lo), column brev(hi).  The block of tile pair (mid, brev(mid)),
// mid <= brev(mid), reads both 32 x 32 tiles (128-byte rows) before writing
// either, so the swap is race-free; blocks with mid > brev(mid) exit.
constexpr uint32_t kBrevT = 5, kBrevS = 1u << kBrevT;
__global__ void __launch_bounds__(256) bit_reverse_tiled_kernel(uint32_t *d, uint32_t log_n) {
    __shared__ uint32_t ta[kBrevS][kBrevS + 1], tb[kBrevS][kBrevS + 1];
    const uint32_t mid_bits = log_n - 2 * kBrevT;
    const uint32_t mid = blockIdx.x;
    const uint32_t bmid = mid_bits ? brev_bits(mid, mid_bits) : 0u;
    if (mid > bmid) return;
    const uint32_t tx = threadIdx.x & (kBrevS - 1u), ty = threadIdx.x >> kBrevT;  // 32 x 8
    const uint32_t hs = log_n - kBrevT;
#pragma unroll
    for (uint32_t r = 0; r < kBrevS; r += 8) {
        const uint32_t h = ty + r;
        ta[h][tx] = d[tx | ((uint64_t)mid << kBrevT) | ((uint64_t)h << hs)];
        if (bmid != mid) tb[h][tx] = d[tx | ((uint64_t)bmid << kBrevT) | ((uint64_t)h << hs)];
    }
    __syncthreads();
    // new[tile t](h', l') = old[tile brev(t)](brev(l'), brev(h'))
#pragma unroll
    for (uint32_t r = 0; r < kBrevS; r += 8) {
        const uint32_t h2 = ty + r, l2 = tx;
        const uint32_t sh = brev_bits(l2, kBrevT), sl = brev_bits(h2, kBrevT);
        d[l2 | ((uint64_t)bmid << kBrevT) | ((uint64_t)h2 << hs)] = ta[sh][sl];
        if (bmid != mid) d[l2 | ((uint64_t)mid << kBrevT) | ((uint64_t)h2 << hs)] = tb[sh][sl];
    }
}

// The same with 64 x 64 tiles (log_n >= 12): rows of 64 words move as one
// 256-byte uint2 access per warp, like the permutation below.
constexpr uint32_t kBrevT6 = 6, kBrevS6 = 1u << kBrevT6;
__global__ void __launch_bounds__(256) bit_reverse_tiled64_kernel(uint32_t *d, uint32_t log_n) {
    __shared__ uint32_t ta[kBrevS6][kBrevS6 + 1], tb[kBrevS6][kBrevS6 + 1];
    const uint32_t mid_bits = log_n - 2 * kBrevT6;
    const uint32_t mid = blockIdx.x;
    const uint32_t bmid = mid_bits ? brev_bits(mid, mid_bits) : 0u;
    if (mid > bmid) return;
    const uint32_t tx = threadIdx.x & 31u, ty = threadIdx.x >> 5;  // 32 lanes x 8 rows, 2 words per lane
    const uint32_t hs = log_n - kBrevT6;
#pragma unroll
    for (uint32_t r = 0; r < kBrevS6; r += 8) {
        const uint32_t h = ty + r;
        const uint2 va = ((const uint2 *)(d + ((uint64_t)mid << kBrevT6) + ((uint64_t)h << hs)))[tx];
        ta[h][2 * tx] = va.x; ta[h][2 * tx + 1] = va.y;
        if (bmid != mid) {
            const uint2 vb = ((const uint2 *)(d + ((uint64_t)bmid << kBrevT6) + ((uint64_t)h << hs)))[tx];
            tb[h][2 * tx] = vb.x; tb[h][2 * tx + 1] = vb.y;
        }
    }
    __syncthreads();
#pragma unroll
    for (uint32_t r = 0; r < kBrevS6; r += 8) {
        const uint32_t h2 = ty + r;
        const uint32_t c = brev_bits(h2, kBrevT6), r0 = brev_bits(2 * tx, kBrevT6), r1 = brev_bits(2 * tx + 1, kBrevT6);
        ((uint2 *)(d + ((uint64_t)bmid << kBrevT6) + ((uint64_t)h2 << hs)))[tx] = make_uint2(ta[r0][c], ta[r1][c]);
        if (bmid != mid)
            ((uint2 *)(d + ((uint64_t)mid << kBrevT6) + ((uint64_t)h2 << hs)))[tx] = make_uint2(tb[r0][c], tb[r1][c]);
    }
}

__global__ void bit_reverse_kernel(uint32_t *d, uint32_t log_n, uint64_t n) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint64_t j = brev_bits((uint32_t)i, log_n);
    if (i < j) { uint32_t t = d[i]; d[i] = d[j]; d[j] = t; }
}

__device__ __forceinline__ uint64_t hc_to_canonic_brt(uint64_t k, uint64_t n, uint32_t log_n) {
    uint64_t cn = (k & 1ull) ? n - 1ull - (k >> 1) : (k >> 1);
    return brev_bits((uint32_t)cn, log_n);
}

// Tiled form of the permutation (log_n >= 12).  With k = 2q + b (b the
// parity) and M = 2^(log_n-1) - 1, j(k) = 2 (brev(q) ^ (b ? M : 0)) + b: a
// bit reversal of the even words and a complemented one of the odd words
// over the (log_n - 1)-bit pair index.  j is an involution, so the forward
// scatter and the inverse gather are the same out-of-place gather
// dst[2u + b] = src[j(2u + b)].  Pairs u = lo | mid << 5 | hi << (L - 5),
// L = log_n - 1: destination tiles m and ~m (complement in the mid bits)
// read exactly the source tiles brev(m) and ~brev(m), 32 x 32 pairs each.
__global__ void __launch_bounds__(256) permute_tiled_kernel(const uint2 *__restrict__ src, uint2 *__restrict__ dst,
                                                            uint32_t log_n) {
    __shared__ uint32_t ax[kBrevS][kBrevS + 1], ay[kBrevS][kBrevS + 1];
    __shared__ uint32_t bx[kBrevS][kBrevS + 1], by[kBrevS][kBrevS + 1];
    const uint32_t L = log_n - 1, mid_bits = L - 2 * kBrevT, mmask = (1u << mid_bits) - 1u;
    const uint32_t m = blockIdx.x, m2 = m ^ mmask;          // m has its top mid bit clear
    const uint32_t sa = brev_bits(m, mid_bits), sb = sa ^ mmask;
    const uint32_t tx = threadIdx.x & (kBrevS - 1u), ty = threadIdx.x >> kBrevT;
    const uint32_t hs = L - kBrevT;
#pragma unroll
    for (uint32_t r = 0; r < kBrevS; r += 8) {
        const uint32_t h = ty + r;
        const uint2 va = src[tx | ((uint64_t)sa << kBrevT) | ((uint64_t)h << hs)];
        const uint2 vb = src[tx | ((uint64_t)sb << kBrevT) | ((uint64_t)h << hs)];
        ax[h][tx] = va.x; ay[h][tx] = va.y;
        bx[h][tx] = vb.x; by[h][tx] = vb.y;
    }
    __syncthreads();
#pragma unroll
    for (uint32_t r = 0; r < kBrevS; r += 8) {
        const uint32_t h2 = ty + r, l2 = tx;
        const uint32_t rr = brev_bits(l2, kBrevT), cc = brev_bits(h2, kBrevT);
        const uint32_t nr = rr ^ (kBrevS - 1u), nc = cc ^ (kBrevS - 1u);
        dst[l2 | ((uint64_t)m << kBrevT) | ((uint64_t)h2 << hs)] = make_uint2(ax[rr][cc], by[nr][nc]);
        dst[l2 | ((uint64_t)m2 << kBrevT) | ((uint64_t)h2 << hs)] = make_uint2(bx[rr][cc], ay[nr][nc]);
    }
}

bool permute_tiled_ok(const uint32_t *src, const uint32_t *dst, uint32_t n, uint32_t log_n) {
    return log_n >= 12 && log_n <= 31 && (1ull << log_n) == n && src != dst &&
           ((((uintptr_t)src) | ((uintptr_t)dst)) & 7u) == 0;
}

// permute.cu:30-58: forward scatters dst[j(k)] = src[k]; inverse gathers.
__global__ void permute_kernel(const uint32_t *src, uint32_t *dst, uint64_t n, uint32_t log_n, int inverse) {
    uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    uint64_t j = hc_to_canonic_brt(k, n, log_n);
    if (inverse) dst[k] = src[j]; else dst[j] = src[k];
}

// ---- Merkle helpers ----
template <class Src>
// `one` (always 1): pipe balance of the Blake2s compression.
__global__ void leaf_hash_kernel(Src src, uint32_t *hashes, uint64_t n, uint32_t one) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    src.init();
    uint32_t m[16];
#pragma unroll
    for (int w = 0; w < 16; w++) m[w] = 0u;
    uint32_t nb = src.load(i, m);
    uint32_t h[8];
    blake2s_block(h, m, nb, one);
    store_hash(hashes + 8 * i, h);
}

__global__ void node_hash_kernel(const uint32_t *children, uint32_t *parents, uint64_t n, uint32_t one) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t m[16];
    const uint4 *c = (const uint4 *)(children + 16 * i);
    uint4 a = c[0], b = c[1], d = c[2], e = c[3];
    m[0] = a.x; m[1] = a.y; m[2] = a.z; m[3] = a.w; m[4] = b.x; m[5] = b.y; m[6] = b.z; m[7] = b.w;
    m[8] = d.x; m[9] = d.y; m[10] = d.z; m[11] = d.w; m[12] = e.x; m[13] = e.y; m[14] = e.z; m[15] = e.w;
    uint32_t h[8];
    blake2s_block(h, m, 64u, one);
    store_hash(parents + 8 * i, h);
}

// Reduce the 8-word hashes in sh[0 .. 8*cnt) to sh[0..8) (block-wide).
__device__ void block_reduce_hashes(uint32_t *sh, uint32_t cnt) {
    for (; cnt > 1; cnt >>= 1) {
        uint32_t h[8];
        uint32_t t = threadIdx.x;
        bool act = t < cnt / 2;
        if (act) blake2s_node(h, sh + 16 * t, sh + 16 * t + 8);
        __syncthreads();
        if (act)
            for (int w = 0; w < 8; w++) sh[8 * t + w] = h[w];
        __syncthreads();
    }
}

__global__ void reduce_to_root_kernel(const uint32_t *nodes, uint32_t *root, uint32_t n) {
    extern __shared__ uint32_t sh[];
    for (uint32_t i = threadIdx.x; i < 8 * n; i += blockDim.x) sh[i] = nodes[i];
    __syncthreads();
    block_reduce_hashes(sh, n);
    if (threadIdx.x < 8) root[threadIdx.x] = sh[threadIdx.x];
}

// Tile of 2^tile_log leaves per block, 2^(tile_log-4) threads each hashing
// 16 leaves into a subtree root, then a shared-memory reduction.
// A warp per TW 1024-leaf tiles (TW = 1, 2, 4): each of a tile's 32 / TW
// lanes hashes a subtree of 32 TW leaves, then the warp reduces its tiles'
// roots together in shared memory with warp barriers only, so no warp waits
// on another.  A reduction step costs the whole warp's issue however few
// lanes are active, so the tail is log2(32 / TW) steps for TW tiles at once.
// Blocks of 4 warps.
template <uint32_t TW, class Src>
__global__ void __launch_bounds__(128) tile_root_warp_kernel(Src src, uint32_t *roots, uint64_t tiles, uint32_t one) {
    constexpr uint32_t LPT = 32 / TW;                      // lanes per tile
    constexpr uint32_t KL = TW == 1 ? 5 : TW == 2 ? 6 : 7;  // log2 leaves per lane
    __shared__ __align__(16) uint32_t sh[4][32 * 8];
    const uint32_t w = threadIdx.x >> 5, l = threadIdx.x & 31u;
    const uint64_t wt = ((uint64_t)blockIdx.x * 4u + w) * TW;  // the warp's first tile
    if (wt >= tiles) return;  // whole warps leave together
    const uint32_t tl = l / LPT, sub = l % LPT;
    const uint64_t tile = wt + tl;
    src.init();
    uint32_t h[8] = {0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u};
    if (tile < tiles) subtree_root<Src, KL>(src, (tile << 10) + ((uint64_t)sub << KL), KL, h, one);
    uint32_t *s = sh[w] + 8 * LPT * tl;  // this tile's digests
    store_hash(s + 8 * sub, h);
    __syncwarp();
    for (uint32_t cnt = LPT / 2; cnt >= 1; cnt >>= 1) {
        uint32_t hv[8];
        if (sub < cnt) blake2s_node(hv, s + 16 * sub, s + 16 * sub + 8, one);
        __syncwarp();
        if (sub < cnt) store_hash(s + 8 * sub, hv);
        __syncwarp();
    }
    if (sub < 8 && tile < tiles) roots[8 * tile + sub] = s[sub];
}

constexpr uint32_t kTileWarp = 4;  // tiles per warp (2^26 leaves: 1 -> 5.50 ms, 2 -> 5.40, 4 -> 5.32)

// Whole small tree of n <= 2048 leaves in one block (blake2s.cu:92-189).
template <class Src>
__global__ void abi_small_tree_kernel(Src src, uint32_t *root, uint32_t n) {
    extern __shared__ uint32_t sh[];
    src.init();
    uint32_t t = threadIdx.x;
    if (2 * t + 1 < n) {
        uint32_t l[8], r[8], m[16];
        for (int w = 0; w < 16; w++) m[w] = 0u;
        uint32_t nb = src.load(2 * t, m);
        blake2s_block(l, m, nb);
        for (int w = 0; w < 16; w++) m[w] = 0u;
        nb = src.load(2 * t + 1, m);
        blake2s_block(r, m, nb);
        uint32_t h[8];
        blake2s_node(h, l, r);
        for (int w = 0; w < 8; w++) sh[8 * t + w] = h[w];
    }
    __syncthreads();
    block_reduce_hashes(sh, n / 2);
    if (t < 8) root[t] = sh[t];
}

template <class Src>
__global__ void leaf_merge_kernel(Src src, uint32_t *parents, uint64_t n_pairs, uint32_t one) {
    uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_pairs) return;
    src.init();
    uint32_t l[8], r[8], m[16];
    for (int w = 0; w < 16; w++) m[w] = 0u;
    uint32_t nb = src.load(2 * t, m);
    blake2s_block(l, m, nb, one);
    for (int w = 0; w < 16; w++) m[w] = 0u;
    nb = src.load(2 * t + 1, m);
    blake2s_block(r, m, nb, one);
    uint32_t h[8];
    blake2s_node(h, l, r, one);
    store_hash(parents + 8 * t, h);
}

// Lifted multi-size leaf (merkle_leaves_lifted.cu:33-98): the LE words of
// every column's lifted row, columns in schedule order, hashed as one
// Blake2s message (full blocks non-final while data follows; the last block
// final even when full).
struct LiftChunk {
    uint32_t col_indices[16];
    uint32_t n_cols;
    uint32_t log_size;
};
__global__ void lifted_leaves_kernel(const uint32_t *const *cols, const LiftChunk *sched, uint32_t n_chunks,
                                     uint32_t S, uint32_t *out, uint64_t n) {
    uint64_t leaf = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (leaf >= n) return;
    uint32_t total = 0;
    for (uint32_t c = 0; c < n_chunks; c++) total += sched[c].n_cols;
    uint32_t h[8];
    blake2s_init(h);
    uint32_t buf[16];
    for (int w = 0; w < 16; w++) buf[w] = 0u;
    uint32_t pos = 0, seen = 0, bytes = 0;
    for (uint32_t c = 0; c < n_chunks; c++) {
        LiftChunk ch = sched[c];
        uint32_t L = ch.log_size;
        uint64_t row = (L == S) ? leaf : (((leaf >> (S - L + 1)) << 1) | (leaf & 1ull));
        for (uint32_t i = 0; i < ch.n_cols; i++) {
            uint32_t v = cols[ch.col_indices[i]][row];
            // register-resident buffer: select the slot without dynamic indexing
#pragma unroll
            for (int w = 0; w < 16; w++) if ((uint32_t)w == pos) buf[w] = v;
            pos++;
            seen++;
            if (pos == 16 && seen < total) {
                bytes += 64;
                blake2s_compress(h, buf, bytes, false);
                pos = 0;
#pragma unroll
                for (int w = 0; w < 16; w++) buf[w] = 0u;
            }
        }
    }
    bytes += 4 * pos;
    blake2s_compress(h, buf, bytes, true);
    store_hash(out + 8 * leaf, h);
}

// ---- FRI folds with host-side alpha (fri.cu:58-126) ----
__global__ void fold_line_kernel(const uint32_t *i0, const uint32_t *i1, const uint32_t *i2, const uint32_t *i3,
                                 const uint32_t *tw, uint32_t *o0, uint32_t *o1, uint32_t *o2, uint32_t *o3, qm31 al,
                                 uint64_t half) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= half) return;
    const qmat am = qmat_of(al);
    qm31 f0{{i0[2 * i], i1[2 * i], i2[2 * i], i3[2 * i]}}, f1{{i0[2 * i + 1], i1[2 * i + 1], i2[2 * i + 1], i3[2 * i + 1]}};
    qm31 r = qadd(qadd(f0, f1), qmul_mat(am, qmulm(qsub(f0, f1), tw[i])));
    o0[i] = r.v[0]; o1[i] = r.v[1]; o2[i] = r.v[2]; o3[i] = r.v[3];
}
__global__ void fold_circle_kernel(uint32_t *d0, uint32_t *d1, uint32_t *d2, uint32_t *d3, const uint32_t *s0,
                                   const uint32_t *s1, const uint32_t *s2, const uint32_t *s3, const uint32_t *tw,
                                   qm31 al, qm31 al2, uint64_t half) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= half) return;
    const qmat am = qmat_of(al), am2 = qmat_of(al2);
    qm31 f0{{s0[2 * i], s1[2 * i], s2[2 * i], s3[2 * i]}}, f1{{s0[2 * i + 1], s1[2 * i + 1], s2[2 * i + 1], s3[2 * i + 1]}};
    qm31 fp = qadd(qadd(f0, f1), qmul_mat(am, qmulm(qsub(f0, f1), tw[i])));
    qm31 prev{{d0[i], d1[i], d2[i], d3[i]}};
    qm31 r = qadd(qmul_mat(am2, prev), fp);
    d0[i] = r.v[0]; d1[i] = r.v[1]; d2[i] = r.v[2]; d3[i] = r.v[3];
}

// Two outputs per thread: one 16-byte load per input column (pairs 2t and
// 2t + 1), 8-byte twiddle, accumulator and output accesses.  Used when every
// pointer is 16-byte (inputs) / 8-byte (the rest) aligned and half is even.
__device__ __forceinline__ qm31 fold_pair(qm31 f0, qm31 f1, const qmat &am, uint32_t t) {
    return qadd(qadd(f0, f1), qmul_mat(am, qmulm(qsub(f0, f1), t)));
}
__global__ void __launch_bounds__(256) fold_line2_kernel(const uint4 *i0, const uint4 *i1, const uint4 *i2,
                                                         const uint4 *i3, const uint2 *tw, uint2 *o0, uint2 *o1,
                                                         uint2 *o2, uint2 *o3, qm31 al, uint64_t half2) {
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= half2) return;
    const qmat am = qmat_of(al);
    const uint4 a = __ldcs(i0 + t), b = __ldcs(i1 + t), c = __ldcs(i2 + t), d = __ldcs(i3 + t);
    const uint2 w = __ldg(tw + t);
    const qm31 r0 = fold_pair(qm31{{a.x, b.x, c.x, d.x}}, qm31{{a.y, b.y, c.y, d.y}}, am, w.x);
    const qm31 r1 = fold_pair(qm31{{a.z, b.z, c.z, d.z}}, qm31{{a.w, b.w, c.w, d.w}}, am, w.y);
    o0[t] = make_uint2(r0.v[0], r1.v[0]); o1[t] = make_uint2(r0.v[1], r1.v[1]);
    o2[t] = make_uint2(r0.v[2], r1.v[2]); o3[t] = make_uint2(r0.v[3], r1.v[3]);
}
__global__ void __launch_bounds__(256) fold_circle2_kernel(uint2 *d0, uint2 *d1, uint2 *d2, uint2 *d3,
                                                           const uint4 *s0, const uint4 *s1, const uint4 *s2,
                                                           const uint4 *s3, const uint2 *tw, qm31 al, qm31 al2,
                                                           uint64_t half2) {
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= half2) return;
    const qmat am = qmat_of(al), am2 = qmat_of(al2);
    const uint4 a = __ldcs(s0 + t), b = __ldcs(s1 + t), c = __ldcs(s2 + t), d = __ldcs(s3 + t);
    const uint2 w = __ldg(tw + t);
    const uint2 p0 = d0[t], p1 = d1[t], p2 = d2[t], p3 = d3[t];
    const qm31 r0 = qadd(qmul_mat(am2, qm31{{p0.x, p1.x, p2.x, p3.x}}),
                         fold_pair(qm31{{a.x, b.x, c.x, d.x}}, qm31{{a.y, b.y, c.y, d.y}}, am, w.x));
    const qm31 r1 = qadd(qmul_mat(am2, qm31{{p0.y, p1.y, p2.y, p3.y}}),
                         fold_pair(qm31{{a.z, b.z, c.z, d.z}}, qm31{{a.w, b.w, c.w, d.w}}, am, w.y));
    d0[t] = make_uint2(r0.v[0], r1.v[0]); d1[t] = make_uint2(r0.v[1], r1.v[1]);
    d2[t] = make_uint2(r0.v[2], r1.v[2]); d3[t] = make_uint2(r0.v[3], r1.v[3]);
}
bool fold_vec_ok(const void *const *in, const void *const *rest, int n_rest, uint32_t half_n) {
    if (half_n < 2 || (half_n & 1u)) return false;
    for (int k = 0; k < 4; k++)
        if ((uintptr_t)in[k] & 15u) return false;
    for (int k = 0; k < n_rest; k++)
        if ((uintptr_t)rest[k] & 7u) return false;
    return true;
}

NttTables ref_tables(const uint32_t *line, const uint32_t *circle, const uint32_t *h_offsets, uint32_t n_line) {
    NttTables t{line, circle, {}};
    for (uint32_t l = 0; l < n_line && l < 32; l++) t.off[l] = h_offsets[l];
    return t;
}

// Reference order (circle_ntt.cu:248-312) as per-layer launches, used when
// the caller's layer count is not the full transform.
void ref_layers(uint32_t *d, const uint32_t *line, const uint32_t *circle, const uint32_t *h_off, uint32_t n_line,
                uint32_t log_n, bool forward) {
    if (forward) {
        for (int l = (int)n_line - 1; l >= 0; l--) ntt_single_layer(d, line + h_off[l], (uint32_t)l + 1, log_n, true, 0);
        ntt_single_layer(d, circle, 0, log_n, true, 0);
    } else {
        ntt_single_layer(d, circle, 0, log_n, false, 0);
        for (uint32_t l = 0; l < n_line; l++) ntt_single_layer(d, line + h_off[l], l + 1, log_n, false, 0);
    }
}

__global__ void scale_kernel(uint32_t *d, uint32_t *const *cols, uint32_t s, uint64_t n) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (cols) d = cols[blockIdx.y];
    if (i < n) d[i] = mmul(d[i], s);
}

// The batched reference order with a partial layer count (n_line line
// layers and the circle layer, then the 2^-log_n scale for the inverse), as
// the reference's batched launchers do for any n_line (circle_ntt.cu:314-404,
// circle_ntt_batch_forge.cu:95-185): per-layer launches over all columns.
cudaError_t ref_layers_cols(uint32_t *const *cols, uint32_t n_cols, const uint32_t *line, const uint32_t *circle,
                            const uint32_t *h_off, uint32_t n_line, uint32_t log_n, bool forward) {
    cudaError_t e = cudaSuccess;
    if (forward) {
        for (int l = (int)n_line - 1; l >= 0 && e == cudaSuccess; l--)
            e = ntt_single_layer_cols(cols, n_cols, line + h_off[l], (uint32_t)l + 1, log_n, true, 0);
        if (e == cudaSuccess) e = ntt_single_layer_cols(cols, n_cols, circle, 0, log_n, true, 0);
    } else {
        e = ntt_single_layer_cols(cols, n_cols, circle, 0, log_n, false, 0);
        for (uint32_t l = 0; l < n_line && e == cudaSuccess; l++)
            e = ntt_single_layer_cols(cols, n_cols, line + h_off[l], l + 1, log_n, false, 0);
        if (e == cudaSuccess) {
            const uint32_t e2 = (30u * log_n) % 31u;
            const uint64_t n = 1ull << log_n;
            scale_kernel<<<dim3(blocks_for(n, 256), n_cols), 256>>>(nullptr, cols, e2 == 0 ? 1u : (1u << e2), n);
            e = cudaGetLastError();
        }
    }
    return e;
}

}  // namespace
}  // namespace vx

using namespace vx;

extern "C" {

const char *vx_last_error(void) { return t_err.c_str(); }
void vx_clear_error(void) { t_err.clear(); }
int vx_version(void) { return 100; }

// ---------------- NTT ----------------
void cuda_circle_ntt_evaluate(uint32_t *d, const uint32_t *tw, const uint32_t *ctw, const uint32_t *h_off,
                              const uint32_t *h_sizes, uint32_t n_line, uint32_t n) {
    (void)h_sizes;
    uint32_t log_n = log2_exact(n);
    if (n_line + 1 == log_n) {
        cudaError_t e = ntt_transform(d, nullptr, 0, 1, log_n, ref_tables(tw, ctw, h_off, n_line), true, nullptr, 0, 0);
        if (e != cudaSuccess) set_last_error(VX_ERR_CUDA, "cuda_circle_ntt_evaluate: %s", cudaGetErrorString(e));
    } else {
        ref_layers(d, tw, ctw, h_off, n_line, log_n, true);
        VX_LAUNCH_CHECK();
    }
    cudaDeviceSynchronize();
}

void cuda_circle_ntt_interpolate(uint32_t *d, const uint32_t *itw, const uint32_t *ictw, const uint32_t *h_off,
                                 const uint32_t *h_sizes, uint32_t n_line, uint32_t n) {
    (void)h_sizes;
    uint32_t log_n = log2_exact(n);
    if (n_line + 1 == log_n) {
        cudaError_t e = ntt_transform(d, nullptr, 0, 1, log_n, ref_tables(itw, ictw, h_off, n_line), false, nullptr, 0, 0);
        if (e != cudaSuccess) set_last_error(VX_ERR_CUDA, "cuda_circle_ntt_interpolate: %s", cudaGetErrorString(e));
    } else {
        ref_layers(d, itw, ictw, h_off, n_line, log_n, false);
        uint32_t e2 = (30u * log_n) % 31u;
        scale_kernel<<<blocks_for(n, 256), 256>>>(d, nullptr, e2 == 0 ? 1u : (1u << e2), n);
        VX_LAUNCH_CHECK();
    }
    cudaDeviceSynchronize();
}

void cuda_circle_ntt_evaluate_batch(uint32_t **cols, const uint32_t *tw, const uint32_t *ctw, const uint32_t *h_off,
                                    const uint32_t *h_sizes, uint32_t n_line, uint32_t n, uint32_t n_cols) {
    (void)h_sizes;
    uint32_t log_n = log2_exact(n);
    if (n_cols) {
        cudaError_t e = n_line + 1 == log_n
                            ? ntt_transform(nullptr, cols, 0, n_cols, log_n, ref_tables(tw, ctw, h_off, n_line), true,
                                            nullptr, 0, 0)
                            : ref_layers_cols(cols, n_cols, tw, ctw, h_off, n_line, log_n, true);
        if (e != cudaSuccess) set_last_error(VX_ERR_CUDA, "cuda_circle_ntt_evaluate_batch: %s", cudaGetErrorString(e));
    }
    cudaDeviceSynchronize();
}

void cuda_circle_ntt_interpolate_batch(uint32_t **cols, const uint32_t *itw, const uint32_t *ictw,
                                       const uint32_t *h_off, const uint32_t *h_sizes, uint32_t n_line, uint32_t n,
                                       uint32_t n_cols) {
    (void)h_sizes;
    uint32_t log_n = log2_exact(n);
    if (n_cols) {
        cudaError_t e = n_line + 1 == log_n
                            ? ntt_transform(nullptr, cols, 0, n_cols, log_n, ref_tables(itw, ictw, h_off, n_line),
                                            false, nullptr, 0, 0)
                            : ref_layers_cols(cols, n_cols, itw, ictw, h_off, n_line, log_n, false);
        if (e != cudaSuccess) set_last_error(VX_ERR_CUDA, "cuda_circle_ntt_interpolate_batch: %s", cudaGetErrorString(e));
    }
    cudaDeviceSynchronize();
}

// The forge-feature forms (ntt.rs:191-281 with `forge-ntt-batch`, on by
// default in the reference's Cargo features): the same transforms, with
// the column pointers as a HOST array (circle_ntt_batch_forge.cu:26-39
// copies them to the device per call).  They go to a per-device device
// array kept across calls; the call is synchronous, so the lock covers its
// use.
namespace {
std::mutex g_forge_cols_mu;
uint32_t **g_forge_cols[64] = {nullptr};
uint32_t g_forge_cols_cap[64] = {0};

int forge_batch(bool fwd, uint32_t *const *col_ptrs, const uint32_t *tw, const uint32_t *ctw, const uint32_t *h_off,
                const uint32_t *h_sizes, uint32_t n_line, uint32_t n, uint32_t n_cols, const char *who) {
    if (n_cols == 0) return VX_OK;
    if (col_ptrs == nullptr) {
        set_last_error(VX_ERR_ARG, "%s: null column pointer array", who);
        return VX_ERR_ARG;
    }
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) {
        set_last_error(VX_ERR_ARG, "%s: device %d out of range", who, dev);
        return VX_ERR_ARG;
    }
    std::lock_guard<std::mutex> lk(g_forge_cols_mu);
    if (g_forge_cols_cap[dev] < n_cols) {
        if (g_forge_cols[dev]) cudaFree(g_forge_cols[dev]);
        g_forge_cols[dev] = nullptr;
        g_forge_cols_cap[dev] = 0;
        if (cudaMalloc(&g_forge_cols[dev], sizeof(uint32_t *) * n_cols) != cudaSuccess) {
            cudaGetLastError();
            set_last_error(VX_ERR_OOM, "%s: cannot allocate the column pointer array", who);
            return VX_ERR_OOM;
        }
        g_forge_cols_cap[dev] = n_cols;
    }
    if (cudaMemcpy(g_forge_cols[dev], col_ptrs, sizeof(uint32_t *) * n_cols, cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaGetLastError();
        set_last_error(VX_ERR_CUDA, "%s: pointer upload failed", who);
        return VX_ERR_CUDA;
    }
    if (fwd)
        cuda_circle_ntt_evaluate_batch(g_forge_cols[dev], tw, ctw, h_off, h_sizes, n_line, n, n_cols);
    else
        cuda_circle_ntt_interpolate_batch(g_forge_cols[dev], tw, ctw, h_off, h_sizes, n_line, n, n_cols);
    return VX_OK;
}
}  // namespace

}  // extern "C"
namespace vx {
// Frees every device's column-pointer array of the forge forms (called by
// vx_release_all; the next forge call allocates a fresh one).
void forge_cols_release() {
    std::lock_guard<std::mutex> lk(g_forge_cols_mu);
    for (int d = 0; d < 64; d++) {
        if (!g_forge_cols[d]) continue;
        int cur = 0;
        cudaGetDevice(&cur);
        if (cudaSetDevice(d) == cudaSuccess) cudaFree(g_forge_cols[d]);
        cudaSetDevice(cur);
        cudaGetLastError();
        g_forge_cols[d] = nullptr;
        g_forge_cols_cap[d] = 0;
    }
}
}  // namespace vx
extern "C" {

void cuda_circle_ntt_evaluate_batch_forge(uint32_t *const *col_ptrs, const uint32_t *tw, const uint32_t *ctw,
                                          const uint32_t *h_off, const uint32_t *h_sizes, uint32_t n_line, uint32_t n,
                                          uint32_t n_cols) {
    forge_batch(true, col_ptrs, tw, ctw, h_off, h_sizes, n_line, n, n_cols, "cuda_circle_ntt_evaluate_batch_forge");
}

void cuda_circle_ntt_interpolate_batch_forge(uint32_t *const *col_ptrs, const uint32_t *itw, const uint32_t *ictw,
                                             const uint32_t *h_off, const uint32_t *h_sizes, uint32_t n_line,
                                             uint32_t n, uint32_t n_cols) {
    forge_batch(false, col_ptrs, itw, ictw, h_off, h_sizes, n_line, n, n_cols,
                "cuda_circle_ntt_interpolate_batch_forge");
}

void cuda_circle_ntt_layer(uint32_t *d, const uint32_t *tw, uint32_t layer_idx, uint32_t n, int forward) {
    ntt_single_layer(d, tw, layer_idx, log2_exact(n), forward != 0, 0);
    VX_LAUNCH_CHECK();
}

// circle_ntt_layer_forge (blake2s_m31.rs): the same layer.
void cuda_circle_ntt_layer_forge(uint32_t *d, const uint32_t *tw, uint32_t layer_idx, uint32_t n, int forward) {
    cuda_circle_ntt_layer(d, tw, layer_idx, n, forward);
}

void cuda_bit_reverse_m31(uint32_t *data, uint32_t log_n) {
    uint64_t n = 1ull << log_n;
    if (log_n >= 2 * kBrevT6 && log_n <= 31 && ((uintptr_t)data & 7u) == 0)
        bit_reverse_tiled64_kernel<<<1u << (log_n - 2 * kBrevT6), 256>>>(data, log_n);
    else if (log_n >= 2 * kBrevT && log_n <= 31)
        bit_reverse_tiled_kernel<<<1u << (log_n - 2 * kBrevT), 256>>>(data, log_n);
    else
        bit_reverse_kernel<<<blocks_for(n, 256), 256>>>(data, log_n, n);
    VX_LAUNCH_CHECK();
}

void cuda_permute_hc_to_canonic_brt(const uint32_t *src, uint32_t *dst, uint32_t n, uint32_t log_n) {
    if (permute_tiled_ok(src, dst, n, log_n))
        permute_tiled_kernel<<<1u << (log_n - 2 - 2 * kBrevT), 256>>>((const uint2 *)src, (uint2 *)dst, log_n);
    else
        permute_kernel<<<blocks_for(n, 256), 256>>>(src, dst, n, log_n, 0);
    VX_LAUNCH_CHECK();
}

void cuda_permute_canonic_brt_to_hc_natural(const uint32_t *src, uint32_t *dst, uint32_t n, uint32_t log_n) {
    if (permute_tiled_ok(src, dst, n, log_n))
        permute_tiled_kernel<<<1u << (log_n - 2 - 2 * kBrevT), 256>>>((const uint2 *)src, (uint2 *)dst, log_n);
    else
        permute_kernel<<<blocks_for(n, 256), 256>>>(src, dst, n, log_n, 1);
    VX_LAUNCH_CHECK();
}

// ---------------- twiddles ----------------
void cuda_compute_coset_points(uint32_t ix, uint32_t iy, uint32_t sx, uint32_t sy, uint32_t *xs, uint32_t *ys,
                               uint32_t n) {
    uint64_t thr = (n + 15ull) / 16ull;
    coset_points_kernel<<<blocks_for(thr, 256), 256>>>(cpoint{ix, iy}, cpoint{sx, sy}, xs, ys, n);
    VX_LAUNCH_CHECK();
}

void cuda_squash_x(const uint32_t *in, uint32_t *out, uint32_t out_n) {
    extract_squash_kernel<<<blocks_for(out_n, 256), 256>>>(in, nullptr, out, out_n);
    VX_LAUNCH_CHECK();
}

void cuda_extract_and_squash(const uint32_t *in, uint32_t *tw_out, uint32_t *sq_out, uint32_t half_n) {
    extract_squash_kernel<<<blocks_for(half_n, 256), 256>>>(in, tw_out, sq_out, half_n);
    VX_LAUNCH_CHECK();
}

void cuda_batch_inverse_m31(const uint32_t *in, uint32_t *out, uint32_t n) {
    cudaError_t e = batch_inverse(in, out, n, 0);
    if (e != cudaSuccess) set_last_error(VX_ERR_CUDA, "cuda_batch_inverse_m31: %s", cudaGetErrorString(e));
}

// batch_inverse_forge.cu:1-20: the same chunk-of-64 prefix-product inverse.
void cuda_batch_inverse_m31_forge(const uint32_t *in, uint32_t *out, uint32_t n) { cuda_batch_inverse_m31(in, out, n); }

void cuda_batch_inverse_m31_stream(const uint32_t *in, uint32_t *out, uint32_t n, void *stream) {
    cudaError_t e = batch_inverse(in, out, n, (cudaStream_t)stream);
    if (e != cudaSuccess) set_last_error(VX_ERR_CUDA, "cuda_batch_inverse_m31_stream: %s", cudaGetErrorString(e));
}

void cuda_compute_fold_twiddle_sources_stream(uint32_t ix, uint32_t iy, uint32_t sx, uint32_t sy, uint32_t *out,
                                              uint32_t n, uint32_t log_n, int extract_y, void *stream) {
    uint64_t half = n / 2;
    fold_sources_generic_kernel<<<blocks_for(half, 256), 256, 0, (cudaStream_t)stream>>>(cpoint{ix, iy}, cpoint{sx, sy},
                                                                                        out, half, log_n, extract_y);
    VX_LAUNCH_CHECK();
}

void cuda_compute_fold_twiddle_sources(uint32_t ix, uint32_t iy, uint32_t sx, uint32_t sy, uint32_t *out, uint32_t n,
                                       uint32_t log_n, int extract_y) {
    cuda_compute_fold_twiddle_sources_stream(ix, iy, sx, sy, out, n, log_n, extract_y, nullptr);
}

// ---------------- glue ----------------
void cuda_zero_pad(const uint32_t *src, uint32_t *dst, uint32_t src_n, uint32_t dst_n) {
    if ((((uintptr_t)src | (uintptr_t)dst) & 15u) == 0)
        zero_pad_kernel<true><<<blocks_for(((uint64_t)dst_n + 3) / 4, 256), 256>>>(src, dst, src_n, dst_n);
    else
        zero_pad_kernel<false><<<blocks_for(dst_n, 256), 256>>>(src, dst, src_n, dst_n);
    VX_LAUNCH_CHECK();
}

void cuda_fibonacci_quotient_chunk_stream(const uint32_t *tr, uint32_t *o0, uint32_t *o1, uint32_t *o2, uint32_t *o3,
                                          const uint32_t *al, uint32_t offset, uint32_t chunk_n, uint32_t global_n,
                                          void *stream) {
    if (chunk_n == 0) return;
    const cudaStream_t st = (cudaStream_t)stream;
    const bool vec = ((((uintptr_t)tr | (uintptr_t)o0 | (uintptr_t)o1 | (uintptr_t)o2 | (uintptr_t)o3) & 15u) == 0) &&
                     offset % 4u == 0 && chunk_n % 4u == 0 && global_n > 2;
    if (vec)
        quotient_kernel<true><<<blocks_for(chunk_n / 4u, 256), 256, 0, st>>>(tr, o0, o1, o2, o3, al[0], al[1], al[2],
                                                                           al[3], offset, chunk_n, global_n);
    else
        quotient_kernel<false><<<blocks_for(chunk_n, 256), 256, 0, st>>>(tr, o0, o1, o2, o3, al[0], al[1], al[2],
                                                                        al[3], offset, chunk_n, global_n);
    VX_LAUNCH_CHECK();
}

void cuda_fibonacci_quotient_chunk(const uint32_t *tr, uint32_t *o0, uint32_t *o1, uint32_t *o2, uint32_t *o3,
                                   const uint32_t *al, uint32_t offset, uint32_t chunk_n, uint32_t global_n) {
    cuda_fibonacci_quotient_chunk_stream(tr, o0, o1, o2, o3, al, offset, chunk_n, global_n, nullptr);
}

void cuda_fibonacci_quotient(const uint32_t *tr, uint32_t *o0, uint32_t *o1, uint32_t *o2, uint32_t *o3,
                             const uint32_t *al, uint32_t n) {
    cuda_fibonacci_quotient_chunk_stream(tr, o0, o1, o2, o3, al, 0, n, n, nullptr);
}

// ---------------- Merkle ----------------
void cuda_merkle_hash_leaves(const uint32_t *const *cols, uint32_t *hashes, uint32_t n_cols, uint32_t n_leaves) {
    const unsigned lb = (unsigned)blocks_for(n_leaves, 128);
    switch (n_cols) {
    case 1: leaf_hash_kernel<<<lb, 128>>>(LeafColsN<1>{cols, {}}, hashes, n_leaves, 1u); break;
    case 2: leaf_hash_kernel<<<lb, 128>>>(LeafColsN<2>{cols, {}}, hashes, n_leaves, 1u); break;
    case 4: leaf_hash_kernel<<<lb, 128>>>(LeafColsN<4>{cols, {}}, hashes, n_leaves, 1u); break;
    case 8: leaf_hash_kernel<<<lb, 128>>>(LeafColsN<8>{cols, {}}, hashes, n_leaves, 1u); break;
    default: leaf_hash_kernel<<<lb, 128>>>(LeafCols{cols, n_cols}, hashes, n_leaves, 1u); break;
    }
    VX_LAUNCH_CHECK();
}

void cuda_merkle_hash_leaves_forge_single(const uint32_t *col, uint32_t *hashes, uint32_t n_leaves) {
    leaf_hash_kernel<<<blocks_for(n_leaves, 128), 128>>>(LeafM31{col}, hashes, n_leaves, 1u);
    VX_LAUNCH_CHECK();
}

void cuda_merkle_hash_leaves_forge_quad(const uint32_t *c0, const uint32_t *c1, const uint32_t *c2,
                                        const uint32_t *c3, uint32_t *hashes, uint32_t n_leaves) {
    leaf_hash_kernel<<<blocks_for(n_leaves, 128), 128>>>(LeafSoA4{c0, c1, c2, c3}, hashes, n_leaves, 1u);
    VX_LAUNCH_CHECK();
}

void cuda_merkle_hash_nodes(const uint32_t *children, uint32_t *parents, uint32_t n_parents) {
    node_hash_kernel<<<blocks_for(n_parents, 128), 128>>>(children, parents, n_parents, 1u);
    VX_LAUNCH_CHECK();
}

void cuda_merkle_reduce_to_root(const uint32_t *nodes, uint32_t *root, uint32_t n) {
    if (n == 0 || n > 1024) { set_last_error(VX_ERR_ARG, "cuda_merkle_reduce_to_root: n_nodes must be in [1, 1024]"); return; }
    uint32_t thr = n / 2 < 32 ? 32 : n / 2;
    reduce_to_root_kernel<<<1, thr, 32 * n>>>(nodes, root, n);
    VX_LAUNCH_CHECK();
}

void cuda_merkle_commit_small_soa4(const uint32_t *c0, const uint32_t *c1, const uint32_t *c2, const uint32_t *c3,
                                   uint32_t *root, uint32_t n_leaves) {
    if (n_leaves < 2 || n_leaves > 2048) { set_last_error(VX_ERR_ARG, "cuda_merkle_commit_small_soa4: n_leaves must be in [2, 2048]"); return; }
    uint32_t thr = n_leaves / 2 < 32 ? 32 : n_leaves / 2;
    abi_small_tree_kernel<<<1, thr, 16 * n_leaves>>>(LeafSoA4{c0, c1, c2, c3}, root, n_leaves);
    VX_LAUNCH_CHECK();
}

void cuda_merkle_hash_leaves_merge_soa4(const uint32_t *c0, const uint32_t *c1, const uint32_t *c2,
                                        const uint32_t *c3, uint32_t *parents, uint32_t n_leaves) {
    uint64_t pairs = n_leaves / 2;
    leaf_merge_kernel<<<blocks_for(pairs, 128), 128>>>(LeafSoA4{c0, c1, c2, c3}, parents, pairs, 1u);
    VX_LAUNCH_CHECK();
}

void cuda_merkle_tiled_soa4_stream(const uint32_t *c0, const uint32_t *c1, const uint32_t *c2, const uint32_t *c3,
                                   uint32_t *roots, uint32_t n_leaves, void *stream) {
    uint32_t tiles = n_leaves / 1024u;
    if (!tiles) return;
    tile_root_warp_kernel<kTileWarp><<<(tiles + 4 * kTileWarp - 1) / (4 * kTileWarp), 128, 0, (cudaStream_t)stream>>>(LeafSoA4{c0, c1, c2, c3}, roots, tiles, 1u);
    VX_LAUNCH_CHECK();
}

void cuda_merkle_tiled_soa4(const uint32_t *c0, const uint32_t *c1, const uint32_t *c2, const uint32_t *c3,
                            uint32_t *roots, uint32_t n_leaves) {
    cuda_merkle_tiled_soa4_stream(c0, c1, c2, c3, roots, n_leaves, nullptr);
}

void cuda_merkle_tiled_generic(const uint32_t *const *cols, uint32_t *roots, uint32_t n_cols, uint32_t n_leaves) {
    uint32_t tiles = n_leaves / 1024u;
    if (!tiles) return;
    switch (n_cols) {  // common column counts with compile-time zero message words
    case 1: tile_root_warp_kernel<kTileWarp><<<(tiles + 4 * kTileWarp - 1) / (4 * kTileWarp), 128, 0>>>(LeafColsN<1>{cols, {}}, roots, tiles, 1u); break;
    case 2: tile_root_warp_kernel<kTileWarp><<<(tiles + 4 * kTileWarp - 1) / (4 * kTileWarp), 128, 0>>>(LeafColsN<2>{cols, {}}, roots, tiles, 1u); break;
    case 4: tile_root_warp_kernel<kTileWarp><<<(tiles + 4 * kTileWarp - 1) / (4 * kTileWarp), 128, 0>>>(LeafColsN<4>{cols, {}}, roots, tiles, 1u); break;
    case 8: tile_root_warp_kernel<kTileWarp><<<(tiles + 4 * kTileWarp - 1) / (4 * kTileWarp), 128, 0>>>(LeafColsN<8>{cols, {}}, roots, tiles, 1u); break;
    default: tile_root_warp_kernel<kTileWarp><<<(tiles + 4 * kTileWarp - 1) / (4 * kTileWarp), 128, 0>>>(LeafCols{cols, n_cols}, roots, tiles, 1u); break;
    }
    VX_LAUNCH_CHECK();
}

void cuda_build_leaves_lifted(const uint32_t *const *cols, const void *schedule, uint32_t n_chunks, uint32_t S,
                              uint32_t *out, uint32_t n_leaves) {
    lifted_leaves_kernel<<<blocks_for(n_leaves, 128), 128>>>(cols, (const LiftChunk *)schedule, n_chunks, S, out,
                                                             n_leaves);
    VX_LAUNCH_CHECK();
}

// ---------------- FRI ----------------
void cuda_fold_line_soa(const uint32_t *i0, const uint32_t *i1, const uint32_t *i2, const uint32_t *i3,
                        const uint32_t *tw, uint32_t *o0, uint32_t *o1, uint32_t *o2, uint32_t *o3,
                        const uint32_t *alpha, uint32_t half_n) {
    qm31 al{{alpha[0], alpha[1], alpha[2], alpha[3]}};
    const void *in[4] = {i0, i1, i2, i3}, *rest[5] = {tw, o0, o1, o2, o3};
    if (fold_vec_ok(in, rest, 5, half_n))
        fold_line2_kernel<<<blocks_for(half_n / 2, 256), 256>>>((const uint4 *)i0, (const uint4 *)i1,
                                                                (const uint4 *)i2, (const uint4 *)i3,
                                                                (const uint2 *)tw, (uint2 *)o0, (uint2 *)o1,
                                                                (uint2 *)o2, (uint2 *)o3, al, half_n / 2);
    else
        fold_line_kernel<<<blocks_for(half_n, 256), 256>>>(i0, i1, i2, i3, tw, o0, o1, o2, o3, al, half_n);
    VX_LAUNCH_CHECK();
}

void cuda_fold_circle_into_line_soa(uint32_t *d0, uint32_t *d1, uint32_t *d2, uint32_t *d3, const uint32_t *s0,
                                    const uint32_t *s1, const uint32_t *s2, const uint32_t *s3, const uint32_t *tw,
                                    const uint32_t *alpha, const uint32_t *alpha_sq, uint32_t half_n) {
    qm31 al{{alpha[0], alpha[1], alpha[2], alpha[3]}}, al2{{alpha_sq[0], alpha_sq[1], alpha_sq[2], alpha_sq[3]}};
    const void *in[4] = {s0, s1, s2, s3}, *rest[5] = {tw, d0, d1, d2, d3};
    if (fold_vec_ok(in, rest, 5, half_n))
        fold_circle2_kernel<<<blocks_for(half_n / 2, 256), 256>>>((uint2 *)d0, (uint2 *)d1, (uint2 *)d2,
                                                                  (uint2 *)d3, (const uint4 *)s0, (const uint4 *)s1,
                                                                  (const uint4 *)s2, (const uint4 *)s3,
                                                                  (const uint2 *)tw, al, al2, half_n / 2);
    else
        fold_circle_kernel<<<blocks_for(half_n, 256), 256>>>(d0, d1, d2, d3, s0, s1, s2, s3, tw, al, al2, half_n);
    VX_LAUNCH_CHECK();
}

void cuda_fold_line_soa_forge(const uint32_t *i0, const uint32_t *i1, const uint32_t *i2, const uint32_t *i3,
                              const uint32_t *tw, uint32_t *o0, uint32_t *o1, uint32_t *o2, uint32_t *o3,
                              const uint32_t *alpha, uint32_t half_n) {
    cuda_fold_line_soa(i0, i1, i2, i3, tw, o0, o1, o2, o3, alpha, half_n);
}

void cuda_fold_circle_into_line_soa_forge(uint32_t *d0, uint32_t *d1, uint32_t *d2, uint32_t *d3, const uint32_t *s0,
                                          const uint32_t *s1, const uint32_t *s2, const uint32_t *s3,
                                          const uint32_t *tw, const uint32_t *alpha, const uint32_t *alpha_sq,
                                          uint32_t half_n) {
    cuda_fold_circle_into_line_soa(d0, d1, d2, d3, s0, s1, s2, s3, tw, alpha, alpha_sq, half_n);
}

void cuda_device_sync(void) { cudaDeviceSynchronize(); }

}  // extern "C"
