// Blake2s Merkle trees for sm_100a.
//
// Tree shape (merkle.rs:28-130): a binary tree over leaves in natural index
// order; leaf = Blake2s(LE words of the row) with t = 4 * words, node =
// Blake2s(left || right) with t = 64 (blake2s.cu:13-87).
//
// Work split: one thread hashes 2^kl consecutive leaves and folds them into
// their subtree root with a small stack, so every lane stays busy and no data
// moves between threads (kl = 4: 16 leaf + 15 node compressions per thread).
// Upper levels are reduced the same way, 2^k hashes per thread.  The
// resulting hash arrays at levels kl, kl + 4, ... are kept: they are the
// tree's stored levels, from which any authentication path is rebuilt by
// re-hashing one 16-node block per stored level.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "vx_blake2s.cuh"
#include "vx_field.cuh"

namespace vx {

// ---- leaf sources: fill m[] (pre-zeroed) and return the byte length ----
struct LeafM31 {
    const uint32_t *col;
    __device__ __forceinline__ void init() {}
    __device__ __forceinline__ uint32_t load(uint64_t i, uint32_t m[16]) const { m[0] = __ldg(col + i); return 4u; }
};
struct LeafSoA4 {
    const uint32_t *c0, *c1, *c2, *c3;
    __device__ __forceinline__ void init() {}
    __device__ __forceinline__ uint32_t load(uint64_t i, uint32_t m[16]) const {
        m[0] = __ldg(c0 + i); m[1] = __ldg(c1 + i); m[2] = __ldg(c2 + i); m[3] = __ldg(c3 + i);
        return 16u;
    }
};
// Up to 16 columns from a device array of column pointers; only the first
// min(n_cols, 16) are hashed and t = 4 * min(n_cols, 16) (blake2s.cu:25-53).
struct LeafCols {
    const uint32_t *const *cols;
    uint32_t n_cols;
    __device__ __forceinline__ void init() {}
    __device__ __forceinline__ uint32_t load(uint64_t i, uint32_t m[16]) const {
        uint32_t n = n_cols > 16u ? 16u : n_cols;
#pragma unroll
        for (uint32_t c = 0; c < 16; c++) if (c < n) m[c] = cols[c][i];
        return 4u * n;
    }
};
// Fibonacci quotient recomputed from the trace evaluation:
// q[i] = alpha * (t[i+2] - (t[i+1] + t[i]))  (constraint.cu:10-33), i mod N.
struct LeafQuotient {
    const uint32_t *eval;
    uint64_t mask;
    const uint32_t *alpha_ptr;
    uint32_t al[4];
    __device__ __forceinline__ void init() {
#pragma unroll
        for (int c = 0; c < 4; c++) al[c] = alpha_ptr[c];
    }
    __device__ __forceinline__ qm31 value(uint64_t i) const {
        uint32_t t0 = __ldg(eval + i), t1 = __ldg(eval + ((i + 1) & mask)), t2 = __ldg(eval + ((i + 2) & mask));
        uint32_t c = msub(t2, madd(t1, t0));
        return {{mmul(al[0], c), mmul(al[1], c), mmul(al[2], c), mmul(al[3], c)}};
    }
    __device__ __forceinline__ uint32_t load(uint64_t i, uint32_t m[16]) const {
        qm31 q = value(i);
        m[0] = q.v[0]; m[1] = q.v[1]; m[2] = q.v[2]; m[3] = q.v[3];
        return 16u;
    }
};

// Fold a subtree of 2^kl leaves starting at `base` into its root.
template <class Src>
__device__ __forceinline__ void subtree_root(const Src &src, uint64_t base, uint32_t kl, uint32_t root[8]) {
    uint32_t stk[5][8];
    uint32_t sp = 0;
    const uint32_t K = 1u << kl;
    for (uint32_t j = 0; j < K; j++) {
        uint32_t m[16];
#pragma unroll
        for (int w = 0; w < 16; w++) m[w] = 0u;
        uint32_t nb = src.load(base + j, m);
        uint32_t h[8];
        blake2s_block(h, m, nb);
        for (uint32_t jj = j; jj & 1u; jj >>= 1) {
            --sp;
            uint32_t mm[16];
#pragma unroll
            for (int w = 0; w < 8; w++) { mm[w] = stk[sp][w]; mm[8 + w] = h[w]; }
            blake2s_block(h, mm, 64u);
        }
#pragma unroll
        for (int w = 0; w < 8; w++) stk[sp][w] = h[w];
        ++sp;
    }
#pragma unroll
    for (int w = 0; w < 8; w++) root[w] = stk[0][w];
}

// Reduce 2^k consecutive 8-word hashes starting at hashes + 8*base.
__device__ __forceinline__ void node_subtree_root(const uint32_t *hashes, uint64_t base, uint32_t k, uint32_t root[8]) {
    uint32_t stk[5][8];
    uint32_t sp = 0;
    const uint32_t K = 1u << k;
    for (uint32_t j = 0; j < K; j++) {
        uint32_t h[8];
        const uint4 *p = (const uint4 *)(hashes + 8ull * (base + j));
        uint4 a = p[0], b = p[1];
        h[0] = a.x; h[1] = a.y; h[2] = a.z; h[3] = a.w; h[4] = b.x; h[5] = b.y; h[6] = b.z; h[7] = b.w;
        for (uint32_t jj = j; jj & 1u; jj >>= 1) {
            --sp;
            uint32_t mm[16];
#pragma unroll
            for (int w = 0; w < 8; w++) { mm[w] = stk[sp][w]; mm[8 + w] = h[w]; }
            blake2s_block(h, mm, 64u);
        }
#pragma unroll
        for (int w = 0; w < 8; w++) stk[sp][w] = h[w];
        ++sp;
    }
#pragma unroll
    for (int w = 0; w < 8; w++) root[w] = stk[0][w];
}

__device__ __forceinline__ void store_hash(uint32_t *dst, const uint32_t h[8]) {
    uint4 *p = (uint4 *)dst;
    p[0] = make_uint4(h[0], h[1], h[2], h[3]);
    p[1] = make_uint4(h[4], h[5], h[6], h[7]);
}

template <class Src>
__global__ void __launch_bounds__(256) leaf_subtree_kernel(Src src, uint32_t *out, uint64_t n_threads, uint32_t kl) {
    uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_threads) return;
    src.init();
    uint32_t h[8];
    subtree_root(src, t << kl, kl, h);
    store_hash(out + 8ull * t, h);
}

__global__ void node_subtree_kernel(const uint32_t *in, uint32_t *out, uint64_t n_threads, uint32_t k);

// Stored levels of one tree: level[0] is the leaf data (via its source),
// level[i] (i >= 1) an array of hashes at tree height h[i]; h[n-1] = depth
// holds the root.
struct TreeLevels {
    uint32_t n;            // number of stored levels including the leaf level
    uint32_t height[12];   // height of each stored level (height[0] = 0)
    uint32_t *hashes[12];  // hashes[0] unused
};

// Plan the stored levels of a tree of 2^depth leaves inside `pool`
// (words); returns words used.
uint64_t tree_plan(uint32_t depth, uint32_t *pool, TreeLevels *lv);
uint64_t tree_pool_words(uint32_t depth);

// Build all stored levels: leaf kernel then node kernels (no host sync).
template <class Src>
cudaError_t tree_build(const Src &src, const TreeLevels &lv, cudaStream_t stream) {
    if (lv.n < 2) return cudaSuccess;
    uint32_t kl = lv.height[1];
    uint64_t n1 = 1ull << (lv.height[lv.n - 1] - kl);
    leaf_subtree_kernel<Src><<<(unsigned)((n1 + 255) / 256), 256, 0, stream>>>(src, lv.hashes[1], n1, kl);
    for (uint32_t i = 2; i < lv.n; i++) {
        uint32_t k = lv.height[i] - lv.height[i - 1];
        uint64_t nt = 1ull << (lv.height[lv.n - 1] - lv.height[i]);
        node_subtree_kernel<<<(unsigned)((nt + 255) / 256), 256, 0, stream>>>(lv.hashes[i - 1], lv.hashes[i], nt, k);
    }
    return cudaGetLastError();
}

// Authentication paths, written straight into a proof in the reference's
// byte layout (stark_cli.rs:1060-1090): for each query q, the path of
// index[q] at paths + q*(1+8*depth) (depth word then siblings leaf->root)
// and the path of index[q]^1 at spaths + q*(1+8*depth).
template <class Src>
__global__ void decommit_paths_kernel(Src src, TreeLevels lv, const uint32_t *qidx, uint32_t shift, uint32_t nq,
                                      uint32_t *paths, uint32_t *spaths) {
    uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t ng = lv.n - 1;
    if (tid >= nq * ng) return;
    uint32_t q = tid / ng, g = tid % ng;
    uint32_t depth = lv.height[lv.n - 1];
    uint64_t idx = (uint64_t)qidx[q] >> shift;
    uint32_t lo = lv.height[g], k = lv.height[g + 1] - lo;
    uint64_t node = idx >> lo;              // node index at height lo
    uint64_t blk = node >> k;               // block of 2^k nodes
    // all hashes of the block, level by level (16 + 8 + 4 + 2 + 1 max)
    uint32_t nh[31][8];
    const uint32_t K = 1u << k;
    if (g == 0) {
        src.init();
        for (uint32_t j = 0; j < K; j++) {
            uint32_t m[16];
#pragma unroll
            for (int w = 0; w < 16; w++) m[w] = 0u;
            uint32_t nb = src.load((blk << k) + j, m);
            blake2s_block(nh[j], m, nb);
        }
    } else {
        const uint32_t *h = lv.hashes[g] + 8ull * (blk << k);
        for (uint32_t j = 0; j < K; j++)
#pragma unroll
            for (int w = 0; w < 8; w++) nh[j][w] = h[8 * j + w];
    }
    uint32_t lvl_off = 0, cnt = K;
    for (uint32_t d = 0; d < k; d++) {
        uint32_t nxt = lvl_off + cnt;
        for (uint32_t j = 0; j < cnt / 2; j++) blake2s_node(nh[nxt + j], nh[lvl_off + 2 * j], nh[lvl_off + 2 * j + 1]);
        lvl_off = nxt;
        cnt /= 2;
    }
    uint32_t *p = paths + (uint64_t)q * (1u + 8u * depth);
    uint32_t *sp = spaths + (uint64_t)q * (1u + 8u * depth);
    lvl_off = 0; cnt = K;
    uint64_t local = node & (K - 1u);
    for (uint32_t d = 0; d < k; d++) {
        uint32_t hgt = lo + d;
        const uint32_t *sib = nh[lvl_off + (uint32_t)(local ^ 1u)];
        const uint32_t *self = nh[lvl_off + (uint32_t)local];
#pragma unroll
        for (int w = 0; w < 8; w++) {
            p[1 + 8 * hgt + w] = sib[w];
            sp[1 + 8 * hgt + w] = (hgt == 0) ? self[w] : sib[w];
        }
        lvl_off += cnt; cnt /= 2; local >>= 1;
    }
    if (g == 0) { p[0] = depth; sp[0] = depth; }
}

}  // namespace vx
