// Blake2s Merkle trees for sm_100a.
//
// Tree shape (merkle.rs:28-130): a binary tree over leaves in natural index
// order; leaf = Blake2s(LE words of the row) with t = 4 * words, node =
// Blake2s(left || right) with t = 64 (blake2s.cu:13-87).
//
// Work split: one thread hashes 2^kl consecutive leaves and folds them into
// their subtree root with a small stack, so every lane stays busy and no data
// moves between threads (kl = 4: 16 leaf + 15 node compressions per thread).
// Big middle levels are reduced the same way, 16 hashes per thread; the
// levels above, where one compression per thread per level is what keeps the
// chain short, by blocks in shared memory (see TreeLevels).  The hash arrays
// at the planned heights are kept: they are the tree's stored levels, from
// which any authentication path is rebuilt by re-hashing one block of at most
// 16 nodes per stored level.
#pragma once
#include <cstdint>
#include <type_traits>
#include <cuda_runtime.h>

#include "vx_blake2s.cuh"
#include "vx_common.cuh"
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
    const uint32_t *c0;  // the first column pointer, read once by init()
    __device__ __forceinline__ void init() { c0 = n_cols ? cols[0] : nullptr; }
    __device__ __forceinline__ uint32_t load(uint64_t i, uint32_t m[16]) const {
        if (n_cols == 1) {  // one column: no pointer reads per leaf
            m[0] = __ldg(c0 + i);
            return 4u;
        }
        uint32_t n = n_cols > 16u ? 16u : n_cols;
#pragma unroll
        for (uint32_t c = 0; c < 16; c++) if (c < n) m[c] = cols[c][i];
        return 4u * n;
    }
};
// The same with the column count fixed at compile time: the message words
// past the N loaded ones are known zeros, whose additions the compression
// drops (a one-column leaf then costs what LeafM31's does).
template <uint32_t N>
struct LeafColsN {
    const uint32_t *const *cols;
    const uint32_t *p[N];  // the column pointers, read once by init()
    __device__ __forceinline__ void init() {
#pragma unroll
        for (uint32_t c = 0; c < N; c++) p[c] = cols[c];
    }
    __device__ __forceinline__ uint32_t load(uint64_t i, uint32_t m[16]) const {
#pragma unroll
        for (uint32_t c = 0; c < N; c++) m[c] = __ldg(p[c] + i);
        return 4u * N;
    }
};
// Up to 16 columns passed by value (host-side pointer list); t = 4 * n.
struct LeafColsV {
    const uint32_t *col[16];
    uint32_t n;
    __device__ __forceinline__ void init() {}
    __device__ __forceinline__ uint32_t load(uint64_t i, uint32_t m[16]) const {
#pragma unroll
        for (uint32_t c = 0; c < 16; c++) if (c < n) m[c] = __ldg(col[c] + i);
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

// A leaf source either fills one message block (load: m[] pre-zeroed, returns
// the byte length) or, when its message spans several blocks, hashes the
// leaf itself (digest).
template <class Src, class = void>
struct is_wide_leaf : std::false_type {};
template <class Src>
struct is_wide_leaf<Src, std::void_t<decltype(&Src::digest)>> : std::true_type {};

// Leaf sources whose load is itself multiply-heavy (the FMA pipe is busy)
// declare `static constexpr bool kPlainAdds = true`; the kernels that hash
// their leaves (and the nodes above them) then use the plain three-input add.
template <class Src, class = void>
struct plain_adds : std::false_type {};
template <class Src>
struct plain_adds<Src, std::void_t<decltype(Src::kPlainAdds)>> : std::bool_constant<Src::kPlainAdds> {};

template <class Src>
__device__ __forceinline__ void leaf_digest(const Src &src, uint64_t i, uint32_t h[8], uint32_t one = 1u) {
    if constexpr (plain_adds<Src>::value) one = 1u;
    if constexpr (is_wide_leaf<Src>::value) {
        src.digest(i, h, one);
    } else {
        uint32_t m[16];
#pragma unroll
        for (int w = 0; w < 16; w++) m[w] = 0u;
        uint32_t nb = src.load(i, m);
        blake2s_block(h, m, nb, one);
    }
}

// Lifted multi-size leaf (merkle_leaves_lifted.cu:25-98): the row of every
// column, columns in ascending size, column c of 2^L rows read at
// ((idx >> (S - L + 1)) << 1) | (idx & 1) (idx itself when L = S); one
// Blake2s over all n_cols words, every full block but the last compressed
// as non-final.
constexpr uint32_t kMaxLiftCols = 64;
struct LeafLifted {
    const uint32_t *col[kMaxLiftCols];
    uint32_t shift[kMaxLiftCols];  // S - L + 1 (1 when L = S, where the formula gives the index itself)
    uint32_t n_cols;
    __device__ __forceinline__ void init() {}
    // Row of column c for tree index idx < 2^S <= 2^31 (32-bit arithmetic).
    __device__ __forceinline__ uint32_t word(uint32_t c, uint64_t idx) const {
        const uint32_t i = (uint32_t)idx, sh = shift[c];
        return __ldg(col[c] + (((i >> sh) << 1) | (i & 1u)));
    }
    __device__ __forceinline__ void digest(uint64_t idx, uint32_t h[8], uint32_t one = 1u) const {
        blake2s_init(h);
        const uint32_t nblk = n_cols ? (n_cols + 15u) / 16u : 1u;
        for (uint32_t b = 0; b < nblk; b++) {
            uint32_t m[16];
#pragma unroll
            for (uint32_t w = 0; w < 16; w++) {
                const uint32_t c = 16u * b + w;
                m[w] = c < n_cols ? word(c, idx) : 0u;
            }
            const bool last = b + 1 == nblk;
            blake2s_compress(h, m, last ? 4u * n_cols : 64u * (b + 1), last, one);
        }
    }
};

// The same leaf with the number of words in the last message block fixed at
// compile time (WL = n_cols - 16 (blocks - 1), 1..16): full blocks load their
// 16 words without per-word bounds, and the zero words past WL fold out of
// the last compression.  Same digests as LeafLifted.
template <uint32_t WL>
struct LeafLiftedW : LeafLifted {
    __device__ __forceinline__ void digest(uint64_t idx, uint32_t h[8], uint32_t one = 1u) const {
        blake2s_init(h);
        const uint32_t nfull = (n_cols - WL) / 16u;
        for (uint32_t b = 0; b < nfull; b++) {
            uint32_t m[16];
#pragma unroll
            for (uint32_t w = 0; w < 16; w++) m[w] = word(16u * b + w, idx);
            blake2s_compress(h, m, 64u * (b + 1), false, one);
        }
        uint32_t m[16];
#pragma unroll
        for (uint32_t w = 0; w < 16; w++) m[w] = w < WL ? word(16u * nfull + w, idx) : 0u;
        blake2s_compress(h, m, 4u * n_cols, true, one);
    }
};

// Fold a subtree of 2^kl leaves (kl <= KMAX) starting at `base` into its root.
template <class Src, uint32_t KMAX = 5>
__device__ __forceinline__ void subtree_root(const Src &src, uint64_t base, uint32_t kl, uint32_t root[8],
                                             uint32_t one = 1u) {
    uint32_t stk[KMAX][8];
    uint32_t sp = 0;
    const uint32_t K = 1u << kl;
    for (uint32_t j = 0; j < K; j++) {
        uint32_t h[8];
        leaf_digest(src, base + j, h, one);
        for (uint32_t jj = j; jj & 1u; jj >>= 1) {
            --sp;
            uint32_t mm[16];
#pragma unroll
            for (int w = 0; w < 8; w++) { mm[w] = stk[sp][w]; mm[8 + w] = h[w]; }
            blake2s_block(h, mm, 64u, one);
        }
#pragma unroll
        for (int w = 0; w < 8; w++) stk[sp][w] = h[w];
        ++sp;
    }
#pragma unroll
    for (int w = 0; w < 8; w++) root[w] = stk[0][w];
}

// Reduce 2^k consecutive 8-word hashes starting at hashes + 8*base.
__device__ __forceinline__ void node_subtree_root(const uint32_t *hashes, uint64_t base, uint32_t k, uint32_t root[8],
                                                  uint32_t one = 1u) {
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
            blake2s_block(h, mm, 64u, one);
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

// The hashing kernels take `one` (always 1) as a parameter for the pipe
// balance of the Blake2s compression.
template <class Src>
__global__ void __launch_bounds__(256) leaf_subtree_kernel(Src src, uint32_t *out, uint64_t n_threads, uint32_t kl,
                                                           uint32_t one) {
    pdl_wait();
    uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_threads) return;
    if constexpr (plain_adds<Src>::value) one = 1u;
    src.init();
    uint32_t h[8];
    subtree_root(src, t << kl, kl, h, one);
    store_hash(out + 8ull * t, h);
}

__global__ void node_subtree_kernel(const uint32_t *in, uint32_t *out, uint64_t n_threads, uint32_t k, uint32_t one);

// Device transcript state (channel.rs:15-185), advanced by the kernel that
// finishes a commitment.
struct DevChannel {
    uint32_t state[8];
    uint32_t n_draws;
    uint32_t err;  // nonzero if a bounded loop gave up
};

// squeeze = Blake2s(state || n_draws_le32 || 0x00), 37 bytes (channel.rs:174-182)
__device__ __forceinline__ void chan_squeeze(const uint32_t state[8], uint32_t n_draws, uint32_t out[8]) {
    uint32_t m[16];
#pragma unroll
    for (int i = 0; i < 8; i++) m[i] = state[i];
    m[8] = n_draws;
#pragma unroll
    for (int i = 9; i < 16; i++) m[i] = 0u;
    blake2s_block(out, m, 37u);
}

// draw_felt (channel.rs:65-84): squeeze until all 8 words < 2P, take words
// 0..3 mod P.  Bounded: after 64 rejections (probability ~2^-1700) the
// status word is set and zeros are returned.
__device__ __forceinline__ void chan_draw_felt(DevChannel *ch, uint32_t out[4]) {
    for (int it = 0; it < 64; it++) {
        uint32_t w[8];
        chan_squeeze(ch->state, ch->n_draws, w);
        ch->n_draws++;
        bool ok = true;
#pragma unroll
        for (int i = 0; i < 8; i++) ok &= w[i] < 2u * VX_P;
        if (ok) {
#pragma unroll
            for (int i = 0; i < 4; i++) out[i] = w[i] % VX_P;
            return;
        }
    }
    ch->err = 1u;
    out[0] = out[1] = out[2] = out[3] = 0u;
}

// After a commitment: mix_digest(root) (channel.rs:31-40), copy the root into
// the proof, optionally draw the next challenge.
struct ChanStep {
    DevChannel *ch;       // null: no transcript step
    uint32_t *proof_root; // 8 words in the proof
    uint32_t *alpha_out;  // null: no draw
};
__device__ __forceinline__ void chan_commit(const ChanStep &c, const uint32_t root[8]) {
    uint32_t m[16];
#pragma unroll
    for (int i = 0; i < 8; i++) { m[i] = c.ch->state[i]; m[8 + i] = root[i]; c.proof_root[i] = root[i]; }
    uint32_t h[8];
    blake2s_block(h, m, 64u);
#pragma unroll
    for (int i = 0; i < 8; i++) c.ch->state[i] = h[i];
    c.ch->n_draws = 0;
    if (c.alpha_out) chan_draw_felt(c.ch, c.alpha_out);
}

// Stored levels of one tree: level[0] is the leaf data (via its source),
// level[i] (i >= 1) an array of hashes at tree height height[i];
// height[n-1] = depth holds the root.  Consecutive heights differ by 1..4,
// so an authentication path is rebuilt from at most 16 nodes per level.
//
// Build: trees of depth <= 16 go to one multi-block reduce launch straight
// from the leaves.  Deeper trees: one thread per 2^k-leaf subtree (k = 1..4,
// chosen so that at least 2^16 threads run), then 16 -> 1 node kernels while
// a level has more than 2^20 hashes, then the reduce launch for the rest.
// The reduce kernel works in stages of up to 8 levels: each block reduces 256
// hashes in shared memory, one compression per thread per level; the last
// block of every group of 256 (found with a counter, no waiting) carries on
// with the group's roots, and the block that reaches the root performs the
// transcript step of the commitment.
struct TreeLevels {
    uint32_t n;            // number of stored levels including the leaf level
    uint32_t top;          // stored level the reduce kernel starts from (0: leaves)
    uint32_t height[12];
    uint32_t *hashes[12];  // hashes[0] unused
    uint32_t *cnt;         // group counters of the reduce kernel (zero between launches)
    uint32_t n_cnt;
};

constexpr uint32_t kStageLog = 8;        // levels per reduce stage (256 hashes per block)
constexpr uint32_t kReduceThreads = 128;

// Carve the stored levels and counters of a 2^depth-leaf tree from `pool`
// (null: size only); returns the words used.  Trees deeper than 16 start
// with the leaf kernel hashing 2^leaf_k leaves per thread (1..4; 0 = the
// current device's choice, tree_leaf_k).  A layout that sizes a pool and
// carves it later passes the same leaf_k to both calls.
uint64_t tree_plan(uint32_t depth, uint32_t *pool, TreeLevels *lv, uint32_t leaf_k);
uint64_t tree_pool_words(uint32_t depth, uint32_t leaf_k);
// Leaf-kernel subtree size (log2 of leaves per thread) for trees of this
// depth on the current device, and the autotuner's override (1..4; 0 resets),
// per leaf kind: narrow leaves (a few M31 words: trace columns, the quotient)
// and wide leaves, whose load is heavy (FRI layers: a QM31 fold of two loaded
// values; lifted rows of many columns; their combinations).  Wide leaves
// want small subtrees: each thread's leaves wait on their loads in turn.
constexpr uint32_t kLeafNarrow = 0, kLeafFold = 1, kLeafKinds = 2;
uint32_t tree_leaf_k(uint32_t depth, uint32_t kind = kLeafNarrow);
void tree_knob_set(int dev, uint32_t depth, uint32_t k, uint32_t kind = kLeafNarrow);
// Zero the group counters of a freshly carved tree.
cudaError_t tree_reset(const TreeLevels &lv, cudaStream_t stream);

// Write this block's part of level `h` if it is a stored level: cnt hashes
// held at sh, chunk index `part` of that level.
__device__ __forceinline__ void store_level_part(const TreeLevels &lv, uint32_t h, const uint32_t *sh, uint32_t cnt,
                                                 uint64_t part) {
    for (uint32_t i = 1; i < lv.n; i++) {
        if (lv.height[i] != h) continue;
        uint4 *dst = (uint4 *)(lv.hashes[i] + 8ull * part * cnt);
        const uint4 *s4 = (const uint4 *)sh;
        for (uint32_t j = threadIdx.x; j < 2u * cnt; j += blockDim.x) dst[j] = s4[j];
    }
}

template <class Src>
__global__ void __launch_bounds__(kReduceThreads) tree_reduce_kernel(Src src, TreeLevels lv, ChanStep cs, uint32_t one) {
    __shared__ __align__(16) uint32_t sh[8u << kStageLog];
    __shared__ uint32_t is_last;
    pdl_wait();
    if constexpr (plain_adds<Src>::value) one = 1u;
    const uint32_t depth = lv.height[lv.n - 1];
    uint32_t h = lv.height[lv.top];
    const uint32_t *in = lv.top ? lv.hashes[lv.top] : nullptr;
    uint64_t part = blockIdx.x;     // this block's chunk of the current stage
    uint64_t chunks = gridDim.x;    // chunks of the current stage
    uint32_t cbase = 0;             // first counter of the current stage
    while (true) {
        const uint32_t c = depth - h < kStageLog ? depth - h : kStageLog;
        const uint32_t m = 1u << c;
        if (!in) {
            src.init();
            for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) {
                uint32_t hv[8];
                leaf_digest(src, (part << c) + i, hv, one);
                store_hash(sh + 8 * i, hv);
            }
        } else {
            const uint4 *p = (const uint4 *)(in + 8ull * (part << c));
            for (uint32_t j = threadIdx.x; j < 2u * m; j += blockDim.x) ((uint4 *)sh)[j] = __ldcg(p + j);
        }
        __syncthreads();
        for (uint32_t d = 0; d < c; d++) {
            const uint32_t half = m >> (d + 1);
            for (uint32_t base = 0; base < half; base += blockDim.x) {
                const uint32_t t = base + threadIdx.x;
                uint32_t hv[8];
                const bool act = t < half;
                if (act) blake2s_node(hv, sh + 16 * t, sh + 16 * t + 8, one);
                __syncthreads();
                if (act) store_hash(sh + 8 * t, hv);
                __syncthreads();
            }
            store_level_part(lv, h + d + 1, sh, half, part);
        }
        h += c;
        if (h == depth) {
            if (threadIdx.x == 0 && cs.ch) chan_commit(cs, sh);
            return;
        }
        // this chunk's root is in the stored level at height h; the last
        // block of each group of 2^cn chunks reduces the group next
        const uint32_t cn = depth - h < kStageLog ? depth - h : kStageLog;
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t *ctr = lv.cnt + cbase + (part >> cn);
            uint32_t old = atomicAdd(ctr, 1u);
            is_last = old == (1u << cn) - 1u;
            if (is_last) *ctr = 0u;  // every block of the group has arrived: ready for the next launch
        }
        __syncthreads();
        if (!is_last) return;
        __threadfence();
        cbase += (uint32_t)(chunks >> cn);
        chunks >>= cn;
        part >>= cn;
        in = nullptr;
        for (uint32_t i = 1; i < lv.n; i++)
            if (lv.height[i] == h) in = lv.hashes[i];
    }
}

// Build all stored levels and the transcript step (no host sync).  Every
// kernel is a programmatic dependent launch: the chain of a commitment (and
// of consecutive commitments, FRI layer after FRI layer) is strictly ordered
// by pdl_wait() at each kernel's start, and only the launch gaps overlap.
template <class Src>
cudaError_t tree_build(const Src &src, const TreeLevels &lv, const ChanStep &cs, cudaStream_t stream) {
    const uint32_t depth = lv.height[lv.n - 1];
    cudaError_t e = cudaSuccess;
    if (lv.top > 0) {
        uint32_t kl = lv.height[1];
        uint64_t n1 = 1ull << (depth - kl);
        e = launch_pdl(leaf_subtree_kernel<Src>, dim3((unsigned)((n1 + 255) / 256)), dim3(256), 0, stream, src,
                       lv.hashes[1], n1, kl, 1u);
        for (uint32_t i = 2; i <= lv.top && e == cudaSuccess; i++) {
            uint32_t k = lv.height[i] - lv.height[i - 1];
            uint64_t nt = 1ull << (depth - lv.height[i]);
            e = launch_pdl(node_subtree_kernel, dim3((unsigned)((nt + 255) / 256)), dim3(256), 0, stream,
                           (const uint32_t *)lv.hashes[i - 1], lv.hashes[i], nt, k, 1u);
        }
    }
    if (e != cudaSuccess) return e;
    const uint32_t u = depth - lv.height[lv.top];
    const uint32_t c0 = u < kStageLog ? u : kStageLog;
    return launch_pdl(tree_reduce_kernel<Src>, dim3((unsigned)(1ull << (u - c0))), dim3(kReduceThreads), 0, stream,
                      src, lv, cs, 1u);
}

// Kernels launched by tree_build for this plan.
inline uint32_t tree_launches(const TreeLevels &lv) { return lv.top + 1u; }

}  // namespace vx
