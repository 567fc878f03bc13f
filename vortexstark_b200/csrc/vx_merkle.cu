// Merkle kernels that are not templated on a leaf source, plus tree planning.
#include <cstring>

#include "vx_common.cuh"
#include "vx_merkle.cuh"

namespace vx {

__global__ void __launch_bounds__(256) node_subtree_kernel(const uint32_t *in, uint32_t *out, uint64_t n_threads,
                                                           uint32_t k, uint32_t one) {
    pdl_wait();
    uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_threads) return;
    uint32_t h[8];
    node_subtree_root(in, t << k, k, h, one);
    store_hash(out + 8ull * t, h);
}

namespace {
// Leaf-kernel subtree size (log2 leaves per thread, 1..4) per device, leaf
// kind and tree depth, written by the autotuner; 0 = the default rule.
uint8_t g_leaf_k[64][kLeafKinds][32];
bool g_leaf_k_init[64] = {false};
}  // namespace

void tree_knob_set(int dev, uint32_t depth, uint32_t k, uint32_t kind) {
    if (dev < 0 || dev >= 64 || depth >= 32 || k > 4 || kind >= kLeafKinds) return;
    if (!g_leaf_k_init[dev]) {
        memset(g_leaf_k[dev], 0, sizeof(g_leaf_k[dev]));
        g_leaf_k_init[dev] = true;
    }
    g_leaf_k[dev][kind][depth] = (uint8_t)k;
}

uint32_t tree_leaf_k(uint32_t depth, uint32_t kind) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (kind >= kLeafKinds) kind = kLeafNarrow;
    if (dev >= 0 && dev < 64 && g_leaf_k_init[dev] && depth < 32 && g_leaf_k[dev][kind][depth])
        return g_leaf_k[dev][kind][depth];
    // Wide leaves (a fold of 32 bytes of input, a lifted row): 4 leaves per
    // thread, so more threads keep their loads in flight (measured on a
    // 2^26-point FRI chain: 6.08 ms against 6.82 ms with 16 per thread).
    if (kind == kLeafFold) return 2u;
    // narrow leaves: 2^k leaves per thread, k = 1..4, at least 2^16 threads
    int k = (int)depth - 17;
    return (uint32_t)(k < 1 ? 1 : (k > 4 ? 4 : k));
}

uint64_t tree_plan(uint32_t depth, uint32_t *pool, TreeLevels *lv, uint32_t leaf_k) {
    lv->n = 1;
    lv->height[0] = 0;
    lv->hashes[0] = nullptr;
    uint64_t used = 0;
    auto add = [&](uint32_t h) {
        lv->height[lv->n] = h;
        lv->hashes[lv->n] = pool ? pool + used : nullptr;
        used += 8ull << (depth - h);
        lv->n++;
    };
    uint32_t h = 0;
    lv->top = 0;
    if (depth > 16) {
        h = (leaf_k >= 1 && leaf_k <= 4) ? leaf_k : tree_leaf_k(depth);  // leaf kernel: 2^h leaves per thread
        add(h);
        while (depth - h > 20) { h += 4; add(h); }  // node kernels, 16 -> 1
        lv->top = lv->n - 1;
    }
    // reduce stages of 8 levels from h: every 4th height is stored, so the
    // stage boundaries h + 8j are stored levels
    while (h < depth) { h = h + 4 < depth ? h + 4 : depth; add(h); }
    // one counter per group of every stage after the first
    uint32_t u = depth - lv->height[lv->top];
    uint32_t x = u - (u < kStageLog ? u : kStageLog);  // log2 of the first stage's chunks
    uint64_t nc = 0;
    while (x > 0) {
        uint32_t cn = x < kStageLog ? x : kStageLog;
        nc += 1ull << (x - cn);
        x -= cn;
    }
    lv->n_cnt = (uint32_t)nc;
    lv->cnt = (pool && nc) ? pool + used : nullptr;
    used += nc;
    return used;
}

uint64_t tree_pool_words(uint32_t depth, uint32_t leaf_k) {
    TreeLevels lv;
    return tree_plan(depth, nullptr, &lv, leaf_k);
}

cudaError_t tree_reset(const TreeLevels &lv, cudaStream_t stream) {
    if (!lv.cnt || !lv.n_cnt) return cudaSuccess;
    return cudaMemsetAsync(lv.cnt, 0, 4ull * lv.n_cnt, stream);
}

}  // namespace vx

namespace vx {
namespace {
// Register-only Blake2s chain: the message is the previous digest twice, so
// every compression depends on the last and nothing touches memory.  Same
// pipe-balanced compression (one == 1) as the tree kernels.
__global__ void __launch_bounds__(256) blake2s_probe_kernel(uint32_t iters, uint32_t *out, uint32_t one) {
    uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t h[8];
    for (int i = 0; i < 8; i++) h[i] = tid * 0x9E3779B9u + i;
    for (uint32_t it = 0; it < iters; it++) {
        uint32_t m[16];
#pragma unroll
        for (int i = 0; i < 8; i++) { m[i] = h[i]; m[8 + i] = h[i] ^ it; }
        blake2s_block(h, m, 64u, one);
    }
    out[tid] = h[0] ^ h[1] ^ h[2] ^ h[3] ^ h[4] ^ h[5] ^ h[6] ^ h[7];
}
}  // namespace
}  // namespace vx

extern "C" int vx_probe_blake2s(uint32_t blocks, uint32_t threads, uint32_t iters, uint32_t *out, void *stream) {
    VX_CHECK_ARG(out != nullptr && blocks > 0 && threads > 0 && threads <= 256, "vx_probe_blake2s: bad launch shape");
    vx::blake2s_probe_kernel<<<blocks, threads, 0, (cudaStream_t)stream>>>(iters, out, 1u);
    VX_CUDA_TRY(cudaGetLastError());
    return VX_OK;
}

extern "C" int vx_tree_plan(uint32_t depth, uint32_t heights[12], uint32_t *n_levels, uint32_t *top,
                            uint32_t *n_counters, uint64_t *pool_words) {
    VX_CHECK_ARG(depth >= 1 && depth <= 31, "vx_tree_plan: depth %u outside 1..31", depth);
    VX_CHECK_ARG(heights && n_levels && top && n_counters && pool_words, "vx_tree_plan: null output");
    vx::TreeLevels lv;
    uint64_t w = vx::tree_plan(depth, nullptr, &lv, 0);
    for (uint32_t i = 0; i < 12; i++) heights[i] = i < lv.n ? lv.height[i] : 0u;
    *n_levels = lv.n;
    *top = lv.top;
    *n_counters = lv.n_cnt;
    *pool_words = w;
    return VX_OK;
}

extern "C" uint64_t vx_merkle_workspace_words(uint32_t log_n_leaves) {
    if (log_n_leaves < 1 || log_n_leaves > 31) return 0;
    return vx::tree_pool_words(log_n_leaves, vx::tree_leaf_k(log_n_leaves));
}

extern "C" int vx_merkle_root_cols(const uint32_t *const *host_col_ptrs, uint32_t n_cols, uint32_t log_n_leaves,
                                   uint32_t *workspace, uint64_t workspace_words, uint32_t *root_out, void *stream) {
    using namespace vx;
    VX_CHECK_ARG(log_n_leaves >= 1 && log_n_leaves <= 31, "vx_merkle_root_cols: log_n_leaves %u outside 1..31",
                 log_n_leaves);
    VX_CHECK_ARG(host_col_ptrs && n_cols >= 1 && n_cols <= 16, "vx_merkle_root_cols: 1..16 columns");
    VX_CHECK_ARG(workspace && root_out, "vx_merkle_root_cols: null workspace or root");
    for (uint32_t c = 0; c < n_cols; c++) VX_CHECK_ARG(host_col_ptrs[c], "vx_merkle_root_cols: column %u is null", c);
    const uint32_t d = log_n_leaves;
    // the device's leaf-kernel shape, or a larger subtree (smaller stored
    // level) if the workspace was sized for one
    uint32_t k = tree_leaf_k(d);
    while (k < 4 && tree_pool_words(d, k) > workspace_words) k++;
    VX_CHECK_ARG(tree_pool_words(d, k) <= workspace_words,
                 "vx_merkle_root_cols: workspace of %llu words, %llu needed", (unsigned long long)workspace_words,
                 (unsigned long long)tree_pool_words(d, k));
    cudaStream_t st = (cudaStream_t)stream;
    TreeLevels lv;
    tree_plan(d, workspace, &lv, k);
    VX_CUDA_TRY(tree_reset(lv, st));
    const ChanStep none{nullptr, nullptr, nullptr};
    cudaError_t e;
    if (n_cols == 1) {
        e = tree_build(LeafM31{host_col_ptrs[0]}, lv, none, st);
    } else if (n_cols == 4) {
        e = tree_build(LeafSoA4{host_col_ptrs[0], host_col_ptrs[1], host_col_ptrs[2], host_col_ptrs[3]}, lv, none, st);
    } else {
        LeafColsV src{};
        for (uint32_t c = 0; c < n_cols; c++) src.col[c] = host_col_ptrs[c];
        src.n = n_cols;
        e = tree_build(src, lv, none, st);
    }
    VX_CUDA_TRY(e);
    VX_CUDA_TRY(cudaMemcpyAsync(root_out, lv.hashes[lv.n - 1], 32, cudaMemcpyDeviceToDevice, st));
    return VX_OK;
}
