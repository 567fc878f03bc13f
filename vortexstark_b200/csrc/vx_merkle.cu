// Merkle kernels that are not templated on a leaf source, plus tree planning.
#include "vx_common.cuh"
#include "vx_merkle.cuh"

namespace vx {

__global__ void __launch_bounds__(256) node_subtree_kernel(const uint32_t *in, uint32_t *out, uint64_t n_threads, uint32_t k) {
    uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_threads) return;
    uint32_t h[8];
    node_subtree_root(in, t << k, k, h);
    store_hash(out + 8ull * t, h);
}

uint64_t tree_plan(uint32_t depth, uint32_t *pool, TreeLevels *lv) {
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
    if (depth > kTopLog) {
        // leaf kernel: 2^k leaves per thread, k = 1..4, at least 2^17 threads when possible
        int k = (int)depth - 17;
        k = k < 1 ? 1 : (k > 4 ? 4 : k);
        h = (uint32_t)k;
        add(h);
        while (depth - h > kTopLog) { h += 4; add(h); }  // node kernels, 16 -> 1
    }
    lv->top = lv->n;                                      // the single-block kernel from here on
    while (h < depth) { h = h + 4 < depth ? h + 4 : depth; add(h); }
    return used;
}

uint64_t tree_pool_words(uint32_t depth) {
    TreeLevels lv;
    return tree_plan(depth, nullptr, &lv);
}

__global__ void __launch_bounds__(1024) top_tree_kernel(const uint32_t *in, uint32_t log_m, TreeLevels lv,
                                                        ChanStep cs) {
    extern __shared__ uint32_t sh[];
    const uint32_t m = 1u << log_m;
    for (uint32_t i = threadIdx.x; i < 8 * m; i += blockDim.x) sh[i] = in[i];
    __syncthreads();
    block_tree_up(sh, log_m, lv.height[lv.top - 1], lv, lv.top);
    if (threadIdx.x == 0 && cs.ch) chan_commit(cs, sh);
}

cudaError_t small_tree_attr(const void *fn) {
    return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(32u << kTopLog));
}

}  // namespace vx

namespace vx {
namespace {
// Register-only Blake2s chain: the message is the previous digest twice, so
// every compression depends on the last and nothing touches memory.
__global__ void __launch_bounds__(256) blake2s_probe_kernel(uint32_t iters, uint32_t *out) {
    uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t h[8];
    for (int i = 0; i < 8; i++) h[i] = tid * 0x9E3779B9u + i;
    for (uint32_t it = 0; it < iters; it++) {
        uint32_t m[16];
#pragma unroll
        for (int i = 0; i < 8; i++) { m[i] = h[i]; m[8 + i] = h[i] ^ it; }
        blake2s_block(h, m, 64u);
    }
    out[tid] = h[0] ^ h[1] ^ h[2] ^ h[3] ^ h[4] ^ h[5] ^ h[6] ^ h[7];
}
}  // namespace
}  // namespace vx

extern "C" int vx_probe_blake2s(uint32_t blocks, uint32_t threads, uint32_t iters, uint32_t *out, void *stream) {
    VX_CHECK_ARG(out != nullptr && blocks > 0 && threads > 0 && threads <= 256, "vx_probe_blake2s: bad launch shape");
    vx::blake2s_probe_kernel<<<blocks, threads, 0, (cudaStream_t)stream>>>(iters, out);
    VX_CUDA_TRY(cudaGetLastError());
    return VX_OK;
}
