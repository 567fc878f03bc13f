// FRI chain of a QM31 codeword with a commitment per layer.
//
// The codeword (4 SoA columns of 2^L words, the evaluation on half_coset(L))
// is folded down to 2 values: layer 0 is its circle fold, layer k >= 1 the
// line fold of layer k-1, each folded with a challenge drawn from the
// transcript after the previous layer's root was mixed in, each committed as
// a 4-word-leaf Blake2s tree (the proof's FRI, prover.rs:860-926, with the
// folds of fri.rs:163-224, run to 2 values).  A circle fold into a zeroed
// destination has the line fold's formula, so every layer is one tree_build
// over a LeafFold source: the fold happens inside the hashing kernels and
// the transcript step inside the kernel that finishes each tree.
#include <cstring>

#include "vx_common.cuh"
#include "vx_fri.cuh"
#include "vx_merkle.cuh"
#include "vx_twiddles.cuh"

using namespace vx;

struct vx_fri_chain {
    int device = 0;
    uint32_t L = 0, nl = 0;
    void *block = nullptr;
    size_t bytes = 0;
    uint32_t *tw_circle = nullptr;
    uint32_t *tw_line[32] = {};  // half_odds(l) twiddles, l = L-1 .. 2
    uint32_t *F[32][4] = {};      // layer k: 2^(L-1-k) values
    TreeLevels lv[32];
    DevChannel *chan = nullptr;
    uint32_t *alphas = nullptr;   // 4 words per layer
    uint32_t *roots = nullptr;    // 8 words per layer
    uint32_t launches = 0;
};

namespace {

struct Digest8v { uint32_t w[8]; };

__global__ void chain_init_kernel(DevChannel *ch, Digest8v state, uint32_t *alpha0) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    for (int i = 0; i < 8; i++) ch->state[i] = state.w[i];
    ch->n_draws = 0;
    ch->err = 0;
    chan_draw_felt(ch, alpha0);
}

uint64_t align64(uint64_t w) { return (w + 63) & ~63ull; }

}  // namespace

extern "C" int vx_fri_chain_create(uint32_t log_size, vx_fri_chain **out) {
    VX_CHECK_ARG(out != nullptr, "vx_fri_chain_create: out is null");
    VX_CHECK_ARG(log_size >= 3 && log_size <= 30, "vx_fri_chain_create: log_size %u outside 3..30", log_size);
    vx_fri_chain *h = new vx_fri_chain();
    cudaGetDevice(&h->device);
    h->L = log_size;
    h->nl = log_size - 1;
    const uint32_t L = h->L;
    // layout (words): circle twiddles, line twiddles, layers, trees, channel, challenges, roots
    uint64_t w = 0;
    const uint64_t o_tc = w; w += align64(1ull << (L - 1));
    uint64_t o_tl[32];
    for (uint32_t l = L - 1; l >= 2; l--) { o_tl[l] = w; w += align64(1ull << (l - 1)); }
    uint64_t o_f[32];
    for (uint32_t k = 0; k < h->nl; k++) { o_f[k] = w; w += 4 * align64(1ull << (L - 1 - k)); }
    uint32_t kk[32];
    uint64_t o_t[32];
    for (uint32_t k = 0; k < h->nl; k++) {
        kk[k] = tree_leaf_k(L - 1 - k, kLeafFold);
        o_t[k] = w;
        w += align64(tree_pool_words(L - 1 - k, kk[k]));
    }
    const uint64_t o_ch = w; w += align64(sizeof(DevChannel) / 4 + 1);
    const uint64_t o_al = w; w += align64(4ull * h->nl);
    const uint64_t o_rt = w; w += align64(8ull * h->nl);
    if (cudaMalloc(&h->block, w * 4) != cudaSuccess) {
        cudaGetLastError();
        delete h;
        set_last_error(VX_ERR_OOM, "cudaMalloc of %llu bytes for a FRI chain failed", (unsigned long long)(w * 4));
        return VX_ERR_OOM;
    }
    h->bytes = w * 4;
    uint32_t *b = (uint32_t *)h->block;
    h->tw_circle = b + o_tc;
    for (uint32_t l = L - 1; l >= 2; l--) h->tw_line[l] = b + o_tl[l];
    for (uint32_t k = 0; k < h->nl; k++) {
        const uint64_t sz = align64(1ull << (L - 1 - k));
        for (int c = 0; c < 4; c++) h->F[k][c] = b + o_f[k] + c * sz;
        tree_plan(L - 1 - k, b + o_t[k], &h->lv[k], kk[k]);
    }
    h->chan = (DevChannel *)(b + o_ch);
    h->alphas = b + o_al;
    h->roots = b + o_rt;
    cudaError_t e = build_fold_twiddles(ecoset_half_coset(L), true, h->tw_circle, nullptr);
    for (uint32_t l = L - 1; l >= 2 && e == cudaSuccess; l--)
        e = build_fold_twiddles(ecoset_half_odds(l), false, h->tw_line[l], nullptr);
    for (uint32_t k = 0; k < h->nl && e == cudaSuccess; k++) e = tree_reset(h->lv[k], nullptr);
    if (e == cudaSuccess) e = cudaStreamSynchronize(nullptr);
    if (e != cudaSuccess) {
        cudaFree(h->block);
        delete h;
        set_last_error(VX_ERR_CUDA, "vx_fri_chain_create: %s", cudaGetErrorString(e));
        return VX_ERR_CUDA;
    }
    *out = h;
    return VX_OK;
}

extern "C" void vx_fri_chain_destroy(vx_fri_chain *h) {
    if (!h) return;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(h->device);
    cudaFree(h->block);
    cudaSetDevice(prev);
    delete h;
}

extern "C" uint32_t vx_fri_chain_layers(const vx_fri_chain *h) { return h ? h->nl : 0u; }

extern "C" int vx_fri_chain_commit_async(vx_fri_chain *h, const uint32_t *const *host_cols, const uint32_t state[8],
                                         void *stream) {
    VX_CHECK_ARG(h && host_cols && state, "vx_fri_chain_commit_async: null argument");
    for (int c = 0; c < 4; c++) {
        VX_CHECK_ARG(host_cols[c] != nullptr, "vx_fri_chain_commit_async: column %d is null", c);
        VX_CHECK_ARG(((uintptr_t)host_cols[c] & 7u) == 0, "vx_fri_chain_commit_async: column %d not 8-byte aligned", c);
    }
    cudaStream_t st = (cudaStream_t)stream;
    Digest8v s8;
    memcpy(s8.w, state, 32);
    chain_init_kernel<<<1, 32, 0, st>>>(h->chan, s8, h->alphas);
    VX_CUDA_TRY(cudaGetLastError());
    uint32_t launches = 1;
    for (uint32_t k = 0; k < h->nl; k++) {
        const uint32_t *const *in = k == 0 ? host_cols : (const uint32_t *const *)h->F[k - 1];
        const uint32_t *tw = k == 0 ? h->tw_circle : h->tw_line[h->L - k];
        LeafFold lf{in[0], in[1], in[2], in[3], tw, h->alphas + 4 * k,
                    h->F[k][0], h->F[k][1], h->F[k][2], h->F[k][3], {}};
        VX_CUDA_TRY(tree_build(lf, h->lv[k],
                               ChanStep{h->chan, h->roots + 8 * k, k + 1 < h->nl ? h->alphas + 4 * (k + 1) : nullptr},
                               st));
        launches += tree_launches(h->lv[k]);
    }
    h->launches = launches;
    return VX_OK;
}

extern "C" uint32_t vx_fri_chain_launches(const vx_fri_chain *h) { return h ? h->launches : 0u; }

extern "C" int vx_fri_chain_fetch(vx_fri_chain *h, uint32_t *roots, uint32_t *alphas, uint32_t last[8], void *stream) {
    VX_CHECK_ARG(h && roots && alphas && last, "vx_fri_chain_fetch: null argument");
    cudaStream_t st = (cudaStream_t)stream;
    VX_CUDA_TRY(cudaMemcpyAsync(roots, h->roots, 32ull * h->nl, cudaMemcpyDeviceToHost, st));
    VX_CUDA_TRY(cudaMemcpyAsync(alphas, h->alphas, 16ull * h->nl, cudaMemcpyDeviceToHost, st));
    uint32_t cols[4][2];
    for (int c = 0; c < 4; c++)
        VX_CUDA_TRY(cudaMemcpyAsync(cols[c], h->F[h->nl - 1][c], 8, cudaMemcpyDeviceToHost, st));
    uint32_t err = 0;
    VX_CUDA_TRY(cudaMemcpyAsync(&err, &h->chan->err, 4, cudaMemcpyDeviceToHost, st));
    VX_CUDA_TRY(cudaStreamSynchronize(st));
    for (int i = 0; i < 2; i++)
        for (int c = 0; c < 4; c++) last[4 * i + c] = cols[c][i];
    if (err) {
        set_last_error(VX_ERR_DEVICE, "vx_fri_chain: a challenge draw gave up after 64 rejections");
        return VX_ERR_DEVICE;
    }
    return VX_OK;
}
