// FRI fold layers with their commitments: per-layer tree builds for the large
// layers, one single-block launch for the small layers at the end of a run.
#include <cstring>

#include "vx_common.cuh"
#include "vx_fri.cuh"
#include "vx_fri_tail.cuh"

namespace vx {
namespace {

constexpr uint32_t kTailThreads = 1u << (kTailMaxLog - 1);  // one thread per leaf pair of the largest layer

struct TailLayer {
    const uint32_t *tw;
    const uint32_t *alpha;
    uint32_t *o[4];
    TreeLevels lv;
    ChanStep cs;
};
struct TailArgs {
    const uint32_t *in[4];  // values folded by the first tail layer (global)
    DevChannel *ch;         // the transcript of every tail layer, or null
    uint32_t d0, n;         // depth of the first tail layer; layer k has depth d0 - k
    TailLayer L[kTailMaxLayers];
};
static_assert(sizeof(TailArgs) <= 4096, "tail kernel arguments exceed the 4 KB parameter space");

// The compressions here use the plain three-input add: this kernel is bound
// by the latency of its dependent compressions, not by pipe throughput.
// Thread t folds and hashes leaves 2t and 2t + 1 and hashes their parent, so
// level 1 of each tree is ready after one barrier; the levels above reduce
// in shared memory, one compression per thread per level, as the reduce
// kernel's stages do.  The folded values of layer k stay in shared memory
// (va for even k, vb for odd k) as the input of layer k + 1, and go to the
// layer's columns for the queries and the decommitment.
__global__ void __launch_bounds__(kTailThreads) fri_tail_kernel(const __grid_constant__ TailArgs a) {
    __shared__ __align__(16) uint32_t dig[8u * kTailThreads];
    __shared__ __align__(16) uint4 va[1u << kTailMaxLog];
    __shared__ __align__(16) uint4 vb[1u << (kTailMaxLog - 1)];
    __shared__ uint32_t al[4];
    __shared__ DevChannel sch;  // the transcript, held here for the whole tail
    const uint32_t tid = threadIdx.x;
    // a.ch: the channel of every layer's transcript step (null: none)
    if (tid == 0 && a.ch) sch = *a.ch;
    for (uint32_t k = 0; k < a.n; k++) {
        const TailLayer &T = a.L[k];
        const uint32_t d = a.d0 - k, half = 1u << (d - 1);
        // the challenge: drawn by thread 0 in the previous layer's transcript
        // step, or by an earlier launch for the first layer
        if (tid == 0)
            for (int i = 0; i < 4; i++) al[i] = T.alpha[i];
        __syncthreads();
        const qmat am = qmat_of(qm31{{al[0], al[1], al[2], al[3]}});
        const uint4 *src = (k & 1u) ? va : vb;
        uint4 *dst = (k & 1u) ? vb : va;
        if (tid < half) {
            uint32_t h2[2][8];
#pragma unroll
            for (int q = 0; q < 2; q++) {
                const uint32_t j = 2u * tid + (uint32_t)q;
                qm31 f0, f1;
                if (k == 0) {
                    const uint2 a0 = __ldg((const uint2 *)a.in[0] + j), a1 = __ldg((const uint2 *)a.in[1] + j);
                    const uint2 a2 = __ldg((const uint2 *)a.in[2] + j), a3 = __ldg((const uint2 *)a.in[3] + j);
                    f0 = qm31{{a0.x, a1.x, a2.x, a3.x}};
                    f1 = qm31{{a0.y, a1.y, a2.y, a3.y}};
                } else {
                    const uint4 x0 = src[2u * j], x1 = src[2u * j + 1u];
                    f0 = qm31{{x0.x, x0.y, x0.z, x0.w}};
                    f1 = qm31{{x1.x, x1.y, x1.z, x1.w}};
                }
                const qm31 r = qadd(qadd(f0, f1), qmul_mat(am, qmulm(qsub(f0, f1), __ldg(T.tw + j))));
                T.o[0][j] = r.v[0]; T.o[1][j] = r.v[1]; T.o[2][j] = r.v[2]; T.o[3][j] = r.v[3];
                dst[j] = make_uint4(r.v[0], r.v[1], r.v[2], r.v[3]);
                uint32_t m[16];
#pragma unroll
                for (int w = 0; w < 16; w++) m[w] = w < 4 ? r.v[w] : 0u;
                blake2s_block(h2[q], m, 16u);
            }
            uint32_t hn[8];
            blake2s_node(hn, h2[0], h2[1]);
            store_hash(dig + 8u * tid, hn);
        }
        __syncthreads();
        store_level_part(T.lv, 1u, dig, half, 0);
        for (uint32_t l = 2; l <= d; l++) {
            const uint32_t cnt = 1u << (d - l);
            uint32_t hv[8];
            const bool act = tid < cnt;
            if (act) blake2s_node(hv, dig + 16u * tid, dig + 16u * tid + 8u);
            __syncthreads();
            if (act) store_hash(dig + 8u * tid, hv);
            __syncthreads();
            store_level_part(T.lv, l, dig, cnt, 0);
        }
        if (tid == 0 && a.ch) chan_commit(ChanStep{&sch, T.cs.proof_root, T.cs.alpha_out}, dig);
        __syncthreads();
    }
    if (tid == 0 && a.ch) *a.ch = sch;
}

uint32_t layer_depth(const FoldLayer &f) { return f.lv.height[f.lv.n - 1]; }

}  // namespace

cudaError_t fold_layers(const FoldLayer *layers, uint32_t n, cudaStream_t st, uint32_t *launches) {
    // the tail: the longest run at the end of consecutive layers (each folding
    // the previous one's output) of 2 .. 2^kTailMaxLog values
    uint32_t t0 = n;
    while (t0 > 0 && n - t0 < kTailMaxLayers) {
        const FoldLayer &f = layers[t0 - 1];
        const uint32_t d = layer_depth(f);
        if (d < 1 || d > kTailMaxLog) break;
        if (t0 < n) {
            const FoldLayer &g = layers[t0];
            if (layer_depth(g) + 1 != d) break;
            bool chained = g.cs.ch == f.cs.ch;  // one transcript for the whole tail
            for (int c = 0; c < 4; c++) chained &= g.in[c] == f.out[c];
            if (!chained) break;
        }
        t0--;
    }
    for (uint32_t k = 0; k < t0; k++) {
        const FoldLayer &f = layers[k];
        LeafFold lf{f.in[0], f.in[1], f.in[2], f.in[3], f.tw, f.alpha, f.out[0], f.out[1], f.out[2], f.out[3], {}};
        cudaError_t e = tree_build(lf, f.lv, f.cs, st);
        if (e != cudaSuccess) return e;
        *launches += tree_launches(f.lv);
    }
    if (t0 == n) return cudaSuccess;
    TailArgs args;
    memset(&args, 0, sizeof(args));
    for (int c = 0; c < 4; c++) args.in[c] = layers[t0].in[c];
    args.ch = layers[t0].cs.ch;
    args.d0 = layer_depth(layers[t0]);
    args.n = n - t0;
    for (uint32_t k = 0; k < args.n; k++) {
        const FoldLayer &f = layers[t0 + k];
        TailLayer &T = args.L[k];
        T.tw = f.tw;
        T.alpha = f.alpha;
        for (int c = 0; c < 4; c++) T.o[c] = f.out[c];
        T.lv = f.lv;
        T.cs = f.cs;
    }
    fri_tail_kernel<<<1, kTailThreads, 0, st>>>(args);
    *launches += 1;
    return cudaGetLastError();
}

}  // namespace vx
