// Batched lifted commitment of uneven-size M31 columns ("LIFT" v1).
//
// All columns are extended in the stwo format (interpolate at 2^L, zero
// pad, evaluate at 2^(L+B); circle_ntt_stwo.cu), hashed into one lifted
// Blake2s tree over rows (merkle_leaves_lifted.cu), combined with powers of
// a transcript challenge into one QM31 codeword C = sum_c alpha^c lift(col_c)
// (the lift map of accumulate_lift.cu:26-31), and C goes through FRI with the
// stwo fold twiddles (fri_ops.rs:44-92): a circle fold, then line folds down
// to 8 values, each layer committed with its root mixed into the transcript
// before the next challenge (the Fibonacci FRI of prover.rs:860-926).
// Queries are drawn with draw_query_indices (channel.rs:102-116) and every
// tree is opened at them.  The word layout follows the KRAK proof: header,
// roots, last layer, query indices, then per tree the values at q and q^1
// and both authentication paths.
//
// Device work: equal-size columns share each NTT launch (one launch per
// pass per size), the combination is formed per size group in one launch and
// lifted inside the hashing kernels of C's tree, every fold inside the
// hashing kernels of its layer, and the
// transcript steps inside the kernels that finish each tree.  The whole
// schedule can be captured once as a CUDA graph.
#include <cstring>
#include <mutex>
#include <vector>

#include "vx_common.cuh"
#include "vx_field.cuh"
#include "vx_fri.cuh"
#include "vx_merkle.cuh"
#include "vx_ntt.cuh"
#include "vx_prover.cuh"
#include "vx_twiddles.cuh"

namespace vx {
namespace {

constexpr uint32_t kLiftMagic = 0x5446494Cu;  // "LIFT"
constexpr uint32_t kMaxFri = 32;

struct LiftLayout {
    uint32_t n_cols, B, S, nfri, nq;
    uint32_t logs[kMaxLiftCols];
    uint64_t words;
    uint64_t hdr, r0, r1, nfri_w, froots, nlast, last, nq_w, qidx, nfd;
    DecomLayout lift, comb, fri[kMaxFri];
};

void decom(DecomLayout *d, uint64_t *w, uint32_t nq, uint32_t width, uint32_t depth) {
    d->width = width; d->depth = depth;
    d->n = (*w)++;
    d->vals = *w; *w += (uint64_t)nq * width;
    d->svals = *w; *w += (uint64_t)nq * width;
    d->paths = *w; *w += (uint64_t)nq * (1 + 8ull * depth);
    d->spaths = *w; *w += (uint64_t)nq * (1 + 8ull * depth);
}

bool lift_layout(uint32_t n_cols, const uint32_t *logs, uint32_t B, uint32_t nq, LiftLayout *L) {
    if (n_cols < 1 || n_cols > kMaxLiftCols || B < 1 || B > 4 || nq < 1 || nq > 1024 || !logs) return false;
    for (uint32_t c = 0; c < n_cols; c++) {
        if (logs[c] < 2 || logs[c] + B > 28) return false;
        if (c && logs[c] < logs[c - 1]) return false;
    }
    memset(L, 0, sizeof(*L));
    L->n_cols = n_cols; L->B = B; L->nq = nq;
    L->S = logs[n_cols - 1] + B;
    if (L->S < 4) return false;
    L->nfri = L->S - 3;
    for (uint32_t c = 0; c < n_cols; c++) L->logs[c] = logs[c];
    uint64_t w = 0;
    L->hdr = w; w += 5 + n_cols;  // magic, version, n_cols, B, S, log sizes
    L->r0 = w; w += 8;
    L->r1 = w; w += 8;
    L->nfri_w = w++;
    L->froots = w; w += 8ull * L->nfri;
    L->nlast = w++;
    L->last = w; w += 32;
    L->nq_w = w++;
    L->qidx = w; w += nq;
    decom(&L->lift, &w, nq, n_cols, L->S);
    decom(&L->comb, &w, nq, 4, L->S);
    L->nfd = w++;
    for (uint32_t k = 0; k < L->nfri; k++) decom(&L->fri[k], &w, nq, 4, L->S - 1 - k);
    L->words = w;
    return true;
}

void lift_template(const LiftLayout &L, std::vector<uint32_t> &t) {
    t.assign(L.words, 0u);
    t[L.hdr] = kLiftMagic; t[L.hdr + 1] = 1u; t[L.hdr + 2] = L.n_cols; t[L.hdr + 3] = L.B; t[L.hdr + 4] = L.S;
    for (uint32_t c = 0; c < L.n_cols; c++) t[L.hdr + 5 + c] = L.logs[c];
    t[L.nfri_w] = L.nfri;
    t[L.nlast] = 8u;
    t[L.nq_w] = L.nq;
    auto dec = [&](const DecomLayout &d) {
        t[d.n] = L.nq;
        for (uint32_t q = 0; q < L.nq; q++) {
            t[d.paths + (uint64_t)q * (1 + 8ull * d.depth)] = d.depth;
            t[d.spaths + (uint64_t)q * (1 + 8ull * d.depth)] = d.depth;
        }
    };
    dec(L.lift); dec(L.comb);
    t[L.nfd] = L.nfri;
    for (uint32_t k = 0; k < L.nfri; k++) dec(L.fri[k]);
}

// x mod P folded once: (x & P) + (x >> 31) < 2^34 for any 64-bit x.
__device__ __forceinline__ uint64_t fold64(uint64_t x) { return (x & VX_P) + (x >> 31); }
// Canonical M31 of an accumulator below 2^34.
__device__ __forceinline__ uint32_t reduce34(uint64_t x) {
    const uint32_t r = (uint32_t)fold64(x);  // < 2^31 + 8
    return umin32(r, r - VX_P);
}

// C[i] = sum_c alpha^c * lift(col_c)[i] in two steps.  Columns of one size
// share their lift index, so with G_g = sum over group g's columns of
// alpha^c * col_c (at the group's own 2^le rows), C[i] = sum_g G_g[lift_g(i)]:
// combine_groups_kernel forms every G_g at HBM speed (each LDE word read
// once, where a per-row combination re-reads a lifted column 2^(S-le) times),
// writing the largest group's (le = S, lift index i) straight into C, and the
// leaf of C's tree adds the smaller groups' values at their lifted rows,
// writes the final C and hashes it.
//
// Each coordinate of G is a 64-bit multiply-accumulate of 31-bit products
// (one IMAD.WIDE per column and coordinate), folded every 3 columns so the
// sum stays below 2^34 + 3 * 2^62 < 2^64, and reduced to canonical M31 once.
struct CombineGroupsArgs {
    const uint32_t *lde[kMaxLiftCols];  // group g's first column; column j at + (j << le)
    uint32_t *dst[kMaxLiftCols];        // group g's G: component k at + k * dstride
    uint64_t dstride[kMaxLiftCols];
    uint64_t rows_end[kMaxLiftCols];    // groups' rows laid end to end: group g ends at rows_end[g]
    uint32_t le[kMaxLiftCols], cnt[kMaxLiftCols], first[kMaxLiftCols];
    uint32_t n_groups;
};
// Four consecutive rows per thread (16-byte loads and stores: every group has
// at least 8 rows, and columns and destinations are 64-word aligned), three
// columns' loads in flight, the powers of alpha in shared memory.
__global__ void __launch_bounds__(256) combine_groups_kernel(const __grid_constant__ CombineGroupsArgs a,
                                                             const uint32_t *__restrict__ pw) {
    __shared__ uint4 spw[kMaxLiftCols];
    pdl_wait();
    for (uint32_t c = threadIdx.x; c < kMaxLiftCols; c += blockDim.x) spw[c] = __ldg((const uint4 *)pw + c);
    __syncthreads();
    const uint64_t r = 4ull * ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x);
    if (r >= a.rows_end[a.n_groups - 1]) return;
    uint32_t g = 0;
    while (r >= a.rows_end[g]) g++;
    const uint64_t row = r - (g ? a.rows_end[g - 1] : 0ull);
    const uint32_t cnt = a.cnt[g], first = a.first[g];
    const uint64_t cs4 = 1ull << (a.le[g] - 2u);  // column stride in 16-byte units
    const uint4 *cp = (const uint4 *)(a.lde[g] + row);
    uint64_t s[4][4];  // [row][coordinate]
#pragma unroll
    for (int k = 0; k < 4; k++)
#pragma unroll
        for (int c = 0; c < 4; c++) s[k][c] = 0;
    auto mac = [&](const uint4 v, const uint4 p) {
        const uint32_t vv[4] = {v.x, v.y, v.z, v.w}, pp[4] = {p.x, p.y, p.z, p.w};
#pragma unroll
        for (int k = 0; k < 4; k++)
#pragma unroll
            for (int c = 0; c < 4; c++) s[k][c] += (uint64_t)pp[c] * vv[k];
    };
    auto fold = [&]() {
#pragma unroll
        for (int k = 0; k < 4; k++)
#pragma unroll
            for (int c = 0; c < 4; c++) s[k][c] = fold64(s[k][c]);
    };
    uint32_t j = 0;
    for (; j + 3u <= cnt; j += 3u) {
        const uint4 v0 = __ldg(cp + j * cs4), v1 = __ldg(cp + (j + 1u) * cs4), v2 = __ldg(cp + (j + 2u) * cs4);
        mac(v0, spw[first + j]);
        mac(v1, spw[first + j + 1u]);
        mac(v2, spw[first + j + 2u]);
        fold();
    }
    for (; j < cnt; j++) mac(__ldg(cp + j * cs4), spw[first + j]);  // at most two more
    fold();
    uint32_t *d = a.dst[g] + row;
    const uint64_t ds = a.dstride[g];
#pragma unroll
    for (int c = 0; c < 4; c++)
        *(uint4 *)(d + c * ds) = make_uint4(reduce34(s[0][c]), reduce34(s[1][c]), reduce34(s[2][c]), reduce34(s[3][c]));
}

// Leaf of C's tree: the largest group's G (already in C) plus the smaller
// groups' G at their lifted rows; writes the final C and hashes it.
struct LeafCombine {
    const uint32_t *g[kMaxLiftCols];  // smaller groups' G: component k at + k * gstride
    uint64_t gstride[kMaxLiftCols];
    uint32_t gshift[kMaxLiftCols];    // S - le + 1
    uint32_t n_small;
    uint32_t *o0, *o1, *o2, *o3;
    __device__ __forceinline__ void init() {}
    __device__ __forceinline__ uint32_t load(uint64_t i, uint32_t m[16]) const {
        qm31 a{{o0[i], o1[i], o2[i], o3[i]}};
        const uint32_t i32 = (uint32_t)i;
        for (uint32_t k = 0; k < n_small; k++) {
            const uint32_t *gp = g[k] + (((i32 >> gshift[k]) << 1) | (i32 & 1u));
            const uint64_t gs = gstride[k];
            a = qadd(a, qm31{{__ldg(gp), __ldg(gp + gs), __ldg(gp + 2 * gs), __ldg(gp + 3 * gs)}});
        }
        o0[i] = a.v[0]; o1[i] = a.v[1]; o2[i] = a.v[2]; o3[i] = a.v[3];
        m[0] = a.v[0]; m[1] = a.v[1]; m[2] = a.v[2]; m[3] = a.v[3];
        return 16u;
    }
};

__global__ void powers_kernel(const uint32_t *alpha, uint32_t *pw, uint32_t n) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const qm31 a{{alpha[0], alpha[1], alpha[2], alpha[3]}};
    qm31 p{{1u, 0u, 0u, 0u}};
    for (uint32_t c = 0; c < n; c++) {
        pw[4 * c] = p.v[0]; pw[4 * c + 1] = p.v[1]; pw[4 * c + 2] = p.v[2]; pw[4 * c + 3] = p.v[3];
        p = qmul(p, a);
    }
}

// mix_felts(last layer) (channel.rs:46-59), then draw_query_indices: squeeze
// t (n_draws = t) gives queries 8t .. 8t+7, word & (2^log_domain - 1)
// (channel.rs:102-116); the squeezes run in parallel.
__global__ void lift_queries_kernel(DevChannel *ch, const uint32_t *l0, const uint32_t *l1, const uint32_t *l2,
                                    const uint32_t *l3, uint32_t *proof_last, uint32_t log_domain, uint32_t nq,
                                    uint32_t *qidx, uint32_t *proof_qidx) {
    __shared__ uint32_t st[8];
    const uint32_t nsq = (nq + 7u) / 8u;
    if (threadIdx.x == 0) {
        uint32_t buf[40];
        for (int i = 0; i < 8; i++) buf[i] = ch->state[i];
        for (int i = 0; i < 8; i++) {
            buf[8 + 4 * i] = l0[i]; buf[9 + 4 * i] = l1[i]; buf[10 + 4 * i] = l2[i]; buf[11 + 4 * i] = l3[i];
        }
        for (int i = 0; i < 32; i++) proof_last[i] = buf[8 + i];
        uint32_t h[8];
        blake2s_words(h, buf, 160u);
        for (int i = 0; i < 8; i++) { ch->state[i] = h[i]; st[i] = h[i]; }
        ch->n_draws = nsq;
    }
    __syncthreads();
    const uint32_t mask = (uint32_t)((1ull << log_domain) - 1ull);
    for (uint32_t t = threadIdx.x; t < nsq; t += blockDim.x) {
        uint32_t w[8];
        chan_squeeze(st, t, w);
        for (uint32_t i = 0; i < 8; i++) {
            const uint32_t j = 8u * t + i;
            if (j < nq) { qidx[j] = w[i] & mask; proof_qidx[j] = w[i] & mask; }
        }
    }
}

// Opened values: thread (tree, q); tree 0 = lifted rows, 1 = C, 2 + k = FRI layer k.
struct LiftValuesArgs {
    LeafLifted cols;
    const uint32_t *C[4];
    const uint32_t *F[kMaxFri][4];
    uint64_t vals[2 + kMaxFri], svals[2 + kMaxFri];
    uint32_t nfri;
};
__global__ void lift_values_kernel(const __grid_constant__ LiftValuesArgs a, const uint32_t *qidx, uint32_t nq,
                                   uint32_t *proof) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= (2 + a.nfri) * nq) return;
    const uint32_t tree = tid / nq, q = tid % nq;
    const uint64_t i = qidx[q];
    if (tree == 0) {
        const uint32_t nc = a.cols.n_cols;
        for (uint32_t c = 0; c < nc; c++) {
            proof[a.vals[0] + (uint64_t)q * nc + c] = a.cols.word(c, i);
            proof[a.svals[0] + (uint64_t)q * nc + c] = a.cols.word(c, i ^ 1ull);
        }
    } else if (tree == 1) {
        for (int c = 0; c < 4; c++) {
            proof[a.vals[1] + 4 * q + c] = a.C[c][i];
            proof[a.svals[1] + 4 * q + c] = a.C[c][i ^ 1ull];
        }
    } else {
        const uint32_t k = tree - 2;
        const uint64_t j = i >> (k + 1);
        for (int c = 0; c < 4; c++) {
            proof[a.vals[tree] + 4 * q + c] = a.F[k][c][j];
            proof[a.svals[tree] + 4 * q + c] = a.F[k][c][j ^ 1ull];
        }
    }
}

// Authentication paths: blockIdx.y = tree, threads over (query, stored-level
// group); each rebuilds the <= 16-leaf block of its group from the level
// below (or the leaves) and writes the siblings of its heights.
struct LiftPathTree {
    TreeLevels lv;
    uint32_t kind;   // 0 lifted rows, 1 SoA4 columns
    uint32_t shift;  // leaf index = query >> shift
    const uint32_t *c[4];
    uint64_t paths, spaths;
};
struct LiftPathsArgs {
    LeafLifted cols;
    LiftPathTree t[2 + kMaxFri];
};
__global__ void __launch_bounds__(64) lift_paths_kernel(const __grid_constant__ LiftPathsArgs a, const uint32_t *qidx,
                                                        uint32_t nq, uint32_t *proof) {
    const LiftPathTree &T = a.t[blockIdx.y];
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t ng = T.lv.n - 1;
    if (tid >= nq * ng) return;
    const uint32_t q = tid / ng, g = tid % ng;
    const uint32_t depth = T.lv.height[T.lv.n - 1];
    const uint64_t idx = (uint64_t)qidx[q] >> T.shift;
    const uint32_t lo = T.lv.height[g], k = T.lv.height[g + 1] - lo;
    const uint64_t node = idx >> lo;
    const uint64_t blk = node >> k;
    const uint32_t K = 1u << k;
    uint32_t nh[31][8];
    if (g == 0) {
        for (uint32_t j = 0; j < K; j++) {
            const uint64_t i = (blk << k) + j;
            if (T.kind == 0) {
                a.cols.digest(i, nh[j]);
            } else {
                uint32_t m[16];
#pragma unroll
                for (int w = 0; w < 16; w++) m[w] = 0u;
                m[0] = T.c[0][i]; m[1] = T.c[1][i]; m[2] = T.c[2][i]; m[3] = T.c[3][i];
                blake2s_block(nh[j], m, 16u);
            }
        }
    } else {
        const uint32_t *h = T.lv.hashes[g] + 8ull * (blk << k);
        for (uint32_t j = 0; j < K; j++)
#pragma unroll
            for (int w = 0; w < 8; w++) nh[j][w] = h[8 * j + w];
    }
    uint32_t off = 0, cnt = K;
    for (uint32_t d = 0; d < k; d++) {
        const uint32_t nxt = off + cnt;
        for (uint32_t j = 0; j < cnt / 2; j++) blake2s_node(nh[nxt + j], nh[off + 2 * j], nh[off + 2 * j + 1]);
        off = nxt;
        cnt /= 2;
    }
    uint32_t *p = proof + T.paths + (uint64_t)q * (1u + 8u * depth);
    uint32_t *sp = proof + T.spaths + (uint64_t)q * (1u + 8u * depth);
    off = 0; cnt = K;
    uint64_t local = node & (K - 1u);
    for (uint32_t d = 0; d < k; d++) {
        const uint32_t hgt = lo + d;
        const uint32_t *sib = nh[off + (uint32_t)(local ^ 1u)];
        const uint32_t *self = nh[off + (uint32_t)local];
#pragma unroll
        for (int w = 0; w < 8; w++) {
            p[1 + 8 * hgt + w] = sib[w];
            sp[1 + 8 * hgt + w] = (hgt == 0) ? self[w] : sib[w];
        }
        off += cnt; cnt /= 2; local >>= 1;
    }
}

uint64_t align64(uint64_t w) { return (w + 63) & ~63ull; }

}  // namespace
}  // namespace vx

using namespace vx;

struct vx_lifted {
    int device = 0;
    LiftLayout L;
    uint32_t n_groups = 0;
    uint32_t glog[kMaxLiftCols], gcnt[kMaxLiftCols], gfirst[kMaxLiftCols];
    uint32_t *in[kMaxLiftCols], *co[kMaxLiftCols], *lde[kMaxLiftCols];
    uint32_t *itw[kMaxLiftCols], *tw[kMaxLiftCols];
    uint32_t *fold_circle = nullptr, *fold_line = nullptr;
    uint64_t fold_line_off[32];
    uint32_t *C[4];
    uint32_t *G[kMaxLiftCols];  // combined codeword of each size group but the largest (4 components)
    uint32_t *F[kMaxFri][4];
    TreeLevels lv0, lv1, flv[kMaxFri];
    DevChannel *chan = nullptr;
    uint32_t *alpha = nullptr, *alpha_f = nullptr, *pw = nullptr, *qidx = nullptr, *proof = nullptr;
    LeafLifted cols;
    void *block = nullptr;
    size_t bytes = 0;
    cudaStream_t st = nullptr;       // capture stream
    cudaGraphExec_t exec = nullptr;  // the whole commitment, captured on first use
    uint32_t launches = 0;
};

namespace {

// The lifted tree with the leaf specialised for the last block's word count.
template <uint32_t W>
cudaError_t lifted_tree_w(const LeafLifted &c, const TreeLevels &lv, const ChanStep &cs, cudaStream_t st) {
    LeafLiftedW<W> leaf;
    static_cast<LeafLifted &>(leaf) = c;
    return tree_build(leaf, lv, cs, st);
}
cudaError_t lifted_tree_build(const LeafLifted &c, const TreeLevels &lv, const ChanStep &cs, cudaStream_t st) {
    switch (c.n_cols ? c.n_cols - 16u * ((c.n_cols - 1u) / 16u) : 0u) {
    case 1: return lifted_tree_w<1>(c, lv, cs, st);
    case 2: return lifted_tree_w<2>(c, lv, cs, st);
    case 3: return lifted_tree_w<3>(c, lv, cs, st);
    case 4: return lifted_tree_w<4>(c, lv, cs, st);
    case 5: return lifted_tree_w<5>(c, lv, cs, st);
    case 6: return lifted_tree_w<6>(c, lv, cs, st);
    case 7: return lifted_tree_w<7>(c, lv, cs, st);
    case 8: return lifted_tree_w<8>(c, lv, cs, st);
    case 9: return lifted_tree_w<9>(c, lv, cs, st);
    case 10: return lifted_tree_w<10>(c, lv, cs, st);
    case 11: return lifted_tree_w<11>(c, lv, cs, st);
    case 12: return lifted_tree_w<12>(c, lv, cs, st);
    case 13: return lifted_tree_w<13>(c, lv, cs, st);
    case 14: return lifted_tree_w<14>(c, lv, cs, st);
    case 15: return lifted_tree_w<15>(c, lv, cs, st);
    case 16: return lifted_tree_w<16>(c, lv, cs, st);
    default: return tree_build(c, lv, cs, st);
    }
}

int lift_stage(vx_lifted *h, uint32_t stage, cudaStream_t st, uint32_t *launches) {
    const LiftLayout &L = h->L;
    uint32_t *proof = h->proof;
    const uint32_t B = L.B, S = L.S;
    switch (stage) {
    case 0: {  // LDE of every column: each pass of all size groups in one launch
        VX_CUDA_TRY(cudaMemsetAsync(h->chan, 0, sizeof(DevChannel), st));
        NttGroup gi[kMaxLiftCols], ge[kMaxLiftCols];
        for (uint32_t g = 0; g < h->n_groups; g++) {
            const uint32_t lg = h->glog[g];
            gi[g] = NttGroup{h->co[g], 1ull << lg, h->gcnt[g], lg, stwo_tables(h->itw[g], lg), h->in[g], lg};
            ge[g] = NttGroup{h->lde[g], 1ull << (lg + B), h->gcnt[g], lg + B, stwo_tables(h->tw[g], lg + B), h->co[g],
                             lg};
        }
        VX_CUDA_TRY(ntt_transform_groups(gi, h->n_groups, false, st, launches));
        VX_CUDA_TRY(ntt_transform_groups(ge, h->n_groups, true, st, launches));
        break;
    }
    case 1:  // lifted tree over the LDE rows, mix its root, draw alpha
        VX_CUDA_TRY(lifted_tree_build(h->cols, h->lv0, ChanStep{h->chan, proof + L.r0, h->alpha}, st));
        *launches += tree_launches(h->lv0);
        break;
    case 2: {  // C = sum alpha^c lift(col_c), committed; draw the first fold challenge
        powers_kernel<<<1, 32, 0, st>>>(h->alpha, h->pw, L.n_cols);
        CombineGroupsArgs ca;
        memset(&ca, 0, sizeof(ca));
        LeafCombine lc;
        memset(&lc, 0, sizeof(lc));
        uint64_t rows = 0;
        for (uint32_t g = 0; g < h->n_groups; g++) {
            const uint32_t le = h->glog[g] + B;
            const bool top = g + 1 == h->n_groups;  // le == S
            ca.lde[g] = h->lde[g];
            ca.dst[g] = top ? h->C[0] : h->G[g];
            ca.dstride[g] = top ? align64(1ull << S) : align64(1ull << le);
            rows += 1ull << le;
            ca.rows_end[g] = rows;
            ca.le[g] = le; ca.cnt[g] = h->gcnt[g]; ca.first[g] = h->gfirst[g];
            if (!top) {
                lc.g[lc.n_small] = h->G[g];
                lc.gstride[lc.n_small] = align64(1ull << le);
                lc.gshift[lc.n_small] = S - le + 1u;
                lc.n_small++;
            }
        }
        ca.n_groups = h->n_groups;
        VX_CUDA_TRY(launch_pdl(combine_groups_kernel, dim3(blocks_for(rows / 4, 256)), dim3(256), 0, st, ca,
                               (const uint32_t *)h->pw));
        lc.o0 = h->C[0]; lc.o1 = h->C[1]; lc.o2 = h->C[2]; lc.o3 = h->C[3];
        VX_CUDA_TRY(tree_build(lc, h->lv1, ChanStep{h->chan, proof + L.r1, h->alpha_f}, st));
        *launches += 2 + tree_launches(h->lv1);
        break;
    }
    case 3: {  // circle fold of C (stwo twiddles) into FRI layer 0
        LeafFold cf{h->C[0], h->C[1], h->C[2], h->C[3], h->fold_circle, h->alpha_f,
                    h->F[0][0], h->F[0][1], h->F[0][2], h->F[0][3], {}};
        VX_CUDA_TRY(tree_build(cf, h->flv[0],
                               ChanStep{h->chan, proof + L.froots, L.nfri > 1 ? h->alpha_f + 4 : nullptr}, st));
        *launches += tree_launches(h->flv[0]);
        break;
    }
    case 4:  // line folds
        for (uint32_t k = 1; k < L.nfri; k++) {
            const uint32_t lsrc = S - k;
            LeafFold lf{h->F[k - 1][0], h->F[k - 1][1], h->F[k - 1][2], h->F[k - 1][3],
                        h->fold_line + h->fold_line_off[lsrc], h->alpha_f + 4 * k,
                        h->F[k][0], h->F[k][1], h->F[k][2], h->F[k][3], {}};
            VX_CUDA_TRY(tree_build(lf, h->flv[k],
                                   ChanStep{h->chan, proof + L.froots + 8 * k,
                                            k + 1 < L.nfri ? h->alpha_f + 4 * (k + 1) : nullptr},
                                   st));
            *launches += tree_launches(h->flv[k]);
        }
        break;
    case 5: {
        const uint32_t kl = L.nfri - 1;
        lift_queries_kernel<<<1, 128, 0, st>>>(h->chan, h->F[kl][0], h->F[kl][1], h->F[kl][2], h->F[kl][3],
                                               proof + L.last, S, L.nq, h->qidx, proof + L.qidx);
        *launches += 1;
        break;
    }
    case 6: {
        LiftValuesArgs va;
        memset(&va, 0, sizeof(va));
        va.cols = h->cols;
        va.nfri = L.nfri;
        for (int c = 0; c < 4; c++) va.C[c] = h->C[c];
        va.vals[0] = L.lift.vals; va.svals[0] = L.lift.svals;
        va.vals[1] = L.comb.vals; va.svals[1] = L.comb.svals;
        for (uint32_t k = 0; k < L.nfri; k++) {
            for (int c = 0; c < 4; c++) va.F[k][c] = h->F[k][c];
            va.vals[2 + k] = L.fri[k].vals; va.svals[2 + k] = L.fri[k].svals;
        }
        lift_values_kernel<<<blocks_for((uint64_t)(2 + L.nfri) * L.nq, 128), 128, 0, st>>>(va, h->qidx, L.nq, proof);
        LiftPathsArgs pa;
        memset(&pa, 0, sizeof(pa));
        pa.cols = h->cols;
        uint32_t max_groups = 0;
        auto add = [&](uint32_t i, const TreeLevels &lv, uint32_t kind, uint32_t shift, uint32_t *const *c,
                       const DecomLayout &d) {
            pa.t[i].lv = lv; pa.t[i].kind = kind; pa.t[i].shift = shift;
            for (int w = 0; w < 4; w++) pa.t[i].c[w] = c ? c[w] : nullptr;
            pa.t[i].paths = d.paths; pa.t[i].spaths = d.spaths;
            if (lv.n - 1 > max_groups) max_groups = lv.n - 1;
        };
        add(0, h->lv0, 0, 0, nullptr, L.lift);
        add(1, h->lv1, 1, 0, h->C, L.comb);
        for (uint32_t k = 0; k < L.nfri; k++) add(2 + k, h->flv[k], 1, k + 1, h->F[k], L.fri[k]);
        dim3 grid(blocks_for((uint64_t)L.nq * max_groups, 64), 2 + L.nfri);
        lift_paths_kernel<<<grid, 64, 0, st>>>(pa, h->qidx, L.nq, proof);
        *launches += 2;
        break;
    }
    default:
        set_last_error(VX_ERR_ARG, "unknown lifted-commitment stage %u", stage);
        return VX_ERR_ARG;
    }
    VX_CUDA_TRY(cudaGetLastError());
    return VX_OK;
}

constexpr uint32_t kLiftStages = 7;

std::mutex g_lift_mu;
std::vector<vx_lifted *> g_lift_cache;

}  // namespace

extern "C" size_t vx_lifted_size(uint32_t n_cols, const uint32_t *log_sizes, uint32_t blowup_bits,
                                 uint32_t n_queries) {
    LiftLayout L;
    if (!lift_layout(n_cols, log_sizes, blowup_bits, n_queries, &L)) return 0;
    return (size_t)L.words * 4;
}

extern "C" void vx_lifted_destroy(vx_lifted *h) {
    if (!h) return;
    if (h->exec) cudaGraphExecDestroy(h->exec);
    if (h->st) cudaStreamDestroy(h->st);
    if (h->block) cudaFree(h->block);
    delete h;
}

extern "C" int vx_lifted_create(uint32_t n_cols, const uint32_t *log_sizes, uint32_t blowup_bits,
                                uint32_t n_queries, vx_lifted **out) {
    VX_CHECK_ARG(out != nullptr, "vx_lifted_create: out is null");
    auto *h = new vx_lifted();
    if (!lift_layout(n_cols, log_sizes, blowup_bits, n_queries, &h->L)) {
        delete h;
        set_last_error(VX_ERR_ARG,
                       "vx_lifted_create: need 1..64 columns in ascending log size, 2 <= log, log + blowup <= 28, "
                       "blowup in 1..4, 1..1024 queries");
        return VX_ERR_ARG;
    }
    cudaGetDevice(&h->device);
    const LiftLayout &L = h->L;
    const uint32_t B = L.B, S = L.S;
    // size groups
    for (uint32_t c = 0; c < n_cols; c++) {
        if (c == 0 || L.logs[c] != L.logs[c - 1]) {
            h->glog[h->n_groups] = L.logs[c];
            h->gfirst[h->n_groups] = c;
            h->gcnt[h->n_groups] = 0;
            h->n_groups++;
        }
        h->gcnt[h->n_groups - 1]++;
    }
    // carve one allocation
    uint64_t w = 0;
    uint64_t o_in[kMaxLiftCols], o_co[kMaxLiftCols], o_lde[kMaxLiftCols], o_itw[kMaxLiftCols], o_tw[kMaxLiftCols];
    for (uint32_t g = 0; g < h->n_groups; g++) {
        const uint32_t lg = h->glog[g], cnt = h->gcnt[g];
        o_in[g] = w; w += align64((uint64_t)cnt << lg);
        o_co[g] = w; w += align64((uint64_t)cnt << lg);
        o_lde[g] = w; w += align64((uint64_t)cnt << (lg + B));
        o_itw[g] = w; w += align64(1ull << (lg - 1));
        o_tw[g] = w; w += align64(1ull << (lg + B - 1));
    }
    const uint64_t o_fc = w; w += align64(1ull << (S - 1));
    const uint64_t o_fl = w;
    for (uint32_t l = S - 1; l >= 4; l--) { h->fold_line_off[l] = w - o_fl; w += align64(1ull << (l - 1)); }
    uint64_t o_C = w; w += 4 * align64(1ull << S);
    uint64_t o_G[kMaxLiftCols];
    for (uint32_t g = 0; g + 1 < h->n_groups; g++) { o_G[g] = w; w += 4 * align64(1ull << (h->glog[g] + B)); }
    uint64_t o_F[kMaxFri];
    for (uint32_t k = 0; k < L.nfri; k++) { o_F[k] = w; w += 4 * align64(1ull << (S - 1 - k)); }
    // leaf-kernel shapes read once: the pools are sized and carved with them
    const uint32_t kt = tree_leaf_k(S, kLeafFold);  // 34-word rows and combinations: wide leaves
    uint32_t kf[kMaxFri];
    for (uint32_t k = 0; k < L.nfri; k++) kf[k] = tree_leaf_k(S - 1 - k, kLeafFold);
    const uint64_t o_t0 = w; w += align64(tree_pool_words(S, kt));
    const uint64_t o_t1 = w; w += align64(tree_pool_words(S, kt));
    uint64_t o_ft[kMaxFri];
    for (uint32_t k = 0; k < L.nfri; k++) { o_ft[k] = w; w += align64(tree_pool_words(S - 1 - k, kf[k])); }
    const uint64_t o_ch = w; w += align64(sizeof(DevChannel) / 4 + 1);
    const uint64_t o_al = w; w += align64(4);
    const uint64_t o_af = w; w += align64(4ull * (L.nfri + 1));
    const uint64_t o_pw = w; w += align64(4ull * kMaxLiftCols);
    const uint64_t o_qi = w; w += align64(L.nq);
    const uint64_t o_pf = w; w += align64(L.words);
    if (cudaMalloc(&h->block, w * 4) != cudaSuccess) {
        cudaGetLastError();
        delete h;
        set_last_error(VX_ERR_OOM, "cudaMalloc of %llu bytes for a lifted commitment failed",
                       (unsigned long long)(w * 4));
        return VX_ERR_OOM;
    }
    h->bytes = w * 4;
    uint32_t *b = (uint32_t *)h->block;
    for (uint32_t g = 0; g < h->n_groups; g++) {
        h->in[g] = b + o_in[g]; h->co[g] = b + o_co[g]; h->lde[g] = b + o_lde[g];
        h->itw[g] = b + o_itw[g]; h->tw[g] = b + o_tw[g];
    }
    h->fold_circle = b + o_fc;
    h->fold_line = b + o_fl;
    for (int c = 0; c < 4; c++) h->C[c] = b + o_C + c * align64(1ull << S);
    for (uint32_t g = 0; g + 1 < h->n_groups; g++) h->G[g] = b + o_G[g];
    for (uint32_t k = 0; k < L.nfri; k++)
        for (int c = 0; c < 4; c++) h->F[k][c] = b + o_F[k] + c * align64(1ull << (S - 1 - k));
    tree_plan(S, b + o_t0, &h->lv0, kt);
    tree_plan(S, b + o_t1, &h->lv1, kt);
    for (uint32_t k = 0; k < L.nfri; k++) tree_plan(S - 1 - k, b + o_ft[k], &h->flv[k], kf[k]);
    h->chan = (DevChannel *)(b + o_ch);
    h->alpha = b + o_al;
    h->alpha_f = b + o_af;
    h->pw = b + o_pw;
    h->qidx = b + o_qi;
    h->proof = b + o_pf;
    // the lifted leaf source: every LDE column with its lift shift
    memset(&h->cols, 0, sizeof(h->cols));
    h->cols.n_cols = n_cols;
    for (uint32_t g = 0; g < h->n_groups; g++)
        for (uint32_t j = 0; j < h->gcnt[g]; j++) {
            const uint32_t c = h->gfirst[g] + j, le = h->glog[g] + B;
            h->cols.col[c] = h->lde[g] + ((uint64_t)j << le);
            h->cols.shift[c] = S - le + 1u;  // 1 when le == S: the row is then the index itself
        }
    // constant tables and words
    GenTables gt;
    cudaError_t e = gen_tables_get(&gt);
    for (uint32_t g = 0; g < h->n_groups && e == cudaSuccess; g++) {
        e = build_stwo_table_with(gt, h->glog[g], true, h->itw[g], nullptr);
        if (e == cudaSuccess) e = build_stwo_table_with(gt, h->glog[g] + B, false, h->tw[g], nullptr);
    }
    if (e == cudaSuccess) e = build_stwo_fold_circle_with(gt, S, h->fold_circle, nullptr);
    for (uint32_t l = S - 1; l >= 4 && e == cudaSuccess; l--)
        e = build_fold_twiddles_with(gt, ecoset_half_odds(l), false, h->fold_line + h->fold_line_off[l], nullptr);
    std::vector<uint32_t> tmpl;
    lift_template(L, tmpl);
    if (e == cudaSuccess) e = cudaMemcpy(h->proof, tmpl.data(), L.words * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = tree_reset(h->lv0, nullptr);
    if (e == cudaSuccess) e = tree_reset(h->lv1, nullptr);
    for (uint32_t k = 0; k < L.nfri && e == cudaSuccess; k++) e = tree_reset(h->flv[k], nullptr);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamSynchronize(nullptr);
    if (e != cudaSuccess) {
        set_last_error(VX_ERR_CUDA, "vx_lifted_create: %s", cudaGetErrorString(e));
        vx_lifted_destroy(h);
        return VX_ERR_CUDA;
    }
    *out = h;
    return VX_OK;
}

extern "C" int vx_lifted_column(vx_lifted *h, uint32_t c, uint32_t **dev_ptr) {
    VX_CHECK_ARG(h != nullptr && dev_ptr != nullptr, "vx_lifted_column: null argument");
    VX_CHECK_ARG(c < h->L.n_cols, "vx_lifted_column: column %u of %u", c, h->L.n_cols);
    for (uint32_t g = 0; g < h->n_groups; g++)
        if (c >= h->gfirst[g] && c < h->gfirst[g] + h->gcnt[g]) {
            *dev_ptr = h->in[g] + ((uint64_t)(c - h->gfirst[g]) << h->glog[g]);
            return VX_OK;
        }
    return VX_ERR_ARG;
}

extern "C" int vx_lifted_upload_async(vx_lifted *h, const uint32_t *const *host_cols, void *stream) {
    VX_CHECK_ARG(h != nullptr && host_cols != nullptr, "vx_lifted_upload_async: null argument");
    for (uint32_t c = 0; c < h->L.n_cols; c++) {
        VX_CHECK_ARG(host_cols[c] != nullptr, "vx_lifted_upload_async: column %u is null", c);
        uint32_t *d = nullptr;
        int rc = vx_lifted_column(h, c, &d);
        if (rc) return rc;
        VX_CUDA_TRY(cudaMemcpyAsync(d, host_cols[c], 4ull << h->L.logs[c], cudaMemcpyHostToDevice,
                                    (cudaStream_t)stream));
    }
    return VX_OK;
}

extern "C" int vx_lifted_stage_async(vx_lifted *h, uint32_t stage, void *stream) {
    VX_CHECK_ARG(h != nullptr, "vx_lifted_stage_async: null handle");
    uint32_t launches = 0;
    return lift_stage(h, stage, (cudaStream_t)stream, &launches);
}

extern "C" int vx_lifted_commit_async(vx_lifted *h, void *stream) {
    VX_CHECK_ARG(h != nullptr, "vx_lifted_commit_async: null handle");
    uint32_t launches = 0;
    for (uint32_t s = 0; s < kLiftStages; s++) {
        int rc = lift_stage(h, s, (cudaStream_t)stream, &launches);
        if (rc) return rc;
    }
    h->launches = launches;
    return VX_OK;
}

extern "C" int vx_lifted_commit_graph(vx_lifted *h, void *stream) {
    VX_CHECK_ARG(h != nullptr, "vx_lifted_commit_graph: null handle");
    if (!h->exec) {
        uint32_t launches = 0;
        VX_CUDA_TRY(cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal));
        int rc = VX_OK;
        for (uint32_t s = 0; s < kLiftStages && rc == VX_OK; s++) rc = lift_stage(h, s, h->st, &launches);
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamEndCapture(h->st, &graph);
        if (rc) { if (graph) cudaGraphDestroy(graph); return rc; }
        VX_CUDA_TRY(e);
        e = cudaGraphInstantiate(&h->exec, graph, 0);
        cudaGraphDestroy(graph);
        VX_CUDA_TRY(e);
        h->launches = launches;
    }
    VX_CUDA_TRY(cudaGraphLaunch(h->exec, (cudaStream_t)stream));
    return VX_OK;
}

extern "C" int vx_lifted_fetch_async(vx_lifted *h, void *dst, void *stream) {
    VX_CHECK_ARG(h != nullptr && dst != nullptr, "vx_lifted_fetch_async: null argument");
    VX_CUDA_TRY(cudaMemcpyAsync(dst, h->proof, h->L.words * 4, cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    return VX_OK;
}

extern "C" int vx_lifted_check(vx_lifted *h) {
    VX_CHECK_ARG(h != nullptr, "vx_lifted_check: null handle");
    uint32_t err = 0;
    VX_CUDA_TRY(cudaMemcpy(&err, &h->chan->err, 4, cudaMemcpyDeviceToHost));
    if (err) {
        set_last_error(VX_ERR_DEVICE, "transcript rejection sampling exceeded its bound");
        return VX_ERR_DEVICE;
    }
    return VX_OK;
}

extern "C" uint32_t vx_lifted_launches(const vx_lifted *h) { return h ? h->launches : 0u; }
extern "C" size_t vx_lifted_device_bytes(const vx_lifted *h) { return h ? h->bytes : 0u; }

extern "C" int vx_commit_lifted(const uint32_t *const *host_cols, const uint32_t *log_sizes, uint32_t n_cols,
                                uint32_t blowup_bits, uint32_t n_queries, uint8_t *out, size_t cap,
                                size_t *out_len) {
    VX_CHECK_ARG(host_cols != nullptr && log_sizes != nullptr && out != nullptr && out_len != nullptr,
                 "vx_commit_lifted: null argument");
    const size_t need = vx_lifted_size(n_cols, log_sizes, blowup_bits, n_queries);
    VX_CHECK_ARG(need != 0, "vx_commit_lifted: unsupported shape (1..64 columns in ascending log size, "
                            "2 <= log, log + blowup <= 28, blowup 1..4, 1..1024 queries)");
    VX_CHECK_ARG(cap >= need, "vx_commit_lifted: output capacity %zu < %zu", cap, need);
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(g_lift_mu);
    vx_lifted *h = nullptr;
    for (vx_lifted *c : g_lift_cache) {
        if (c->device != dev || c->L.n_cols != n_cols || c->L.B != blowup_bits || c->L.nq != n_queries) continue;
        if (memcmp(c->L.logs, log_sizes, 4ull * n_cols) == 0) { h = c; break; }
    }
    if (!h) {
        int rc = vx_lifted_create(n_cols, log_sizes, blowup_bits, n_queries, &h);
        if (rc) return rc;
        g_lift_cache.push_back(h);
    }
    int rc = vx_lifted_upload_async(h, host_cols, nullptr);
    if (!rc) rc = vx_lifted_commit_async(h, nullptr);
    if (!rc) rc = vx_lifted_fetch_async(h, out, nullptr);
    if (rc) return rc;
    VX_CUDA_TRY(cudaStreamSynchronize(nullptr));
    rc = vx_lifted_check(h);
    if (rc) return rc;
    *out_len = need;
    return VX_OK;
}

extern "C" void vx_lifted_release_all(void) {
    std::lock_guard<std::mutex> lk(g_lift_mu);
    for (vx_lifted *h : g_lift_cache) vx_lifted_destroy(h);
    g_lift_cache.clear();
}
