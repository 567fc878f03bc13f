// Device-resident Fibonacci prover (prover.rs:264-619 restated for B200).
//
// One proof is a fixed sequence of kernels on one stream with no host
// synchronisation: trace generation, iNTT, LDE, trace commitment, quotient
// commitment (quotient recomputed from the LDE inside the hashing kernel),
// circle fold fused with the first FRI commitment, line folds fused with their
// commitments, the Fiat-Shamir transcript on the device, query sampling and
// decommitment written straight into the proof's byte layout.
#include <cstdarg>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "vx_common.cuh"
#include "vx_field.cuh"
#include "vx_fri.cuh"
#include "vx_merkle.cuh"
#include "vx_ntt.cuh"
#include "vx_prover.cuh"
#include "vx_twiddles.cuh"

namespace vx {

// ---------------------------------------------------------------------
// proof layout (stark_cli.rs:1092-1123)
// ---------------------------------------------------------------------
static void decom_layout(DecomLayout *d, uint64_t *w, uint32_t nq, uint32_t width, uint32_t depth) {
    d->width = width; d->depth = depth;
    d->n = (*w)++;
    d->vals = *w; *w += (uint64_t)nq * width;
    d->svals = *w; *w += (uint64_t)nq * width;
    d->paths = *w; *w += (uint64_t)nq * (1 + 8ull * depth);
    d->spaths = *w; *w += (uint64_t)nq * (1 + 8ull * depth);
}

void proof_layout(uint32_t log_n, uint32_t blowup, uint32_t nq, ProofLayout *L) {
    memset(L, 0, sizeof(*L));
    L->log_n = log_n; L->blowup = blowup; L->le = log_n + blowup; L->nfri = L->le - 3; L->nq = nq;
    uint64_t w = 0;
    L->magic = w; w += 5;                 // magic, version, log_n, a, b
    L->troot = w; w += 8;
    L->qroot = w; w += 8;
    L->nfri_w = w++;
    L->froots = w; w += 8ull * L->nfri;
    L->nlast = w++;
    L->last = w; w += 32;
    L->nq_w = w++;
    L->qidx = w; w += nq;
    decom_layout(&L->trace, &w, nq, 1, L->le);
    decom_layout(&L->quot, &w, nq, 4, L->le);
    L->nfd = w++;
    for (uint32_t k = 0; k < L->nfri; k++) decom_layout(&L->fri[k], &w, nq, 4, L->le - 1 - k);
    L->words = w;
}

// Constant words of the layout (everything except a, b, roots, last layer,
// query indices, values and path hashes).
// `t` holds L.words words; both the allocating path and the no-allocation
// entry point fill their staging buffer here.
static void proof_template(const ProofLayout &L, uint32_t *t) {
    memset(t, 0, (size_t)L.words * 4);
    t[L.magic] = 0x4B52414Bu; t[L.magic + 1] = 1u; t[L.magic + 2] = L.log_n;
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
    dec(L.trace); dec(L.quot);
    t[L.nfd] = L.nfri;
    for (uint32_t k = 0; k < L.nfri; k++) dec(L.fri[k]);
}

// ---------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------
namespace {

// Chunk seeds by matrix powers, as the reference's parallel trace does
// (air.rs:85-131).  Standard Fibonacci numbers mod P, built at compile time: fib(k - 1),
// fib(k), fib(k + 1) for k = 32 t (t < 256) and for k = 2^j (j < 32).
// With G(k) = a fib(k - 1) + b fib(k), the sequence from (a, b) satisfies
// G(s + k) = G(s) fib(k - 1) + G(s + 1) fib(k) and
// G(s + k + 1) = G(s) fib(k) + G(s + 1) fib(k + 1).
struct FibTab { uint32_t chunk[256][3]; uint32_t pow2[32][3]; };
constexpr uint32_t cadd_(uint32_t x, uint32_t y) { return (uint32_t)(((uint64_t)x + y) % VX_P); }
constexpr uint32_t cmul_(uint32_t x, uint32_t y) { return (uint32_t)(((uint64_t)x * y) % VX_P); }
constexpr FibTab make_fib_tab() {
    FibTab t{};
    uint32_t f0 = 1, f1 = 0;  // fib(-1), fib(0)
    for (uint32_t k = 0; k <= 8192; k++) {   // at step k: f0 = fib(k - 1), f1 = fib(k)
        if (k % 32 == 0 && k / 32 < 256) {
            t.chunk[k / 32][0] = f0; t.chunk[k / 32][1] = f1; t.chunk[k / 32][2] = cadd_(f0, f1);
        }
        const uint32_t f2 = cadd_(f0, f1);
        f0 = f1; f1 = f2;
    }
    // the matrix [[fib(k+1), fib(k)], [fib(k), fib(k-1)]] squared gives 2k
    uint32_t m = 0, p = 1, q = 1;  // fib(k-1), fib(k), fib(k+1) for k = 1
    for (uint32_t j = 0; j < 32; j++) {
        t.pow2[j][0] = m; t.pow2[j][1] = p; t.pow2[j][2] = q;
        const uint32_t m2 = cadd_(cmul_(p, p), cmul_(m, m)), p2 = cadd_(cmul_(q, p), cmul_(p, m)),
                       q2 = cadd_(cmul_(q, q), cmul_(p, p));
        m = m2; p = p2; q = q2;
    }
    return t;
}
__constant__ FibTab kFib = make_fib_tab();

// (G(s + k), G(s + k + 1)) from (G(s), G(s + 1)) and (fib(k-1), fib(k), fib(k+1)).
__device__ __forceinline__ void fib_step(uint32_t &g0, uint32_t &g1, const uint32_t f[3]) {
    const uint32_t n0 = madd(mmul(g0, f[0]), mmul(g1, f[1]));
    const uint32_t n1 = madd(mmul(g0, f[1]), mmul(g1, f[2]));
    g0 = n0; g1 = n1;
}

// Fibonacci trace t0 = a, t1 = b, t_{i+2} = t_i + t_{i+1} (air.rs:16-25).
// A block of 256 threads writes 8192 rows: thread 0 builds the block's seed
// (G(base), G(base + 1)) from the powers-of-two table, every thread derives
// its 32-row chunk's seed with one table step, runs the recurrence into
// shared memory, and the block writes its rows coalesced.  Also stamps
// (a, b) into the proof header.
constexpr uint32_t kTraceRows = 8192;
__global__ void __launch_bounds__(256) fib_trace_kernel(uint32_t a, uint32_t b, const uint32_t *ab_dev, uint32_t *out,
                                                        uint64_t n, uint32_t *proof_ab) {
    __shared__ uint32_t rows[256 * 33];
    __shared__ uint32_t seed[2];
    if (ab_dev) { a = ab_dev[0]; b = ab_dev[1]; }
    if (blockIdx.x == 0 && threadIdx.x == 0) { proof_ab[0] = a; proof_ab[1] = b; }
    const uint64_t base = (uint64_t)blockIdx.x * kTraceRows;
    if (threadIdx.x == 0) {
        uint32_t g0 = a, g1 = b;
        for (uint32_t j = 13; j < 32 && (base >> j); j++)  // base < 2^31
            if ((base >> j) & 1ull) fib_step(g0, g1, kFib.pow2[j]);
        seed[0] = g0; seed[1] = g1;
    }
    __syncthreads();
    const uint32_t t = threadIdx.x;
    uint32_t f0 = seed[0], f1 = seed[1];
    fib_step(f0, f1, kFib.chunk[t]);
    uint32_t *r = rows + 33 * t;
    r[0] = f0;
    r[1] = f1;
#pragma unroll
    for (uint32_t i = 2; i < 32; i++) {
        const uint32_t f2 = madd(f0, f1);
        r[i] = f2;
        f0 = f1; f1 = f2;
    }
    __syncthreads();
    const uint64_t cnt = (n - base) < kTraceRows ? (n - base) : kTraceRows;
    for (uint32_t e = t; e < cnt; e += 256) out[base + e] = rows[33 * (e >> 5) + (e & 31u)];
}

// mix_felts(last layer) (channel.rs:46-59) then n_queries x draw_number(N)
// (channel.rs:93-97, prover.rs:1056-1059).  Draw j squeezes with
// n_draws = j, so the draws run in parallel.
__global__ void chan_queries_kernel(DevChannel *ch, const uint32_t *l0, const uint32_t *l1, const uint32_t *l2,
                                    const uint32_t *l3, uint32_t *proof_last, uint64_t bound, uint32_t nq,
                                    uint32_t *qidx, uint32_t *proof_qidx) {
    __shared__ uint32_t st[8];
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
        ch->n_draws = nq;
    }
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < nq; j += blockDim.x) {
        uint32_t w[8];
        chan_squeeze(st, j, w);
        uint64_t raw = (uint64_t)w[0] | ((uint64_t)w[1] << 32);
        uint32_t v = (uint32_t)(raw % bound);
        qidx[j] = v;
        proof_qidx[j] = v;
    }
}

// ---- fused fold + commitment leaf sources (fri.cu:58-126) ----
// Circle fold of the quotient into FRI layer 0: output j pairs q[2j], q[2j+1].
// Both values are alpha_q times an M31 word (c0, c1), so
//   (f0 + f1) + alpha_f tw (f0 - f1) = alpha_q s + beta d,
// with s = c0 + c1, d = tw (c0 - c1) in M31 and beta = alpha_f alpha_q
// formed once per thread: each output word is a dot product of two
// products, reduced once (the same field values as folding the two QM31s).
struct LeafCircleFold {
    LeafQuotient q;
    const uint32_t *tw;
    const uint32_t *alpha_ptr;
    uint32_t *o0, *o1, *o2, *o3;
    uint32_t beta[4];
    __device__ __forceinline__ void init() {
        q.init();
        const qm31 b = qmul(qm31{{alpha_ptr[0], alpha_ptr[1], alpha_ptr[2], alpha_ptr[3]}},
                            qm31{{q.al[0], q.al[1], q.al[2], q.al[3]}});
#pragma unroll
        for (int c = 0; c < 4; c++) beta[c] = b.v[c];
    }
    __device__ __forceinline__ uint32_t load(uint64_t j, uint32_t m[16]) const {
        const uint64_t i = 2 * j, mk = q.mask;
        const uint32_t t0 = __ldg(q.eval + i), t1 = __ldg(q.eval + ((i + 1) & mk));
        const uint32_t t2 = __ldg(q.eval + ((i + 2) & mk)), t3 = __ldg(q.eval + ((i + 3) & mk));
        const uint32_t c0 = msub(t2, madd(t1, t0)), c1 = msub(t3, madd(t2, t1));
        const uint32_t s = madd(c0, c1), d = mmul(msub(c0, c1), __ldg(tw + j));
        qm31 r;
#pragma unroll
        for (int c = 0; c < 4; c++) r.v[c] = reduce64((uint64_t)q.al[c] * s + (uint64_t)beta[c] * d);
        o0[j] = r.v[0]; o1[j] = r.v[1]; o2[j] = r.v[2]; o3[j] = r.v[3];
        m[0] = r.v[0]; m[1] = r.v[1]; m[2] = r.v[2]; m[3] = r.v[3];
        return 16u;
    }
};

// Line fold of FRI layer k-1 into layer k.
using LeafLineFold = LeafFold;

// Query values and sibling values of every committed column, written
// into the proof.  Thread (tree, q): tree 0 = trace, 1 = quotient, 2 + k
// = FRI layer k.
struct ValuesArgs {
    const uint32_t *eval;
    uint64_t mask;
    const uint32_t *alpha_q;
    const uint32_t *fri[32][4];
    uint64_t vals[34], svals[34];
    uint32_t nfri;
};
__global__ void decommit_values_kernel(ValuesArgs a, const uint32_t *qidx, uint32_t nq, uint32_t *proof) {
    uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t ntree = 2 + a.nfri;
    if (tid >= ntree * nq) return;
    uint32_t tree = tid / nq, q = tid % nq;
    uint64_t i = qidx[q];
    if (tree == 0) {
        proof[a.vals[0] + q] = a.eval[i];
        proof[a.svals[0] + q] = a.eval[i ^ 1];
    } else if (tree == 1) {
        LeafQuotient src{a.eval, a.mask, a.alpha_q, {0, 0, 0, 0}};
        src.init();
        qm31 v = src.value(i), s = src.value(i ^ 1);
        for (int c = 0; c < 4; c++) { proof[a.vals[1] + 4 * q + c] = v.v[c]; proof[a.svals[1] + 4 * q + c] = s.v[c]; }
    } else {
        uint32_t k = tree - 2;
        uint64_t j = i >> (k + 1);
        for (int c = 0; c < 4; c++) {
            proof[a.vals[tree] + 4 * q + c] = a.fri[k][c][j];
            proof[a.svals[tree] + 4 * q + c] = a.fri[k][c][j ^ 1];
        }
    }
}

// All authentication paths of a proof in one launch: blockIdx.y selects the
// tree (0 trace, 1 quotient, 2 + k FRI layer k), threads cover
// (query, stored-level group) pairs of that tree.
struct PathTree {
    TreeLevels lv;
    uint32_t kind;    // 0: M31 eval column, 1: quotient from eval, 2: SoA4 layer
    uint32_t shift;   // query index >> shift is the leaf index
    const uint32_t *c[4];
    uint64_t paths, spaths;
};
struct PathsArgs {
    PathTree t[34];
    const uint32_t *eval;
    uint64_t mask;
    const uint32_t *alpha_q;
};
__global__ void __launch_bounds__(64) decommit_all_kernel(const __grid_constant__ PathsArgs a, const uint32_t *qidx,
                                                          uint32_t nq, uint32_t *proof) {
    const PathTree &T = a.t[blockIdx.y];
    uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t ng = T.lv.n - 1;
    if (tid >= nq * ng) return;
    uint32_t q = tid / ng, g = tid % ng;
    uint32_t depth = T.lv.height[T.lv.n - 1];
    uint64_t idx = (uint64_t)qidx[q] >> T.shift;
    uint32_t lo = T.lv.height[g], k = T.lv.height[g + 1] - lo;
    uint64_t node = idx >> lo;
    uint64_t blk = node >> k;
    const uint32_t K = 1u << k;
    uint32_t nh[31][8];
    if (g == 0) {
        LeafQuotient lq{a.eval, a.mask, a.alpha_q, {0, 0, 0, 0}};
        if (T.kind == 1) lq.init();
        for (uint32_t j = 0; j < K; j++) {
            uint32_t m[16];
#pragma unroll
            for (int w = 0; w < 16; w++) m[w] = 0u;
            uint64_t i = (blk << k) + j;
            uint32_t nb;
            if (T.kind == 0) { m[0] = T.c[0][i]; nb = 4u; }
            else if (T.kind == 1) { nb = lq.load(i, m); }
            else { m[0] = T.c[0][i]; m[1] = T.c[1][i]; m[2] = T.c[2][i]; m[3] = T.c[3][i]; nb = 16u; }
            blake2s_block(nh[j], m, nb);
        }
    } else {
        const uint32_t *h = T.lv.hashes[g] + 8ull * (blk << k);
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
    uint32_t *p = proof + T.paths + (uint64_t)q * (1u + 8u * depth);
    uint32_t *sp = proof + T.spaths + (uint64_t)q * (1u + 8u * depth);
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
}

}  // namespace

// ---------------------------------------------------------------------
// tables and slots
// ---------------------------------------------------------------------
static uint64_t align_words(uint64_t w) { return (w + 63) & ~63ull; }  // 256-byte alignment

static int tables_create(int device, uint32_t log_n, uint32_t blowup, SizeTables **out) {
    auto *t = new SizeTables();
    memset(t, 0, sizeof(*t));
    t->device = device; t->log_n = log_n; t->blowup = blowup; t->le = log_n + blowup;
    uint64_t n = 1ull << log_n, N = 1ull << t->le;
    uint64_t w = 0;
    uint64_t o_itl = w; w += align_words(n - 1);
    uint64_t o_itc = w; w += align_words(n / 2);
    uint64_t o_ftl = w; w += align_words(N - 1);
    uint64_t o_ftc = w; w += align_words(N / 2);
    uint64_t o_fc = w; w += align_words(N / 2);
    uint64_t o_fl = w;
    for (uint32_t l = t->le - 1; l >= 4; l--) { t->fold_line_off[l] = w - o_fl; w += align_words(1ull << (l - 1)); }
    void *blk = nullptr;
    if (cudaMalloc(&blk, w * 4) != cudaSuccess) {
        cudaGetLastError();
        delete t;
        set_last_error(VX_ERR_OOM, "cudaMalloc of %llu bytes for twiddle tables failed", (unsigned long long)(w * 4));
        return VX_ERR_OOM;
    }
    uint32_t *b = (uint32_t *)blk;
    t->block = blk;
    t->itw_line = b + o_itl; t->itw_circle = b + o_itc;
    t->ftw_line = b + o_ftl; t->ftw_circle = b + o_ftc;
    t->fold_circle = b + o_fc; t->fold_line = b + o_fl;
    ntt_table_offsets(log_n, t->itw_off);
    ntt_table_offsets(t->le, t->ftw_off);
    cudaStream_t s = nullptr;
    cudaError_t e = build_ntt_tables(ecoset_half_coset(log_n), true, t->itw_line, t->itw_circle, s);
    if (e == cudaSuccess) e = build_ntt_tables(ecoset_eval_domain(t->le), false, t->ftw_line, t->ftw_circle, s);
    if (e == cudaSuccess) e = build_fold_twiddles(ecoset_eval_domain(t->le), true, t->fold_circle, s);
    for (uint32_t l = t->le - 1; l >= 4 && e == cudaSuccess; l--)
        e = build_fold_twiddles(ecoset_half_odds(l), false, t->fold_line + t->fold_line_off[l], s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        cudaFree(blk);
        delete t;
        set_last_error(VX_ERR_CUDA, "building twiddle tables: %s", cudaGetErrorString(e));
        return VX_ERR_CUDA;
    }
    *out = t;
    return VX_OK;
}

static void tables_destroy(SizeTables *t) {
    if (!t) return;
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(t->device);
    cudaFree(t->block);
    cudaSetDevice(cur);
    delete t;
}

static size_t tables_bytes(const SizeTables *t) {
    uint64_t n = 1ull << t->log_n, N = 1ull << t->le;
    uint64_t w = align_words(n - 1) + align_words(n / 2) + align_words(N - 1) + align_words(N / 2) + align_words(N / 2);
    for (uint32_t l = t->le - 1; l >= 4; l--) w += align_words(1ull << (l - 1));
    return (size_t)(w * 4);
}

// Per-(device, log_n, blowup) shared tables.
static std::mutex g_tab_mu;
static std::map<std::tuple<int, uint32_t, uint32_t>, std::pair<SizeTables *, int>> g_tables;

static int tables_acquire(uint32_t log_n, uint32_t blowup, SizeTables **out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) { set_last_error(VX_ERR_CUDA, "cudaGetDevice failed"); return VX_ERR_CUDA; }
    std::lock_guard<std::mutex> lk(g_tab_mu);
    auto key = std::make_tuple(dev, log_n, blowup);
    auto it = g_tables.find(key);
    if (it != g_tables.end()) { it->second.second++; *out = it->second.first; return VX_OK; }
    SizeTables *t = nullptr;
    int rc = tables_create(dev, log_n, blowup, &t);
    if (rc) return rc;
    g_tables[key] = {t, 1};
    *out = t;
    return VX_OK;
}

static void tables_release(SizeTables *t) {
    std::lock_guard<std::mutex> lk(g_tab_mu);
    for (auto it = g_tables.begin(); it != g_tables.end(); ++it) {
        if (it->second.first == t) {
            if (--it->second.second == 0) { tables_destroy(t); g_tables.erase(it); }
            return;
        }
    }
}

}  // namespace vx

struct vx_prover {
    vx::ProofSlot s;
    int device;
    uint32_t launches;  // kernels enqueued by the last vx_prover_prove_async
};

using namespace vx;

extern "C" size_t vx_proof_size(uint32_t log_n, uint32_t blowup_bits, uint32_t n_queries) {
    if (log_n < 4 || blowup_bits < 1 || log_n + blowup_bits > 31) return 0;
    ProofLayout L;
    proof_layout(log_n, blowup_bits, n_queries, &L);
    return (size_t)(L.words * 4);
}

extern "C" int vx_prover_create(uint32_t log_n, uint32_t blowup_bits, uint32_t n_queries, vx_prover **out) {
    VX_CHECK_ARG(out != nullptr, "vx_prover_create: out is null");
    VX_CHECK_ARG(log_n >= 4 && blowup_bits >= 1 && log_n + blowup_bits <= 31,
                 "vx_prover_create: need log_n >= 4, blowup_bits >= 1, log_n + blowup_bits <= 31 (got %u, %u)",
                 log_n, blowup_bits);
    VX_CHECK_ARG(n_queries >= 1 && n_queries <= 4096, "vx_prover_create: n_queries must be in [1, 4096]");
    auto *p = new vx_prover();
    memset(&p->s, 0, sizeof(p->s));
    cudaGetDevice(&p->device);
    ProofSlot &S = p->s;
    int rc = tables_acquire(log_n, blowup_bits, &S.tw);
    if (rc) { delete p; return rc; }
    proof_layout(log_n, blowup_bits, n_queries, &S.L);
    const ProofLayout &L = S.L;
    uint32_t le = L.le;
    uint64_t n = 1ull << log_n, N = 1ull << le;
    // carve one allocation
    uint64_t w = 0;
    uint64_t o_coeffs = w; w += align_words(n);
    uint64_t o_eval = w; w += align_words(N);
    uint64_t o_fri[32];
    for (uint32_t k = 0; k < L.nfri; k++) { o_fri[k] = w; w += 4 * align_words(1ull << (le - 1 - k)); }
    // leaf-kernel shapes read once: the pools are sized and carved with them
    const uint32_t kt = tree_leaf_k(le);
    uint32_t kf[32];
    for (uint32_t k = 0; k < L.nfri; k++) kf[k] = tree_leaf_k(le - 1 - k, kLeafFold);
    uint64_t o_tt = w; w += align_words(tree_pool_words(le, kt));
    uint64_t o_qt = w; w += align_words(tree_pool_words(le, kt));
    uint64_t o_ft[32];
    for (uint32_t k = 0; k < L.nfri; k++) { o_ft[k] = w; w += align_words(tree_pool_words(le - 1 - k, kf[k])); }
    uint64_t o_chan = w; w += align_words(sizeof(DevChannel) / 4 + 1);
    uint64_t o_aq = w; w += align_words(4);
    uint64_t o_af = w; w += align_words(4ull * (L.nfri + 1));
    uint64_t o_qi = w; w += align_words(n_queries);
    uint64_t o_proof = w; w += align_words(L.words);
    void *blk = nullptr;
    if (cudaMalloc(&blk, w * 4) != cudaSuccess) {
        cudaGetLastError();
        tables_release(S.tw);
        delete p;
        set_last_error(VX_ERR_OOM, "cudaMalloc of %llu bytes for a proof slot failed", (unsigned long long)(w * 4));
        return VX_ERR_OOM;
    }
    uint32_t *b = (uint32_t *)blk;
    S.block = blk;
    S.block_bytes = w * 4;
    S.coeffs = b + o_coeffs;
    S.eval = b + o_eval;
    for (uint32_t k = 0; k < L.nfri; k++) {
        uint64_t sz = align_words(1ull << (le - 1 - k));
        for (int c = 0; c < 4; c++) S.fri[k][c] = b + o_fri[k] + c * sz;
    }
    tree_plan(le, b + o_tt, &S.trace_lv, kt);
    tree_plan(le, b + o_qt, &S.quot_lv, kt);
    for (uint32_t k = 0; k < L.nfri; k++) tree_plan(le - 1 - k, b + o_ft[k], &S.fri_lv[k], kf[k]);
    S.chan = (DevChannel *)(b + o_chan);
    S.alpha_q = b + o_aq;
    S.alpha_f = b + o_af;
    S.qidx = b + o_qi;
    S.proof = b + o_proof;
    std::vector<uint32_t> tmpl(L.words);
    proof_template(L, tmpl.data());
    cudaError_t e = cudaMemcpy(S.proof, tmpl.data(), L.words * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(S.chan, 0, sizeof(DevChannel));
    if (e == cudaSuccess) e = tree_reset(S.trace_lv, nullptr);
    if (e == cudaSuccess) e = tree_reset(S.quot_lv, nullptr);
    for (uint32_t k = 0; k < L.nfri && e == cudaSuccess; k++) e = tree_reset(S.fri_lv[k], nullptr);
    if (e == cudaSuccess) e = cudaStreamSynchronize(nullptr);  // slot streams may be non-blocking
    if (e != cudaSuccess) {
        vx_prover_destroy(p);
        set_last_error(VX_ERR_CUDA, "initialising proof slot: %s", cudaGetErrorString(e));
        return VX_ERR_CUDA;
    }
    *out = p;
    return VX_OK;
}

extern "C" void vx_prover_destroy(vx_prover *p) {
    if (!p) return;
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(p->device);
    if (p->s.block) cudaFree(p->s.block);
    cudaSetDevice(cur);
    if (p->s.tw) tables_release(p->s.tw);
    delete p;
}

extern "C" size_t vx_prover_slot_bytes(const vx_prover *p) { return p ? p->s.block_bytes : 0; }
extern "C" size_t vx_prover_table_bytes(const vx_prover *p) { return p && p->s.tw ? tables_bytes(p->s.tw) : 0; }

// Stages of one proof, in order (prover.rs:264-619):
//   0 trace, 1 interpolate, 2 LDE evaluate, 3 trace commitment,
//   4 quotient commitment, 5 circle fold + FRI layer 0, 6 line folds,
//   7 last layer + queries, 8 decommitment.
// Stage 6 folds FRI layers k = 1 .. nfri-1; enqueue_stage(..., k_lo, k_hi)
// enqueues only layers [k_lo, k_hi) of it (the other stages ignore them).
static int enqueue_stage(vx_prover *p, uint32_t stage, uint32_t a, uint32_t b, cudaStream_t st, uint32_t *launches,
                         uint32_t k_lo = 1, uint32_t k_hi = ~0u) {
    ProofSlot &S = p->s;
    const ProofLayout &L = S.L;
    const SizeTables &T = *S.tw;
    const uint32_t log_n = L.log_n, le = L.le;
    const uint64_t n = 1ull << log_n, N = 1ull << le;
    uint32_t *proof = S.proof;
    LeafQuotient lq{S.eval, N - 1, S.alpha_q, {0, 0, 0, 0}};
    auto ntt_launches = [](uint32_t layers, uint32_t elems_log) { return ntt_pass_count(layers, elems_log); };
    switch (stage) {
    case 0:
        VX_CUDA_TRY(cudaMemsetAsync(S.chan, 0, sizeof(DevChannel), st));
        fib_trace_kernel<<<(unsigned)((n + kTraceRows - 1) / kTraceRows), 256, 0, st>>>(a, b, S.inputs, S.coeffs, n,
                                                                         proof + L.magic + 3);
        *launches += 1;
        break;
    case 1: {
        NttTables it{T.itw_line, T.itw_circle, {}};
        memcpy(it.off, T.itw_off, sizeof(it.off));
        VX_CUDA_TRY(ntt_transform(S.coeffs, nullptr, 0, 1, log_n, it, false, nullptr, 0, st));
        *launches += ntt_launches(log_n, log_n);
        break;
    }
    case 2: {
        NttTables ft{T.ftw_line, T.ftw_circle, {}};
        memcpy(ft.off, T.ftw_off, sizeof(ft.off));
        VX_CUDA_TRY(ntt_transform(S.eval, nullptr, 0, 1, le, ft, true, S.coeffs, log_n, st));
        *launches += ntt_launches(log_n, le);
        break;
    }
    case 3:
        VX_CUDA_TRY(tree_build(LeafM31{S.eval}, S.trace_lv, ChanStep{S.chan, proof + L.troot, S.alpha_q}, st));
        *launches += tree_launches(S.trace_lv);
        break;
    case 4:
        VX_CUDA_TRY(tree_build(lq, S.quot_lv, ChanStep{S.chan, proof + L.qroot, S.alpha_f}, st));
        *launches += tree_launches(S.quot_lv);
        break;
    case 5: {
        LeafCircleFold cf{lq, T.fold_circle, S.alpha_f, S.fri[0][0], S.fri[0][1], S.fri[0][2], S.fri[0][3], {}};
        VX_CUDA_TRY(tree_build(cf, S.fri_lv[0], ChanStep{S.chan, proof + L.froots, L.nfri > 1 ? S.alpha_f + 4 : nullptr},
                               st));
        *launches += tree_launches(S.fri_lv[0]);
        break;
    }
    case 6:
        for (uint32_t k = k_lo < 1 ? 1 : k_lo; k < L.nfri && k < k_hi; k++) {
            uint32_t lsrc = le - k;  // log size of the layer being folded
            LeafLineFold lf{S.fri[k - 1][0], S.fri[k - 1][1], S.fri[k - 1][2], S.fri[k - 1][3],
                            T.fold_line + T.fold_line_off[lsrc], S.alpha_f + 4 * k,
                            S.fri[k][0], S.fri[k][1], S.fri[k][2], S.fri[k][3], {}};
            VX_CUDA_TRY(tree_build(lf, S.fri_lv[k],
                                   ChanStep{S.chan, proof + L.froots + 8 * k,
                                            k + 1 < L.nfri ? S.alpha_f + 4 * (k + 1) : nullptr},
                                   st));
            *launches += tree_launches(S.fri_lv[k]);
        }
        break;
    case 7: {
        uint32_t kl = L.nfri - 1;
        chan_queries_kernel<<<1, 128, 0, st>>>(S.chan, S.fri[kl][0], S.fri[kl][1], S.fri[kl][2], S.fri[kl][3],
                                               proof + L.last, N, L.nq, S.qidx, proof + L.qidx);
        *launches += 1;
        break;
    }
    case 8: {
        ValuesArgs va;
        memset(&va, 0, sizeof(va));
        va.eval = S.eval; va.mask = N - 1; va.alpha_q = S.alpha_q; va.nfri = L.nfri;
        va.vals[0] = L.trace.vals; va.svals[0] = L.trace.svals;
        va.vals[1] = L.quot.vals; va.svals[1] = L.quot.svals;
        for (uint32_t k = 0; k < L.nfri; k++) {
            for (int c = 0; c < 4; c++) va.fri[k][c] = S.fri[k][c];
            va.vals[2 + k] = L.fri[k].vals; va.svals[2 + k] = L.fri[k].svals;
        }
        decommit_values_kernel<<<blocks_for((uint64_t)(2 + L.nfri) * L.nq, 128), 128, 0, st>>>(va, S.qidx, L.nq, proof);
        PathsArgs pa;
        memset(&pa, 0, sizeof(pa));
        pa.eval = S.eval; pa.mask = N - 1; pa.alpha_q = S.alpha_q;
        uint32_t max_groups = 0;
        auto add = [&](uint32_t i, const TreeLevels &lv, uint32_t kind, uint32_t shift, const uint32_t *const *c,
                       const DecomLayout &d) {
            pa.t[i].lv = lv; pa.t[i].kind = kind; pa.t[i].shift = shift;
            for (int q = 0; q < 4; q++) pa.t[i].c[q] = c ? c[q] : nullptr;
            pa.t[i].paths = d.paths; pa.t[i].spaths = d.spaths;
            if (lv.n - 1 > max_groups) max_groups = lv.n - 1;
        };
        const uint32_t *ev4[4] = {S.eval, nullptr, nullptr, nullptr};
        add(0, S.trace_lv, 0, 0, ev4, L.trace);
        add(1, S.quot_lv, 1, 0, nullptr, L.quot);
        for (uint32_t k = 0; k < L.nfri; k++) add(2 + k, S.fri_lv[k], 2, k + 1, S.fri[k], L.fri[k]);
        dim3 grid(blocks_for((uint64_t)L.nq * max_groups, 64), 2 + L.nfri);
        decommit_all_kernel<<<grid, 64, 0, st>>>(pa, S.qidx, L.nq, proof);
        *launches += 2;
        break;
    }
    default:
        set_last_error(VX_ERR_ARG, "unknown proof stage %u", stage);
        return VX_ERR_ARG;
    }
    VX_CUDA_TRY(cudaGetLastError());
    return VX_OK;
}

extern "C" int vx_prover_stage_async(vx_prover *p, uint32_t stage, uint32_t a, uint32_t b, void *stream_v) {
    VX_CHECK_ARG(p != nullptr, "vx_prover_stage_async: null prover");
    VX_CHECK_ARG(a < VX_P && b < VX_P, "vx_prover_stage_async: public inputs must be canonical M31 (< 2^31-1)");
    uint32_t launches = 0;
    return enqueue_stage(p, stage, a, b, (cudaStream_t)stream_v, &launches);
}

extern "C" int vx_prover_prove_async(vx_prover *p, uint32_t a, uint32_t b, void *stream_v) {
    VX_CHECK_ARG(p != nullptr, "vx_prover_prove_async: null prover");
    VX_CHECK_ARG(a < VX_P && b < VX_P, "vx_prover_prove_async: public inputs must be canonical M31 (< 2^31-1)");
    uint32_t launches = 0;
    for (uint32_t stage = 0; stage < VX_N_STAGES; stage++) {
        int rc = enqueue_stage(p, stage, a, b, (cudaStream_t)stream_v, &launches);
        if (rc) return rc;
    }
    p->launches = launches;
    return VX_OK;
}

extern "C" uint32_t vx_prover_launches(const vx_prover *p) { return p ? p->launches : 0u; }

extern "C" int vx_prover_fetch_async(vx_prover *p, void *dst, void *stream_v) {
    VX_CHECK_ARG(p != nullptr && dst != nullptr, "vx_prover_fetch_async: null argument");
    VX_CUDA_TRY(cudaMemcpyAsync(dst, p->s.proof, p->s.L.words * 4, cudaMemcpyDeviceToHost, (cudaStream_t)stream_v));
    return VX_OK;
}

extern "C" int vx_prover_proof_device(vx_prover *p, const void **dptr, size_t *bytes) {
    VX_CHECK_ARG(p != nullptr && dptr != nullptr && bytes != nullptr, "vx_prover_proof_device: null argument");
    *dptr = p->s.proof;
    *bytes = (size_t)(p->s.L.words * 4);
    return VX_OK;
}

extern "C" int vx_prover_check(vx_prover *p) {
    VX_CHECK_ARG(p != nullptr, "vx_prover_check: null prover");
    uint32_t err = 0;
    VX_CUDA_TRY(cudaMemcpy(&err, &p->s.chan->err, 4, cudaMemcpyDeviceToHost));
    if (err) {
        set_last_error(VX_ERR_DEVICE, "transcript rejection sampling exceeded its bound");
        return VX_ERR_DEVICE;
    }
    return VX_OK;
}

// ---- synchronous convenience with a per-size slot cache ----
namespace {
std::mutex g_slot_mu;
std::map<std::tuple<int, uint32_t, uint32_t, uint32_t>, vx_prover *> g_slots;
}  // namespace

extern "C" int vx_prove_fib(uint32_t a, uint32_t b, uint32_t log_n, uint32_t blowup_bits, uint32_t n_queries,
                            uint8_t *out, size_t cap, size_t *out_len) {
    VX_CHECK_ARG(out != nullptr && out_len != nullptr, "vx_prove_fib: null output");
    size_t need = vx_proof_size(log_n, blowup_bits, n_queries);
    VX_CHECK_ARG(need != 0, "vx_prove_fib: unsupported size log_n=%u blowup_bits=%u", log_n, blowup_bits);
    VX_CHECK_ARG(cap >= need, "vx_prove_fib: output capacity %zu < proof size %zu", cap, need);
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(g_slot_mu);
    auto key = std::make_tuple(dev, log_n, blowup_bits, n_queries);
    vx_prover *p = nullptr;
    auto it = g_slots.find(key);
    if (it != g_slots.end()) {
        p = it->second;
    } else {
        int rc = vx_prover_create(log_n, blowup_bits, n_queries, &p);
        if (rc) return rc;
        g_slots[key] = p;
    }
    int rc = vx_prover_prove_async(p, a, b, nullptr);
    if (rc) return rc;
    rc = vx_prover_fetch_async(p, out, nullptr);
    if (rc) return rc;
    VX_CUDA_TRY(cudaStreamSynchronize(nullptr));
    rc = vx_prover_check(p);
    if (rc) return rc;
    *out_len = need;
    return VX_OK;
}

// ---- batch: ProverPipeline::prove_batch (prover.rs:2278-2311) ----
// Up to four slots of one size on their own non-blocking streams keep that
// many proofs in flight: one proof's latency-bound FRI tail overlaps the
// next ones' trace, LDE and hashing.  Each slot's proof bytes and status
// word come back through its own pinned buffer while the other slots prove.
namespace {
constexpr int kBatchSlots = 4;  // proofs in flight (log_n = 24: 16.58 / 15.95 / 15.79 / 15.74 ms per proof for 1..4)
struct BatchCtx {
    int n = 0;  // slots created so far
    vx_prover *slot[kBatchSlots] = {};
    cudaStream_t st[kBatchSlots] = {};
    uint8_t *pinned[kBatchSlots] = {};
    cudaEvent_t done[kBatchSlots] = {};
};
std::map<std::tuple<int, uint32_t, uint32_t, uint32_t>, BatchCtx> g_batch;

void batch_free(BatchCtx &c) {
    for (int k = 0; k < kBatchSlots; k++) {
        if (c.done[k]) cudaEventDestroy(c.done[k]);
        if (c.pinned[k]) cudaFreeHost(c.pinned[k]);
        if (c.st[k]) cudaStreamDestroy(c.st[k]);
        if (c.slot[k]) vx_prover_destroy(c.slot[k]);
    }
    c = BatchCtx{};
}

// Slot k of a batch context: a prover slot, a non-blocking stream, a pinned
// buffer for the proof bytes and status word, a completion event.
int batch_add_slot(BatchCtx &c, uint32_t log_n, uint32_t blowup_bits, uint32_t n_queries, size_t bytes) {
    const int k = c.n;
    int rc = vx_prover_create(log_n, blowup_bits, n_queries, &c.slot[k]);
    if (rc == VX_OK && (cudaStreamCreateWithFlags(&c.st[k], cudaStreamNonBlocking) != cudaSuccess ||
                        cudaHostAlloc((void **)&c.pinned[k], bytes + 16, cudaHostAllocDefault) != cudaSuccess ||
                        cudaEventCreateWithFlags(&c.done[k], cudaEventDisableTiming) != cudaSuccess)) {
        cudaGetLastError();
        set_last_error(VX_ERR_OOM, "vx_prove_fib_batch: stream, pinned buffer or event creation failed");
        rc = VX_ERR_OOM;
    }
    if (rc != VX_OK) {
        if (c.done[k]) cudaEventDestroy(c.done[k]);
        if (c.pinned[k]) cudaFreeHost(c.pinned[k]);
        if (c.st[k]) cudaStreamDestroy(c.st[k]);
        if (c.slot[k]) vx_prover_destroy(c.slot[k]);
        c.done[k] = nullptr; c.pinned[k] = nullptr; c.st[k] = nullptr; c.slot[k] = nullptr;
        return rc;
    }
    c.n = k + 1;
    return VX_OK;
}

// The context of this device and proof size with up to `want` slots: a
// second and later slot is added only while it fits in half of the free
// device memory, so large proofs run with fewer proofs in flight.
int batch_ctx(int dev, uint32_t log_n, uint32_t blowup_bits, uint32_t n_queries, size_t bytes, int want,
              BatchCtx **out) {
    BatchCtx &c = g_batch[std::make_tuple(dev, log_n, blowup_bits, n_queries)];
    if (want > kBatchSlots) want = kBatchSlots;
    while (c.n < want) {
        if (c.n >= 1) {
            size_t free_b = 0, total_b = 0;
            if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) { cudaGetLastError(); break; }
            if (2 * vx_prover_slot_bytes(c.slot[0]) > free_b) break;
        }
        const int rc = batch_add_slot(c, log_n, blowup_bits, n_queries, bytes);
        if (rc != VX_OK) {
            if (c.n == 0) return rc;
            break;  // run with the slots that fit
        }
    }
    *out = &c;
    return VX_OK;
}
}  // namespace

extern "C" int vx_prove_fib_batch(const uint32_t *a, const uint32_t *b, uint32_t count, uint32_t log_n,
                                  uint32_t blowup_bits, uint32_t n_queries, uint8_t *out, size_t cap,
                                  size_t *proof_size) {
    VX_CHECK_ARG(a != nullptr && b != nullptr && out != nullptr && proof_size != nullptr,
                 "vx_prove_fib_batch: null argument");
    const size_t need = vx_proof_size(log_n, blowup_bits, n_queries);
    VX_CHECK_ARG(need != 0, "vx_prove_fib_batch: unsupported size log_n=%u blowup_bits=%u", log_n, blowup_bits);
    VX_CHECK_ARG(cap / need >= count, "vx_prove_fib_batch: output capacity %zu < %u proofs of %zu bytes", cap, count,
                 need);
    for (uint32_t i = 0; i < count; i++)
        VX_CHECK_ARG(a[i] < VX_P && b[i] < VX_P, "vx_prove_fib_batch: input %u is not canonical M31", i);
    *proof_size = need;
    if (count == 0) return VX_OK;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(g_slot_mu);
    BatchCtx *c = nullptr;
    int rc = batch_ctx(dev, log_n, blowup_bits, n_queries, need, count < (uint32_t)kBatchSlots ? (int)count : kBatchSlots,
                       &c);
    if (rc) return rc;
    const uint32_t ns = (uint32_t)c->n;
    // collect proof i (slot i % ns): wait for its stream, copy out, check its status word
    auto collect = [&](uint32_t i) -> int {
        const uint32_t k = i % ns;
        VX_CUDA_TRY(cudaEventSynchronize(c->done[k]));
        uint32_t err = 0;
        memcpy(&err, c->pinned[k] + need, 4);
        if (err) {
            set_last_error(VX_ERR_DEVICE, "vx_prove_fib_batch: proof %u: transcript rejection sampling exceeded its bound",
                           i);
            return VX_ERR_DEVICE;
        }
        memcpy(out + (size_t)i * need, c->pinned[k], need);
        return VX_OK;
    };
    uint32_t launched = 0, collected = 0;
    for (uint32_t i = 0; i < count && rc == VX_OK; i++) {
        const uint32_t k = i % ns;
        if (i >= ns) {
            rc = collect(i - ns);
            collected = i - ns + 1;
            if (rc) break;
        }
        vx_prover *p = c->slot[k];
        rc = vx_prover_prove_async(p, a[i], b[i], c->st[k]);
        if (rc) break;
        VX_CUDA_TRY(cudaMemcpyAsync(c->pinned[k], p->s.proof, need, cudaMemcpyDeviceToHost, c->st[k]));
        VX_CUDA_TRY(cudaMemcpyAsync(c->pinned[k] + need, &p->s.chan->err, 4, cudaMemcpyDeviceToHost, c->st[k]));
        VX_CUDA_TRY(cudaEventRecord(c->done[k], c->st[k]));
        launched = i + 1;
    }
    // drain what is still in flight, even after an error, so no copy lands later
    for (uint32_t i = collected; i < launched; i++) {
        const int r2 = collect(i);
        if (rc == VX_OK) rc = r2;
    }
    return rc;
}

extern "C" void vx_release_all(void) {
    // the forge batch launchers' column-pointer arrays
    forge_cols_release();
    // the cached slots of vx_prove_fib and vx_prove_fib_batch; each size's
    // tables go with their last slot
    std::lock_guard<std::mutex> lk(g_slot_mu);
    for (auto &kv : g_slots) vx_prover_destroy(kv.second);
    g_slots.clear();
    for (auto &kv : g_batch) batch_free(kv.second);
    g_batch.clear();
}

// ---------------------------------------------------------------------
// vx_prove_fib_noalloc: the whole proof without any device allocation.
//
// For callers that cannot call cudaMalloc: hosts whose device memory is
// owned by another allocator (a Rust arena, a framework's caching pool) and
// sandboxes that forbid cudaMalloc after start-up.  Every byte of device
// scratch — generator tables, twiddle tables, the LDE, FRI layers, stored
// tree levels, transcript state and the proof — lives in one file-scope
// static __device__ array of kNoAllocWords words (8 MiB), which every GPU
// that loads this library keeps until the process exits.  Each call copies
// synchronously and runs on the legacy default stream, so it must not be
// called while a stream capture is active.  g_na_mu serialises the calls:
// they share the array, which keeps the last call's contents.
// ---------------------------------------------------------------------
namespace {
constexpr uint64_t kNoAllocWords = 1ull << 21;   // 8 MiB of device scratch
constexpr uint32_t kNoAllocMaxLogEval = 14;       // log_n + blowup_bits <= 14
constexpr uint32_t kNoAllocMaxQueries = 80;
static __device__ __align__(256) uint32_t g_noalloc_scratch[kNoAllocWords];

struct NoAllocDevice {
    bool ready;
    uint32_t *base;                 // device address of g_noalloc_scratch
    uint32_t tab_log_n, tab_blowup; // size whose tables are resident (0 = none)
};
std::mutex g_na_mu;
NoAllocDevice g_na[64];
uint32_t g_na_host[kGenTableWords];       // staging for the generator tables
uint32_t g_na_proof_tmpl[1u << 18];       // staging for the proof template
}  // namespace

extern "C" int vx_prove_fib_noalloc(uint32_t a, uint32_t b, uint32_t log_n, uint32_t blowup_bits,
                                    uint32_t n_queries, uint8_t *out, size_t cap, size_t *out_len) {
    VX_CHECK_ARG(out != nullptr && out_len != nullptr, "vx_prove_fib_noalloc: null output");
    VX_CHECK_ARG(a < VX_P && b < VX_P, "vx_prove_fib_noalloc: public inputs must be canonical M31 (< 2^31-1)");
    VX_CHECK_ARG(log_n >= 4 && blowup_bits >= 1 && log_n + blowup_bits <= kNoAllocMaxLogEval,
                 "vx_prove_fib_noalloc: needs 4 <= log_n, blowup_bits >= 1 and log_n + blowup_bits <= %u "
                 "(got %u, %u); larger proofs need vx_prove_fib",
                 kNoAllocMaxLogEval, log_n, blowup_bits);
    VX_CHECK_ARG(n_queries >= 1 && n_queries <= kNoAllocMaxQueries,
                 "vx_prove_fib_noalloc: n_queries must be in [1, %u]", kNoAllocMaxQueries);
    ProofLayout L;
    proof_layout(log_n, blowup_bits, n_queries, &L);
    size_t need = (size_t)(L.words * 4);
    VX_CHECK_ARG(cap >= need, "vx_prove_fib_noalloc: output capacity %zu < proof size %zu", cap, need);
    VX_CHECK_ARG(L.words <= (sizeof(g_na_proof_tmpl) / 4), "vx_prove_fib_noalloc: proof layout too large");
    int dev = 0;
    VX_CUDA_TRY(cudaGetDevice(&dev));
    VX_CHECK_ARG(dev >= 0 && dev < 64, "vx_prove_fib_noalloc: device ordinal %d out of range", dev);
    std::lock_guard<std::mutex> lk(g_na_mu);
    NoAllocDevice &D = g_na[dev];
    if (!D.ready) {
        // once per device: the array's device address (the host symbol is
        // only a stand-in) and the generator tables
        void *p = nullptr;
        VX_CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        gen_tables_host(g_na_host);
        VX_CUDA_TRY(cudaMemcpy(p, g_na_host, sizeof(g_na_host), cudaMemcpyHostToDevice));
        D.base = (uint32_t *)p;
        D.tab_log_n = D.tab_blowup = 0;
        D.ready = true;
    }
    uint32_t *base = D.base;
    GenTables g{(const cpoint *)base, (const cpoint *)base + (1u << 16)};
    const uint32_t le = L.le;
    const uint64_t n = 1ull << log_n, N = 1ull << le;
    uint64_t w = align_words(kGenTableWords);
    // tables, laid out as tables_create does
    SizeTables T;
    memset(&T, 0, sizeof(T));
    T.device = dev; T.log_n = log_n; T.blowup = blowup_bits; T.le = le;
    T.itw_line = base + w; w += align_words(n - 1);
    T.itw_circle = base + w; w += align_words(n / 2);
    T.ftw_line = base + w; w += align_words(N - 1);
    T.ftw_circle = base + w; w += align_words(N / 2);
    T.fold_circle = base + w; w += align_words(N / 2);
    T.fold_line = base + w;
    uint64_t fl = 0;
    for (uint32_t l = le - 1; l >= 4; l--) { T.fold_line_off[l] = fl; fl += align_words(1ull << (l - 1)); }
    w += fl;
    ntt_table_offsets(log_n, T.itw_off);
    ntt_table_offsets(le, T.ftw_off);
    // slot, laid out as vx_prover_create does
    vx_prover P;
    memset(&P.s, 0, sizeof(P.s));
    P.device = dev;
    P.launches = 0;
    ProofSlot &S = P.s;
    S.tw = &T;
    S.L = L;
    S.coeffs = base + w; w += align_words(n);
    S.eval = base + w; w += align_words(N);
    for (uint32_t k = 0; k < L.nfri; k++) {
        uint64_t sz = align_words(1ull << (le - 1 - k));
        for (int c = 0; c < 4; c++) S.fri[k][c] = base + w + c * sz;
        w += 4 * sz;
    }
    w += align_words(tree_plan(le, base + w, &S.trace_lv, 0));
    w += align_words(tree_plan(le, base + w, &S.quot_lv, 0));
    for (uint32_t k = 0; k < L.nfri; k++)
        w += align_words(tree_plan(le - 1 - k, base + w, &S.fri_lv[k], tree_leaf_k(le - 1 - k, kLeafFold)));
    S.chan = (DevChannel *)(base + w); w += align_words(sizeof(DevChannel) / 4 + 1);
    S.alpha_q = base + w; w += align_words(4);
    S.alpha_f = base + w; w += align_words(4ull * (L.nfri + 1));
    S.qidx = base + w; w += align_words(n_queries);
    S.proof = base + w; w += align_words(L.words);
    VX_CHECK_ARG(w <= kNoAllocWords, "vx_prove_fib_noalloc: layout of %llu words exceeds the static scratch of %llu",
                 (unsigned long long)w, (unsigned long long)kNoAllocWords);
    cudaStream_t st = nullptr;  // legacy default stream
    // the counters of the tree reduce kernels sit where another size's
    // layout may have left data
    VX_CUDA_TRY(tree_reset(S.trace_lv, st));
    VX_CUDA_TRY(tree_reset(S.quot_lv, st));
    for (uint32_t k = 0; k < L.nfri; k++) VX_CUDA_TRY(tree_reset(S.fri_lv[k], st));
    if (D.tab_log_n != log_n || D.tab_blowup != blowup_bits) {
        D.tab_log_n = D.tab_blowup = 0;
        VX_CUDA_TRY(build_ntt_tables_with(g, ecoset_half_coset(log_n), true, T.itw_line, T.itw_circle, st));
        VX_CUDA_TRY(build_ntt_tables_with(g, ecoset_eval_domain(le), false, T.ftw_line, T.ftw_circle, st));
        VX_CUDA_TRY(build_fold_twiddles_with(g, ecoset_eval_domain(le), true, T.fold_circle, st));
        for (uint32_t l = le - 1; l >= 4; l--)
            VX_CUDA_TRY(build_fold_twiddles_with(g, ecoset_half_odds(l), false, T.fold_line + T.fold_line_off[l], st));
        D.tab_log_n = log_n;
        D.tab_blowup = blowup_bits;
    }
    // the proof's constant words; everything else is overwritten by the stages
    proof_template(L, g_na_proof_tmpl);
    VX_CUDA_TRY(cudaMemcpy(S.proof, g_na_proof_tmpl, L.words * 4, cudaMemcpyHostToDevice));
    uint32_t launches = 0;
    for (uint32_t stage = 0; stage < VX_N_STAGES; stage++) {
        int rc = enqueue_stage(&P, stage, a, b, st, &launches);
        if (rc) return rc;
    }
    VX_CUDA_TRY(cudaMemcpy(out, S.proof, need, cudaMemcpyDeviceToHost));
    uint32_t err = 0;
    VX_CUDA_TRY(cudaMemcpy(&err, &S.chan->err, 4, cudaMemcpyDeviceToHost));
    if (err) {
        set_last_error(VX_ERR_DEVICE, "transcript rejection sampling exceeded its bound");
        return VX_ERR_DEVICE;
    }
    *out_len = need;
    return VX_OK;
}

namespace vx {
// Capture one whole proof of slot `p` as a CUDA graph whose public inputs
// come from `pinned_ab` (two words of pinned host memory, copied to the
// device by the graph's first node) and whose proof bytes land in
// `pinned_out`.  Used by the serving engine, one graph per slot.
int prover_capture_graph(vx_prover *p, cudaStream_t st, uint32_t *dev_ab, const uint32_t *pinned_ab,
                         void *pinned_out, cudaGraphExec_t *exec) {
    ProofSlot &S = p->s;
    // one plain proof first so every lazily set kernel attribute exists
    uint32_t launches = 0;
    for (uint32_t stage = 0; stage < VX_N_STAGES; stage++) {
        int rc = enqueue_stage(p, stage, 1u, 1u, st, &launches);
        if (rc) return rc;
    }
    VX_CUDA_TRY(cudaStreamSynchronize(st));
    S.inputs = dev_ab;
    cudaGraph_t g = nullptr;
    VX_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    int rc = VX_OK;
    if (cudaMemcpyAsync(dev_ab, pinned_ab, 8, cudaMemcpyHostToDevice, st) != cudaSuccess) rc = VX_ERR_CUDA;
    launches = 0;
    for (uint32_t stage = 0; stage < VX_N_STAGES && rc == VX_OK; stage++) rc = enqueue_stage(p, stage, 0u, 0u, st, &launches);
    if (rc == VX_OK && cudaMemcpyAsync(pinned_out, S.proof, S.L.words * 4, cudaMemcpyDeviceToHost, st) != cudaSuccess)
        rc = VX_ERR_CUDA;
    // the transcript status word right after the proof bytes
    if (rc == VX_OK && cudaMemcpyAsync((uint8_t *)pinned_out + S.L.words * 4, &S.chan->err, 4, cudaMemcpyDeviceToHost,
                                       st) != cudaSuccess)
        rc = VX_ERR_CUDA;
    cudaError_t e = cudaStreamEndCapture(st, &g);
    S.inputs = nullptr;
    if (rc != VX_OK) { if (g) cudaGraphDestroy(g); return rc; }
    if (e != cudaSuccess) { set_last_error(VX_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e)); return VX_ERR_CUDA; }
    e = cudaGraphInstantiate(exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) { set_last_error(VX_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e)); return VX_ERR_CUDA; }
    p->launches = launches;
    return VX_OK;
}
// The same proof as two graphs: `head` copies (a, b) in and runs stages
// [0, split); `tail` runs stages [split, VX_N_STAGES) and copies the proof
// bytes and the transcript status word out.  The caller launches tail after
// head (on the same stream, or on another stream that waits for an event
// recorded after head).
int prover_capture_graph_split(vx_prover *p, cudaStream_t st, uint32_t *dev_ab, const uint32_t *pinned_ab,
                               void *pinned_out, uint32_t split, cudaGraphExec_t *head, cudaGraphExec_t *tail) {
    VX_CHECK_ARG(split >= 1 && split < VX_N_STAGES, "prover_capture_graph_split: split %u outside 1..%u", split,
                 VX_N_STAGES - 1);
    ProofSlot &S = p->s;
    // Split at the line folds (stage 6): the FRI layers whose trees start with
    // the leaf kernel (deeper than 16, GPU-filling) go to the head, the small
    // layers, reduced by one latency-bound launch each, to the tail.
    uint32_t k_split = 1;
    if (split == 6)
        while (k_split < S.L.nfri && S.L.le - 1 - k_split > 16u) k_split++;
    uint32_t launches = 0;
    for (uint32_t stage = 0; stage < VX_N_STAGES; stage++) {
        int rc = enqueue_stage(p, stage, 1u, 1u, st, &launches);
        if (rc) return rc;
    }
    VX_CUDA_TRY(cudaStreamSynchronize(st));
    S.inputs = dev_ab;
    launches = 0;
    cudaGraphExec_t ex[2] = {nullptr, nullptr};
    int rc = VX_OK;
    for (int part = 0; part < 2 && rc == VX_OK; part++) {
        cudaGraph_t g = nullptr;
        if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) { rc = VX_ERR_CUDA; break; }
        if (part == 0) {
            if (cudaMemcpyAsync(dev_ab, pinned_ab, 8, cudaMemcpyHostToDevice, st) != cudaSuccess) rc = VX_ERR_CUDA;
            for (uint32_t stage = 0; stage < split && rc == VX_OK; stage++)
                rc = enqueue_stage(p, stage, 0u, 0u, st, &launches);
            if (rc == VX_OK && split == 6 && k_split > 1) rc = enqueue_stage(p, 6, 0u, 0u, st, &launches, 1, k_split);
        } else {
            for (uint32_t stage = split; stage < VX_N_STAGES && rc == VX_OK; stage++)
                rc = enqueue_stage(p, stage, 0u, 0u, st, &launches, stage == 6 ? k_split : 1);
            if (rc == VX_OK &&
                cudaMemcpyAsync(pinned_out, S.proof, S.L.words * 4, cudaMemcpyDeviceToHost, st) != cudaSuccess)
                rc = VX_ERR_CUDA;
            if (rc == VX_OK && cudaMemcpyAsync((uint8_t *)pinned_out + S.L.words * 4, &S.chan->err, 4,
                                               cudaMemcpyDeviceToHost, st) != cudaSuccess)
                rc = VX_ERR_CUDA;
        }
        cudaError_t e = cudaStreamEndCapture(st, &g);
        if (rc == VX_OK && e != cudaSuccess) {
            set_last_error(VX_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
            rc = VX_ERR_CUDA;
        }
        if (rc == VX_OK && (e = cudaGraphInstantiate(&ex[part], g, 0)) != cudaSuccess) {
            set_last_error(VX_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
            rc = VX_ERR_CUDA;
        }
        if (g) cudaGraphDestroy(g);
    }
    S.inputs = nullptr;
    if (rc != VX_OK) {
        for (auto &x : ex)
            if (x) cudaGraphExecDestroy(x);
        return rc;
    }
    *head = ex[0];
    *tail = ex[1];
    p->launches = launches;
    return VX_OK;
}

// Device bytes vx_prover_create takes for one slot of this size, and the
// shared tables of the size (same arithmetic as the carving above).
void prover_footprint(uint32_t log_n, uint32_t blowup, uint32_t nq, size_t *slot_b, size_t *tab_b) {
    ProofLayout L;
    proof_layout(log_n, blowup, nq, &L);
    uint32_t le = L.le;
    uint64_t n = 1ull << log_n, N = 1ull << le;
    uint64_t w = align_words(n) + align_words(N);
    for (uint32_t k = 0; k < L.nfri; k++) w += 4 * align_words(1ull << (le - 1 - k));
    w += 2 * align_words(tree_pool_words(le, 0));
    for (uint32_t k = 0; k < L.nfri; k++) w += align_words(tree_pool_words(le - 1 - k, tree_leaf_k(le - 1 - k, kLeafFold)));
    w += align_words(sizeof(DevChannel) / 4 + 1) + align_words(4) + align_words(4ull * (L.nfri + 1)) +
         align_words(nq) + align_words(L.words);
    *slot_b = (size_t)(w * 4);
    uint64_t t = align_words(n - 1) + align_words(n / 2) + align_words(N - 1) + align_words(N / 2) + align_words(N / 2);
    for (uint32_t l = le - 1; l >= 4; l--) t += align_words(1ull << (l - 1));
    *tab_b = (size_t)(t * 4);
}
uint32_t prover_log_n(const vx_prover *p) { return p->s.L.log_n; }
size_t prover_proof_bytes(const vx_prover *p) { return (size_t)(p->s.L.words * 4); }
const uint32_t *prover_chan_err(const vx_prover *p) { return &p->s.chan->err; }
}  // namespace vx
