// Circle NTT passes for sm_100a (see vx_ntt.cuh for the layout).
#include <cstring>

#include "vx_ntt.cuh"
#include "vx_field.cuh"
#include "vx_common.cuh"

namespace vx {

namespace {

constexpr uint32_t kMaxPassLayers = 11;  // 2^11 rows x 8 columns x 4 B = 64 KB tile
constexpr uint32_t kMaxTileWords = (1u << kMaxPassLayers) * 8u;

struct PassOff { uint32_t v[32]; };

// Circle-layer twiddle of butterfly h (see NttTables::circle_mode).
__device__ __forceinline__ uint32_t circle_tw(const uint32_t *__restrict__ circle, uint32_t mode, uint64_t h) {
    if (!mode) return __ldg(circle + h);
    const uint32_t sub = (uint32_t)h & 3u;
    const uint32_t v = __ldg(circle + 2 * (h >> 2) + (sub < 2u ? 1u : 0u));
    return (sub == 1u || sub == 2u) ? msub(0u, v) : v;
}

template <bool FWD>
__global__ void __launch_bounds__(512) ntt_pass_kernel(
    uint32_t *data, uint32_t *const *dev_cols, uint64_t col_stride,
    const uint32_t *src, uint64_t src_mask, uint64_t src_stride,
    const uint32_t *__restrict__ line, const uint32_t *__restrict__ circle, uint32_t cmode, PassOff off,
    uint32_t s, uint32_t r, uint32_t wlog, uint32_t scale) {
    extern __shared__ uint32_t sm[];
    const uint32_t W = 1u << wlog;
    const uint32_t cshift = s - wlog;
    const uint64_t tile = blockIdx.x;
    const uint64_t cb = tile & ((1ull << cshift) - 1ull);
    const uint64_t hb = tile >> cshift;
    uint32_t *col = dev_cols ? dev_cols[blockIdx.y] : data + (uint64_t)blockIdx.y * col_stride;
    const uint32_t *in = src ? src + (uint64_t)blockIdx.y * src_stride : col;
    const uint64_t base = (hb << (s + r)) | (cb << wlog);
    const uint32_t tsz = (1u << r) << wlog;

    for (uint32_t e = threadIdx.x; e < tsz; e += blockDim.x) {
        uint64_t g = base | ((uint64_t)(e >> wlog) << s) | (e & (W - 1u));
        sm[e] = in[src ? (g & src_mask) : g];
    }
    __syncthreads();

    const uint32_t nb = tsz >> 1;
    for (uint32_t jj = 0; jj < r; jj++) {
        const uint32_t j = FWD ? r - 1u - jj : jj;
        const uint32_t L = s + j;
        for (uint32_t b = threadIdx.x; b < nb; b += blockDim.x) {
            uint32_t c = b & (W - 1u), p = b >> wlog;
            uint32_t row0 = ((p >> j) << (j + 1)) | (p & ((1u << j) - 1u));
            uint32_t e0 = (row0 << wlog) | c, e1 = e0 + (1u << (j + wlog));
            uint64_t h = (hb << (r - 1u - j)) | (uint64_t)(row0 >> (j + 1));
            uint32_t t = L ? __ldg(line + off.v[L - 1] + h) : circle_tw(circle, cmode, h);
            uint32_t v0 = sm[e0], v1 = sm[e1];
            if (FWD) {
                uint32_t tmp = mmul(v1, t);
                sm[e0] = madd(v0, tmp);
                sm[e1] = msub(v0, tmp);
            } else {
                sm[e0] = madd(v0, v1);
                sm[e1] = mmul(msub(v0, v1), t);
            }
        }
        __syncthreads();
    }

    for (uint32_t e = threadIdx.x; e < tsz; e += blockDim.x) {
        uint64_t g = base | ((uint64_t)(e >> wlog) << s) | (e & (W - 1u));
        uint32_t v = sm[e];
        col[g] = scale != 1u ? mmul(v, scale) : v;
    }
}

__global__ void ntt_layer_kernel(uint32_t *d, const uint32_t *__restrict__ tw, uint32_t L, uint64_t half_n, int fwd) {
    uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= half_n) return;
    uint64_t stride = 1ull << L;
    uint64_t h = tid >> L;
    uint64_t i0 = (h << (L + 1)) + (tid & (stride - 1ull)), i1 = i0 + stride;
    uint32_t v0 = d[i0], v1 = d[i1], t = tw[h];
    if (fwd) {
        uint32_t tmp = mmul(v1, t);
        d[i0] = madd(v0, tmp);
        d[i1] = msub(v0, tmp);
    } else {
        d[i0] = madd(v0, v1);
        d[i1] = mmul(msub(v0, v1), t);
    }
}

// ---------------------------------------------------------------------
// Register-radix pass: a tile of 2^(R+WL) elements (2^R rows of 2^WL
// columns), 16 elements per thread.  The pass's R layers run in stages of up
// to 4 layers; in a stage each thread holds the 16 elements that differ in
// one contiguous block of 4 tile bits [A, A+4) covering the stage's layer
// bits, and does all the stage's butterflies in registers.  Between stages
// the tile goes through shared memory (padded by one word per 32 to spread
// the strided accesses over the banks).  The tile's twiddles (2^R - 1 words,
// one contiguous run of the reference table per layer) are staged in shared
// memory once per tile.
// ---------------------------------------------------------------------
struct Pass2Args {
    uint32_t *data;
    uint32_t *const *dev_cols;
    uint64_t col_stride;
    const uint32_t *src;
    uint64_t src_mask, src_stride;
    const uint32_t *line, *circle;
    uint32_t cmode;
    PassOff off;
    uint32_t s;       // lowest layer of the pass
    uint32_t scale;   // 1 = none
    uint32_t vec;     // 1: columns and source 16-byte aligned, 4 consecutive elements per access
};

__device__ __forceinline__ uint32_t pad32(uint32_t e) { return e + (e >> 5); }
// pad32(a | b) = pad32(a) + b + (b >> 5) when a and b have no bit in common
// (a shift distributes over OR, and an OR of disjoint fields is a sum).  The
// stage and tile accesses below are all of this form with b a compile-time
// offset, so each thread computes one padded base and the accesses use
// immediate offsets.

template <bool FWD, int R, int WL, int LO, int HI, int A>
__device__ __forceinline__ void ntt_stage(uint32_t *sm, const uint32_t *smtw, uint32_t tid) {
    constexpr int TB = R + WL;
    const uint32_t base = (tid & ((1u << A) - 1u)) | ((tid >> A) << (A + 4));  // bits [A, A+4) zero
    const uint32_t pb = pad32(base);
    uint32_t v[16];
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = sm[pb + ((uint32_t)i << A) + (((uint32_t)i << A) >> 5)];
#pragma unroll
    for (int jj = 0; jj < HI - LO; jj++) {
        const int j = FWD ? (HI - 1 - jj) : (LO + jj);
        const int rb = j + WL - A;            // register bit of layer j
        const int S = j + 1 + WL;             // tile-index shift giving the twiddle index
        const uint32_t *tw = smtw + ((1u << (R - 1 - j)) - 1u) + (base >> S);
#pragma unroll
        for (int i0 = 0; i0 < 16; i0++) {
            if (i0 & (1 << rb)) continue;
            const int i1 = i0 | (1 << rb);
            const uint32_t t = tw[i0 >> (rb + 1)];
            if (FWD) {
                uint32_t x = mmul(v[i1], t);
                v[i1] = msub(v[i0], x);
                v[i0] = madd(v[i0], x);
            } else {
                uint32_t a = v[i0], b = v[i1];
                v[i0] = madd(a, b);
                v[i1] = mmul(msub(a, b), t);
            }
        }
    }
#pragma unroll
    for (int i = 0; i < 16; i++) sm[pb + ((uint32_t)i << A) + (((uint32_t)i << A) >> 5)] = v[i];
    (void)TB;
}

// Compile-time stage list: stage k covers pass layers [lo, hi), at most 4,
// from the top for forward and from the bottom for inverse; the register
// block A is the contiguous 4-bit block of the tile index covering them.
template <bool FWD, int R, int WL, int K>
struct StageIdx {
    static constexpr int NST = (R + 3) / 4;
    static constexpr int HI = FWD ? R - 4 * K : ((4 * K + 4) < R ? (4 * K + 4) : R);
    static constexpr int LO = FWD ? ((R - 4 * K - 4) > 0 ? (R - 4 * K - 4) : 0) : 4 * K;
    static constexpr int TB = R + WL;
    static constexpr int A0 = (LO + WL) < (TB - 4) ? (LO + WL) : (TB - 4);
    static constexpr int A = (HI + WL - A0) <= 4 ? A0 : (HI + WL - 4);
};

template <bool FWD, int R, int WL, int K>
__device__ __forceinline__ void run_stages(uint32_t *sm, const uint32_t *smtw, uint32_t tid) {
    if constexpr (K < StageIdx<FWD, R, WL, K>::NST) {
        using St = StageIdx<FWD, R, WL, K>;
        ntt_stage<FWD, R, WL, St::LO, St::HI, St::A>(sm, smtw, tid);
        __syncthreads();
        run_stages<FWD, R, WL, K + 1>(sm, smtw, tid);
    }
}

template <bool FWD, int R, int WL>
__global__ void __launch_bounds__((1 << (R + WL)) / 16) ntt_pass2_kernel(Pass2Args p) {
    constexpr int TB = R + WL, TS = 1 << TB, NT = TS / 16, W = 1 << WL;
    extern __shared__ uint32_t dsm[];
    uint32_t *sm = dsm;                          // TS + TS/32 words
    uint32_t *smtw = dsm + TS + TS / 32;         // 2^R - 1 twiddles
    const uint32_t tid = threadIdx.x;
    const uint32_t s = p.s;
    const uint32_t cshift = s - WL;
    const uint64_t tile = blockIdx.x;
    const uint64_t cb = tile & ((1ull << cshift) - 1ull);
    const uint64_t hb = tile >> cshift;
    uint32_t *col = p.dev_cols ? p.dev_cols[blockIdx.y] : p.data + (uint64_t)blockIdx.y * p.col_stride;
    const uint32_t *in = p.src ? p.src + (uint64_t)blockIdx.y * p.src_stride : col;
    const uint64_t gbase = (hb << (s + R)) | (cb << WL);

    constexpr int DPT = TS / NT;                // 16 data elements per thread
    // Data loads first (their latency overlaps the twiddle loads).  The
    // vector form moves 4 consecutive tile elements per access: a row of the
    // tile is 2^WL >= 4 contiguous words (or the whole tile is contiguous,
    // WL = 0 with s = 0), and 4-element groups start on multiples of 4.
    uint32_t dv[DPT];
    if (p.vec) {
#pragma unroll
        for (int k = 0; k < DPT / 4; k++) {
            const uint32_t e = 4u * (tid + (uint32_t)k * NT);
            const uint64_t g = gbase | ((uint64_t)(e >> WL) << s) | (e & (W - 1u));
            const uint4 q = *(const uint4 *)(in + (p.src ? (g & p.src_mask) : g));
            dv[4 * k] = q.x; dv[4 * k + 1] = q.y; dv[4 * k + 2] = q.z; dv[4 * k + 3] = q.w;
        }
    } else {
#pragma unroll
        for (int k = 0; k < DPT; k++) {
            const uint32_t e = tid + (uint32_t)k * NT;
            const uint64_t g = gbase | ((uint64_t)(e >> WL) << s) | (e & (W - 1u));
            dv[k] = in[p.src ? (g & p.src_mask) : g];
        }
    }
    // Twiddles of pass layer j are table words h in [hb 2^(R-1-j), (hb+1) 2^(R-1-j)),
    // staged at smtw[2^(R-1-j) - 1 ..]; a flat index f decodes to (layer, offset).
    // All loads are issued before the shared-memory stores.  (Per-layer loops
    // over the contiguous runs measured slower: most of their predicated loads idle.)
    {
        constexpr int TWN = (1 << R) - 1;
        constexpr int TWPT = (TWN + NT - 1) / NT;
        uint32_t tv[TWPT];
#pragma unroll
        for (int k = 0; k < TWPT; k++) {
            uint32_t f = tid + (uint32_t)k * NT;
            if (f < (uint32_t)TWN) {
                uint32_t lg = 31u - __clz(f + 1u);
                uint32_t j = R - 1 - lg;
                uint32_t t = f + 1u - (1u << lg);
                uint32_t L = s + j;
                uint64_t h = (hb << lg) | t;
                tv[k] = L ? __ldg(p.line + p.off.v[L - 1] + h) : circle_tw(p.circle, p.cmode, h);
            }
        }
#pragma unroll
        for (int k = 0; k < TWPT; k++) {
            uint32_t f = tid + (uint32_t)k * NT;
            if (f < (uint32_t)TWN) smtw[f] = tv[k];
        }
    }
    // tid < NT and k NT (resp. 4 tid + q and 4 k NT) have disjoint bits
    const uint32_t ps1 = pad32(tid), ps4 = pad32(4u * tid);
    if (p.vec) {
#pragma unroll
        for (int k = 0; k < DPT / 4; k++) {
            const uint32_t o = 4u * (uint32_t)k * NT;
#pragma unroll
            for (int q = 0; q < 4; q++) sm[ps4 + q + o + (o >> 5)] = dv[4 * k + q];
        }
    } else {
#pragma unroll
        for (int k = 0; k < DPT; k++) {
            const uint32_t o = (uint32_t)k * NT;
            sm[ps1 + o + (o >> 5)] = dv[k];
        }
    }
    __syncthreads();
    run_stages<FWD, R, WL, 0>(sm, smtw, tid);
    if (p.vec) {
#pragma unroll
        for (int k = 0; k < DPT / 4; k++) {
            const uint32_t e = 4u * (tid + (uint32_t)k * NT);
            const uint64_t g = gbase | ((uint64_t)(e >> WL) << s) | (e & (W - 1u));
            const uint32_t o = 4u * (uint32_t)k * NT;
            uint32_t v[4];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const uint32_t w = sm[ps4 + q + o + (o >> 5)];
                v[q] = p.scale != 1u ? mmul(w, p.scale) : w;
            }
            *(uint4 *)(col + g) = make_uint4(v[0], v[1], v[2], v[3]);
        }
    } else {
#pragma unroll
        for (int k = 0; k < DPT; k++) {
            const uint32_t e = tid + (uint32_t)k * NT;
            const uint64_t g = gbase | ((uint64_t)(e >> WL) << s) | (e & (W - 1u));
            const uint32_t o = (uint32_t)k * NT;
            const uint32_t v = sm[ps1 + o + (o >> 5)];
            col[g] = p.scale != 1u ? mmul(v, p.scale) : v;
        }
    }
}

template <bool FWD, int R, int WL>
cudaError_t launch_pass2(const Pass2Args &a, uint64_t tiles, uint32_t n_cols, cudaStream_t st) {
    constexpr int TS = 1 << (R + WL);
    size_t smem = (TS + TS / 32 + (1 << R)) * 4;
    ntt_pass2_kernel<FWD, R, WL><<<dim3((unsigned)tiles, n_cols), TS / 16, smem, st>>>(a);
    return cudaGetLastError();
}

template <bool FWD>
cudaError_t dispatch_pass2(uint32_t r, uint32_t wl, const Pass2Args &a, uint64_t tiles, uint32_t n_cols,
                           cudaStream_t st) {
    if (wl == 0) {
        switch (r) {
        case 4: return launch_pass2<FWD, 4, 0>(a, tiles, n_cols, st);
        case 5: return launch_pass2<FWD, 5, 0>(a, tiles, n_cols, st);
        case 6: return launch_pass2<FWD, 6, 0>(a, tiles, n_cols, st);
        case 7: return launch_pass2<FWD, 7, 0>(a, tiles, n_cols, st);
        case 8: return launch_pass2<FWD, 8, 0>(a, tiles, n_cols, st);
        case 9: return launch_pass2<FWD, 9, 0>(a, tiles, n_cols, st);
        case 10: return launch_pass2<FWD, 10, 0>(a, tiles, n_cols, st);
        case 11: return launch_pass2<FWD, 11, 0>(a, tiles, n_cols, st);
        case 12: return launch_pass2<FWD, 12, 0>(a, tiles, n_cols, st);
        }
    } else if (wl + r == 12) {
        switch (r) {
        case 3: return launch_pass2<FWD, 3, 9>(a, tiles, n_cols, st);
        case 4: return launch_pass2<FWD, 4, 8>(a, tiles, n_cols, st);
        case 5: return launch_pass2<FWD, 5, 7>(a, tiles, n_cols, st);
        case 6: return launch_pass2<FWD, 6, 6>(a, tiles, n_cols, st);
        case 7: return launch_pass2<FWD, 7, 5>(a, tiles, n_cols, st);
        case 8: return launch_pass2<FWD, 8, 4>(a, tiles, n_cols, st);
        case 9: return launch_pass2<FWD, 9, 3>(a, tiles, n_cols, st);
        }
    }
    return cudaErrorInvalidValue;
}

bool g_attr_done = false;

cudaError_t ensure_attrs() {
    if (g_attr_done) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(ntt_pass_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)(kMaxTileWords * 4));
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(ntt_pass_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(kMaxTileWords * 4));
    if (e == cudaSuccess) g_attr_done = true;
    return e;
}

}  // namespace

NttTables stwo_tables(const uint32_t *tw, uint32_t log_n) {
    NttTables t;
    t.line = tw;
    t.circle = tw;
    t.circle_mode = 1u;
    for (uint32_t l = 0; l < 32; l++)
        t.off[l] = (l + 1 < log_n) ? (uint32_t)((1ull << (log_n - 1)) - (1ull << (log_n - 1 - l))) : 0u;
    return t;
}

void ntt_table_offsets(uint32_t log_n, uint32_t off[32]) {
    uint64_t m = 1ull << log_n;
    for (uint32_t l = 0; l < 32; l++) off[l] = (l + 1 < log_n) ? (uint32_t)(m - (m >> l)) : 0u;
}

namespace {

// Pass-plan knobs per device and transform length (in layers): the bottom
// pass's maximum layers (10..12) and the upper passes' maximum (6..9).  The
// autotuner writes them; every choice computes the same values.
struct PlanKnobs { uint8_t bottom, upper; };
PlanKnobs g_knobs[64][32];
bool g_knobs_init[64] = {false};

PlanKnobs knobs_for(uint32_t total) {
    int dev = 0;
    cudaGetDevice(&dev);
    PlanKnobs k{12, 9};
    if (dev >= 0 && dev < 64 && g_knobs_init[dev] && total < 32 && g_knobs[dev][total].bottom) k = g_knobs[dev][total];
    return k;
}

}  // namespace

// Pass plan for `total` layers (0 .. total-1): a bottom pass of up to
// `bottom` layers on contiguous tiles (WL = 0), then passes of 3..`upper`
// layers, sizes balanced, on tiles of 2^(12-R) contiguous columns (every tile
// 4096 elements; rows of at least 8 words = one 32-byte sector).  An upper
// pass starting at layer s reads rows 2^s apart, so its 2^(12-R) columns
// must fit in one row gap: 12 - R <= s.  Transforms of at most 12 layers are
// therefore one bottom pass, and a longer one keeps a bottom pass of at
// least 9 layers (bottom_max >= 9; at least 10 after the 3-layer rule).
// Transforms of fewer than 4 layers use the one-tile shared-memory kernel.
uint32_t ntt_plan(uint32_t total, uint32_t bottom_max, uint32_t upper_max, uint32_t ps[32], uint32_t pr[32],
                  uint32_t pw[32]) {
    uint32_t np = 0;
    if (bottom_max < 9u) bottom_max = 9u;
    uint32_t bottom = (total <= 12u || total < bottom_max) ? total : bottom_max;
    if (total > bottom && total - bottom < 3u) bottom = total - 3u;  // leave at least 3 layers above
    ps[np] = 0; pr[np] = bottom; pw[np] = 0; np++;
    uint32_t rest = total - bottom;
    if (rest) {
        uint32_t nu = (rest + upper_max - 1u) / upper_max;
        if (rest < 3u * nu) nu = rest / 3u;  // every upper pass has at least 3 layers
        uint32_t lo = bottom;
        for (uint32_t i = 0; i < nu; i++) {
            uint32_t r = rest / nu + (i < rest % nu ? 1u : 0u);
            ps[np] = lo; pr[np] = r; pw[np] = 12u - r; np++;
            lo += r;
        }
    }
    return np;
}

void ntt_knobs_set(int dev, uint32_t total, uint32_t bottom, uint32_t upper) {
    if (dev < 0 || dev >= 64 || total >= 32) return;
    if (!g_knobs_init[dev]) {
        memset(g_knobs[dev], 0, sizeof(g_knobs[dev]));
        g_knobs_init[dev] = true;
    }
    g_knobs[dev][total] = PlanKnobs{(uint8_t)bottom, (uint8_t)upper};
}

void ntt_knobs_get(uint32_t total, uint32_t *bottom, uint32_t *upper) {
    PlanKnobs k = knobs_for(total);
    *bottom = k.bottom;
    *upper = k.upper;
}

namespace {
uint32_t plan_passes(uint32_t total, uint32_t ps[32], uint32_t pr[32], uint32_t pw[32]) {
    PlanKnobs k = knobs_for(total);
    return ntt_plan(total, k.bottom, k.upper, ps, pr, pw);
}
}  // namespace

uint32_t ntt_pass_count(uint32_t layers) {
    if (layers == 0) return 0;
    if (layers < 4) return 1;
    uint32_t ps[32], pr[32], pw[32];
    return plan_passes(layers, ps, pr, pw);
}

cudaError_t ntt_transform(uint32_t *data, uint32_t *const *dev_cols, uint64_t col_stride, uint32_t n_cols,
                          uint32_t log_n, const NttTables &tw, bool forward, const uint32_t *src,
                          uint32_t src_log, cudaStream_t stream) {
    return ntt_transform_planned(data, dev_cols, col_stride, n_cols, log_n, tw, forward, src, src_log, 0, 0, stream);
}

cudaError_t ntt_transform_planned(uint32_t *data, uint32_t *const *dev_cols, uint64_t col_stride, uint32_t n_cols,
                                  uint32_t log_n, const NttTables &tw, bool forward, const uint32_t *src,
                                  uint32_t src_log, uint32_t bottom_max, uint32_t upper_max, cudaStream_t stream) {
    if (log_n == 0 || n_cols == 0) return cudaSuccess;
    if (src && !forward && src_log != log_n) return cudaErrorInvalidValue;
    cudaError_t e = ensure_attrs();
    if (e != cudaSuccess) return e;
    const uint32_t total = (src && forward) ? src_log : log_n;  // layers applied: total-1 .. 0
    PassOff off;
    for (int i = 0; i < 32; i++) off.v[i] = tw.off[i];
    uint32_t e2 = (30u * log_n) % 31u;
    uint32_t inv_n = e2 == 0 ? 1u : (1u << e2);
    const uint64_t mask = src ? ((1ull << src_log) - 1ull) : ~0ull;
    const uint64_t src_stride = src ? (1ull << src_log) : 0ull;
    if (total < 4) {
        // tiny transform: one tile of 2^total rows, single-layer smem kernel
        uint32_t r = total, wlog = 0, tsz = 1u << r;
        uint64_t tiles = (1ull << log_n) / tsz;
        if (forward)
            ntt_pass_kernel<true><<<dim3((unsigned)tiles, n_cols), 32, tsz * 4, stream>>>(
                data, dev_cols, col_stride, src, mask, src_stride, tw.line, tw.circle, tw.circle_mode, off, 0, r, wlog,
                1u);
        else
            ntt_pass_kernel<false><<<dim3((unsigned)tiles, n_cols), 32, tsz * 4, stream>>>(
                data, dev_cols, col_stride, src, mask, src_stride, tw.line, tw.circle, tw.circle_mode, off, 0, r,
                wlog, inv_n);
        return cudaGetLastError();
    }
    uint32_t ps[32], pr[32], pw[32];
    const uint32_t np = bottom_max ? ntt_plan(total, bottom_max, upper_max, ps, pr, pw) : plan_passes(total, ps, pr, pw);
    // 16-byte accesses of 4 consecutive elements: contiguous columns with
    // 16-byte aligned bases (a device pointer array is not inspected on the
    // host, so it keeps the scalar form), a source of at least 4 words
    const bool vec = !dev_cols && (((uintptr_t)data & 15u) == 0) && (n_cols == 1 || col_stride % 4u == 0) &&
                     (!src || ((((uintptr_t)src & 15u) == 0) && src_log >= 2 && (n_cols == 1 || src_stride % 4u == 0)));
    for (uint32_t q = 0; q < np; q++) {
        uint32_t i = forward ? np - 1u - q : q;   // forward: top pass first
        Pass2Args a;
        a.data = data; a.dev_cols = dev_cols; a.col_stride = col_stride;
        a.src = (q == 0 && src) ? src : nullptr;
        a.src_mask = mask; a.src_stride = src_stride;
        a.line = tw.line; a.circle = tw.circle; a.cmode = tw.circle_mode; a.off = off;
        a.s = ps[i];
        a.scale = (!forward && q == np - 1u) ? inv_n : 1u;
        a.vec = (vec && (pw[i] >= 2u || ps[i] == 0u)) ? 1u : 0u;
        uint64_t tiles = (1ull << log_n) >> (pr[i] + pw[i]);
        e = forward ? dispatch_pass2<true>(pr[i], pw[i], a, tiles, n_cols, stream)
                    : dispatch_pass2<false>(pr[i], pw[i], a, tiles, n_cols, stream);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t ntt_single_layer(uint32_t *data, const uint32_t *tw, uint32_t layer_idx, uint32_t log_n, bool forward,
                             cudaStream_t stream) {
    uint64_t half = (1ull << log_n) / 2;
    if (!half) return cudaSuccess;
    ntt_layer_kernel<<<blocks_for(half, 256), 256, 0, stream>>>(data, tw, layer_idx, half, forward ? 1 : 0);
    return cudaGetLastError();
}

}  // namespace vx
