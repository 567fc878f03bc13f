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

// One layer over a whole array; with `cols` non-null, over column
// cols[blockIdx.y] instead of d.
__global__ void ntt_layer_kernel(uint32_t *d, uint32_t *const *cols, const uint32_t *__restrict__ tw, uint32_t L,
                                 uint64_t half_n, int fwd) {
    uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= half_n) return;
    if (cols) d = cols[blockIdx.y];
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
// columns) held in shared memory by NT threads, DPT = 2^(R+WL) / NT = 16 or
// 32 elements per thread.  The pass's R layers run in stages of up to 4
// layers; in a stage each thread takes groups of the 16 elements that
// differ in one contiguous block of 4 tile bits [A, A+4) covering the
// stage's layer bits, and does all the stage's butterflies on them in
// registers.  Between stages the tile goes through shared memory (padded by
// one word per 32 to spread the strided accesses over the banks).  The
// tile's twiddles (2^R - 1 words, one contiguous run of the reference table
// per layer) are staged in shared memory once per tile, doubled when the
// butterflies multiply with mmul_t2 (kTwiddleX2).  All values stay canonical.
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
    uint32_t scale;   // output scale (1 = none)
    uint32_t vec;     // 1: columns and source 16-byte aligned, 4 consecutive elements per access
    uint32_t hb_log;  // > 0: the 2^hb_log tiles that read the same source tile are consecutive blocks
};

// Butterfly products: with a doubled twiddle (mmul_t2: one multiply, one
// shift-add, one conditional subtract) or the plain one (mmul: a fold of the
// 64-bit product); both exact, the choice is the faster on the device.
constexpr bool kTwiddleX2 = true;
__device__ __forceinline__ uint32_t tw_stage(uint32_t t) { return kTwiddleX2 ? 2u * t : t; }
__device__ __forceinline__ uint32_t tw_mul(uint32_t v, uint32_t t) { return kTwiddleX2 ? mmul_t2(v, t) : mmul(v, t); }

__device__ __forceinline__ uint32_t pad32(uint32_t e) { return e + (e >> 5); }
// Word offset of the staged twiddles after a padded tile of ts words, rounded
// up to 16 bytes for the vector reads.
constexpr uint32_t tw_base(uint32_t ts) { return (ts + ts / 32 + 3u) & ~3u; }
// pad32(a | b) = pad32(a) + b + (b >> 5) when a and b have no bit in common
// (a shift distributes over OR, and an OR of disjoint fields is a sum).  The
// stage and tile accesses below are all of this form with b a compile-time
// offset, so each thread computes one padded base and the accesses use
// immediate offsets.

// One layer of a stage on the 16 register values of a group.  The layer's
// 16 >> (rb + 1) twiddles are one aligned run: layer j sits at
// smtw[2^(R-1-j) ..] and base >> S (S = A + rb + 1, base's bits [A, A+4)
// zero) is a multiple of the run length, so the run is read with 16-, 8- or
// 4-byte loads.
template <bool FWD, int R, int WL, int A, int J>
__device__ __forceinline__ void stage_layer(uint32_t v[16], uint32_t base, const uint32_t *smtw) {
    constexpr int rb = J + WL - A;  // register bit of layer J
    constexpr int S = J + 1 + WL;   // tile-index shift giving the twiddle index
    constexpr int RL = 8 >> rb;
    const uint32_t *tp = smtw + (1u << (R - 1 - J)) + (base >> S);
    uint32_t tw[RL];
    if constexpr (RL >= 4) {
#pragma unroll
        for (int q = 0; q < RL / 4; q++) {
            const uint4 x = ((const uint4 *)tp)[q];
            tw[4 * q] = x.x; tw[4 * q + 1] = x.y; tw[4 * q + 2] = x.z; tw[4 * q + 3] = x.w;
        }
    } else if constexpr (RL == 2) {
        const uint2 x = *(const uint2 *)tp;
        tw[0] = x.x; tw[1] = x.y;
    } else {
        tw[0] = tp[0];
    }
#pragma unroll
    for (int i0 = 0; i0 < 16; i0++) {
        if (i0 & (1 << rb)) continue;
        const int i1 = i0 | (1 << rb);
        const uint32_t t = tw[i0 >> (rb + 1)];
        if (FWD) {
            const uint32_t x = tw_mul(v[i1], t);
            v[i1] = msub(v[i0], x);
            v[i0] = madd(v[i0], x);
        } else {
            const uint32_t a = v[i0], b = v[i1];
            v[i0] = madd(a, b);
            v[i1] = tw_mul(msub(a, b), t);
        }
    }
}

template <bool FWD, int R, int WL, int A, int LO, int HI, int JJ>
__device__ __forceinline__ void stage_layers(uint32_t v[16], uint32_t base, const uint32_t *smtw) {
    if constexpr (JJ < HI - LO) {
        constexpr int J = FWD ? (HI - 1 - JJ) : (LO + JJ);
        stage_layer<FWD, R, WL, A, J>(v, base, smtw);
        stage_layers<FWD, R, WL, A, LO, HI, JJ + 1>(v, base, smtw);
    }
}

template <bool FWD, int R, int WL, int NT, int LO, int HI, int A>
__device__ __forceinline__ void ntt_stage(uint32_t *sm, const uint32_t *smtw, uint32_t tid) {
    constexpr int G = (1 << (R + WL)) / 16 / NT;  // 16-element groups per thread
#pragma unroll
    for (int g = 0; g < G; g++) {
        const uint32_t bi = tid + (uint32_t)g * NT;
        const uint32_t base = (bi & ((1u << A) - 1u)) | ((bi >> A) << (A + 4));  // bits [A, A+4) zero
        const uint32_t pb = pad32(base);
        uint32_t v[16];
#pragma unroll
        for (int i = 0; i < 16; i++) v[i] = sm[pb + ((uint32_t)i << A) + (((uint32_t)i << A) >> 5)];
        stage_layers<FWD, R, WL, A, LO, HI, 0>(v, base, smtw);
#pragma unroll
        for (int i = 0; i < 16; i++) sm[pb + ((uint32_t)i << A) + (((uint32_t)i << A) >> 5)] = v[i];
    }
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

template <bool FWD, int R, int WL, int NT, int K>
__device__ __forceinline__ void run_stages(uint32_t *sm, const uint32_t *smtw, uint32_t tid) {
    if constexpr (K < StageIdx<FWD, R, WL, K>::NST) {
        using St = StageIdx<FWD, R, WL, K>;
        ntt_stage<FWD, R, WL, NT, St::LO, St::HI, St::A>(sm, smtw, tid);
        __syncthreads();
        run_stages<FWD, R, WL, NT, K + 1>(sm, smtw, tid);
    }
}

// Resident threads per SM the pass kernels are compiled for (registers per
// thread = 65536 / this).
#ifndef VX_NTT_THREADS_PER_SM
#define VX_NTT_THREADS_PER_SM 1024
#endif
constexpr int min_blocks_for(int nt) {
    return (VX_NTT_THREADS_PER_SM / nt) < 32 ? (VX_NTT_THREADS_PER_SM / nt) : 32;
}

// One tile of one column: tile index `tile` of column `ci`.
template <bool FWD, int R, int WL, int NT>
__device__ __forceinline__ void tile_pass(const Pass2Args &p, uint64_t tile, uint32_t ci, uint32_t *dsm) {
    constexpr int TB = R + WL, TS = 1 << TB, W = 1 << WL;
    constexpr int DPT = TS / NT;                // 16 or 32 data elements per thread
    static_assert(DPT == 16 || DPT == 32, "16 or 32 elements per thread");
    uint32_t *sm = dsm;                          // TS + TS/32 words
    uint32_t *smtw = dsm + tw_base(TS);          // 2^R words: layer j's twiddles at [2^(R-1-j), 2^(R-j))
    const uint32_t tid = threadIdx.x;
    const uint32_t s = p.s;
    // tile = (hb, cb): the high index bits above the pass and the column
    // block.  Column blocks are consecutive by default (neighbouring blocks
    // share DRAM pages); the first pass of an LDE, whose hb values above the
    // source's length are replicas reading the same source tile, puts those
    // replicas in consecutive blocks so the source comes from L2 after its
    // first read.
    const uint32_t cshift = s - WL;
    const uint64_t cb = p.hb_log ? tile >> p.hb_log : tile & ((1ull << cshift) - 1ull);
    const uint64_t hb = p.hb_log ? tile & ((1ull << p.hb_log) - 1ull) : tile >> cshift;
    uint32_t *col = p.dev_cols ? p.dev_cols[ci] : p.data + (uint64_t)ci * p.col_stride;
    const uint32_t *in = p.src ? p.src + (uint64_t)ci * p.src_stride : col;
    const uint64_t gbase = (hb << (s + R)) | (cb << WL);

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
    // staged at smtw[2^(R-1-j) ..]; a flat index f decodes to (layer, offset).
    // Loads are issued in batches of up to 8 per thread before their stores.
    {
        constexpr int TWN = (1 << R) - 1;
        constexpr int TWPT = (TWN + NT - 1) / NT;
        constexpr int BATCH = TWPT < 8 ? TWPT : 8;
#pragma unroll
        for (int k0 = 0; k0 < TWPT; k0 += BATCH) {
            uint32_t tv[BATCH];
#pragma unroll
            for (int kk = 0; kk < BATCH; kk++) {
                const uint32_t f = tid + (uint32_t)(k0 + kk) * NT;
                if (k0 + kk < TWPT && f < (uint32_t)TWN) {
                    const uint32_t lg = 31u - __clz(f + 1u);
                    const uint32_t j = R - 1 - lg;
                    const uint32_t t = f + 1u - (1u << lg);
                    const uint32_t L = s + j;
                    const uint64_t h = (hb << lg) | t;
                    tv[kk] = L ? __ldg(p.line + p.off.v[L - 1] + h) : circle_tw(p.circle, p.cmode, h);
                }
            }
#pragma unroll
            for (int kk = 0; kk < BATCH; kk++) {
                const uint32_t f = tid + (uint32_t)(k0 + kk) * NT;
                if (k0 + kk < TWPT && f < (uint32_t)TWN) smtw[f + 1u] = tw_stage(tv[kk]);
            }
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
    run_stages<FWD, R, WL, NT, 0>(sm, smtw, tid);
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
            const uint32_t w = sm[ps1 + o + (o >> 5)];
            col[g] = p.scale != 1u ? mmul(w, p.scale) : w;
        }
    }
}

// Passes are programmatic dependent launches (launch_pdl): a pass's blocks may
// be scheduled while the previous kernel on the stream drains, and wait here
// before reading what it wrote.
template <bool FWD, int R, int WL, int NT>
__global__ void __launch_bounds__(NT, min_blocks_for(NT)) ntt_tile_kernel(Pass2Args p) {
    extern __shared__ uint32_t dsm[];
    pdl_wait();
    tile_pass<FWD, R, WL, NT>(p, blockIdx.x, blockIdx.y, dsm);
}

// Several transforms of different lengths in one launch: group g's columns
// and tiles are blocks [first[g], first[g+1]) of a 1-D grid, each group with
// its own pass shape, all on 4096-element tiles of 256 threads (bottom
// passes of 12 layers, upper passes of 3..9).  Used for columns of uneven
// sizes, so a small size group does not run as a launch of its own that
// leaves most SMs idle.
constexpr uint32_t kMaxNttGroups = 4;
struct MultiPassArgs {
    Pass2Args g[kMaxNttGroups];
    uint32_t R[kMaxNttGroups];
    uint32_t first[kMaxNttGroups + 1];
    uint32_t tiles[kMaxNttGroups];  // tiles per column
    uint32_t n_groups;
};

template <bool FWD>
__global__ void __launch_bounds__(256, 4) ntt_multi_kernel(MultiPassArgs a) {
    extern __shared__ uint32_t dsm[];
    pdl_wait();
    const uint32_t b = blockIdx.x;
    uint32_t gi = 0;
    while (gi + 1 < a.n_groups && b >= a.first[gi + 1]) gi++;
    const uint32_t local = b - a.first[gi];
    const uint32_t ci = local / a.tiles[gi];
    const uint64_t tile = local - ci * a.tiles[gi];
    const Pass2Args &p = a.g[gi];
    switch (a.R[gi]) {
    case 12: tile_pass<FWD, 12, 0, 256>(p, tile, ci, dsm); break;
    case 9: tile_pass<FWD, 9, 3, 256>(p, tile, ci, dsm); break;
    case 8: tile_pass<FWD, 8, 4, 256>(p, tile, ci, dsm); break;
    case 7: tile_pass<FWD, 7, 5, 256>(p, tile, ci, dsm); break;
    case 6: tile_pass<FWD, 6, 6, 256>(p, tile, ci, dsm); break;
    case 5: tile_pass<FWD, 5, 7, 256>(p, tile, ci, dsm); break;
    case 4: tile_pass<FWD, 4, 8, 256>(p, tile, ci, dsm); break;
    case 3: tile_pass<FWD, 3, 9, 256>(p, tile, ci, dsm); break;
    default: break;
    }
}

// Threads per tile: 16 elements per thread up to 2^12-element tiles (at most
// 256 threads), 32 for 2^13 (256 threads) and 2^14 (512 threads).
constexpr int threads_for(int tb) { return tb <= 12 ? (1 << tb) / 16 : (1 << tb) / 32; }

template <bool FWD, int R, int WL>
cudaError_t launch_pass2(const Pass2Args &a, uint64_t tiles, uint32_t n_cols, cudaStream_t st) {
    constexpr int TB = R + WL, TS = 1 << TB, NT = threads_for(TB);
    const size_t smem = (tw_base(TS) + (1u << R)) * 4;
    if (smem > 48 * 1024) {  // large tiles need the opt-in shared-memory size, once per device
        static bool attr_done[64] = {false};
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return e;
        if (dev < 0 || dev >= 64 || !attr_done[dev]) {
            e = cudaFuncSetAttribute(ntt_tile_kernel<FWD, R, WL, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem);
            if (e != cudaSuccess) return e;
            if (dev >= 0 && dev < 64) attr_done[dev] = true;
        }
    }
    return launch_pdl(ntt_tile_kernel<FWD, R, WL, NT>, dim3((unsigned)tiles, n_cols), dim3(NT), smem, st, a);
}

// Pass shapes the kernels are built for (ntt_plan only emits these):
// bottom passes (WL = 0) of 4..14 layers; upper passes of 3..9 layers on
// 2^12-element tiles (WL = 12 - R), of 10 and 11 layers on 2^13-element
// tiles (WL = 13 - R) and of 12 layers on 2^14-element tiles (WL = 2): rows
// of at least 16 bytes.
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
        case 13: return launch_pass2<FWD, 13, 0>(a, tiles, n_cols, st);
        case 14: return launch_pass2<FWD, 14, 0>(a, tiles, n_cols, st);
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
    } else if (wl + r == 13) {
        switch (r) {
        case 10: return launch_pass2<FWD, 10, 3>(a, tiles, n_cols, st);
        case 11: return launch_pass2<FWD, 11, 2>(a, tiles, n_cols, st);
        }
    } else if (wl + r == 14 && r == 12) {
        return launch_pass2<FWD, 12, 2>(a, tiles, n_cols, st);
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

// Pass-plan knobs per device and transform length (log2 of the elements): the bottom
// pass's maximum layers (9..14) and the upper passes' maximum (3..12).  The
// autotuner writes them; every choice computes the same values.  Larger
// tiles (2 passes for 24 layers) measured slower than 4096-element tiles
// with 3 passes: 32 elements per thread lose more to load latency and
// barriers than the third pass costs in HBM traffic.
struct PlanKnobs { uint8_t bottom, upper; };
PlanKnobs g_knobs[64][32];
bool g_knobs_init[64] = {false};

PlanKnobs knobs_for(uint32_t total) {
    int dev = 0;
    cudaGetDevice(&dev);
    PlanKnobs k{11, 8};  // the fastest plans measured on a B200 without tuning (3 passes for 24..27 layers)
    if (dev >= 0 && dev < 64 && g_knobs_init[dev] && total < 32 && g_knobs[dev][total].bottom) k = g_knobs[dev][total];
    return k;
}

}  // namespace

// Pass plan for `total` layers (0 .. total-1): a bottom pass of up to
// `bottom` layers on contiguous tiles (WL = 0), then passes of 3..`upper`
// layers, sizes balanced.  An upper pass of R <= 9 layers runs on tiles of
// 2^12 elements, 2^(12-R) contiguous columns (rows of at least 8 words, one
// 32-byte sector); one of 10 or 11 layers on tiles of 2^13 elements, 2^(13-R)
// columns; one of 12 layers on tiles of 2^14 elements, 4 columns (rows of 16
// bytes).  An upper pass starting at layer s reads
// rows 2^s apart, so its columns must fit in one row gap: WL <= s.  A
// transform of at most max(12, bottom) layers is therefore one bottom pass,
// and a longer one keeps a bottom pass of at least 9 layers (bottom_max >=
// 9), so every WL (at most 9) fits.  Transforms of fewer than 4 layers use
// the one-tile shared-memory kernel.
uint32_t ntt_plan(uint32_t total, uint32_t bottom_max, uint32_t upper_max, uint32_t ps[32], uint32_t pr[32],
                  uint32_t pw[32]) {
    uint32_t np = 0;
    if (bottom_max < 9u) bottom_max = 9u;
    if (bottom_max > 14u) bottom_max = 14u;
    if (upper_max < 3u) upper_max = 3u;
    if (upper_max > 12u) upper_max = 12u;
    uint32_t bottom = (total <= 12u || total <= bottom_max) ? total : bottom_max;
    if (total > bottom && total - bottom < 3u) bottom = total - 3u;  // leave at least 3 layers above
    ps[np] = 0; pr[np] = bottom; pw[np] = 0; np++;
    uint32_t rest = total - bottom;
    if (rest) {
        uint32_t nu = (rest + upper_max - 1u) / upper_max;
        if (rest < 3u * nu) nu = rest / 3u;  // every upper pass has at least 3 layers
        uint32_t lo = bottom;
        for (uint32_t i = 0; i < nu; i++) {
            uint32_t r = rest / nu + (i < rest % nu ? 1u : 0u);
            ps[np] = lo; pr[np] = r; pw[np] = (r <= 9u ? 12u : r <= 11u ? 13u : 14u) - r; np++;
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
// The knobs are looked up by the transform's length in elements (2^log_n),
// which sets its memory regime (an LDE applies 24 layers to 2^26 elements
// in HBM, an interpolation of 2^24 elements stays in L2), and applied to
// the `total` layers it runs.
uint32_t plan_passes(uint32_t total, uint32_t log_n, uint32_t ps[32], uint32_t pr[32], uint32_t pw[32]) {
    PlanKnobs k = knobs_for(log_n);
    return ntt_plan(total, k.bottom, k.upper, ps, pr, pw);
}
}  // namespace

uint32_t ntt_pass_count(uint32_t layers, uint32_t log_n) {
    if (layers == 0) return 0;
    if (layers < 4) return 1;
    uint32_t ps[32], pr[32], pw[32];
    return plan_passes(layers, log_n ? log_n : layers, ps, pr, pw);
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
    const uint32_t np =
        bottom_max ? ntt_plan(total, bottom_max, upper_max, ps, pr, pw) : plan_passes(total, log_n, ps, pr, pw);
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
        // the first forward pass of an LDE reads each source tile for 2^(log_n - src_log) replicas
        a.hb_log = (q == 0 && src && forward && log_n > src_log && ps[i] + pr[i] == src_log) ? log_n - src_log : 0u;
        uint64_t tiles = (1ull << log_n) >> (pr[i] + pw[i]);
        e = forward ? dispatch_pass2<true>(pr[i], pw[i], a, tiles, n_cols, stream)
                    : dispatch_pass2<false>(pr[i], pw[i], a, tiles, n_cols, stream);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t ntt_transform_groups(const NttGroup *grp, uint32_t n_groups, bool forward, cudaStream_t stream,
                                 uint32_t *launches) {
    // groups whose transform is exactly a 12-layer bottom pass plus one upper
    // pass of 3..9 layers (15..21 layers) share the launches; the others run
    // as transforms of their own
    if (n_groups > 64) return cudaErrorInvalidValue;
    bool merge[64] = {false};
    uint32_t n_merge = 0;
    for (uint32_t g = 0; g < n_groups; g++) {
        const uint32_t total = (grp[g].src && forward) ? grp[g].src_log : grp[g].log_n;
        merge[g] = n_merge < kMaxNttGroups && grp[g].n_cols > 0 && total >= 15 && total <= 21 &&
                   !(grp[g].src && !forward && grp[g].src_log != grp[g].log_n);
        n_merge += merge[g];
    }
    for (uint32_t g = 0; g < n_groups; g++) {
        if (merge[g] && n_merge >= 2) continue;
        const NttGroup &G = grp[g];
        cudaError_t e = ntt_transform(G.data, nullptr, G.col_stride, G.n_cols, G.log_n, G.tw, forward, G.src,
                                      G.src_log, stream);
        if (e != cudaSuccess) return e;
        if (launches) *launches += ntt_pass_count((G.src && forward) ? G.src_log : G.log_n, G.log_n);
    }
    if (n_merge < 2) return cudaSuccess;
    static bool attr_done[64] = {false};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const size_t smem = (tw_base(4096) + 4096) * 4;
    if (dev < 0 || dev >= 64 || !attr_done[dev]) {
        e = cudaFuncSetAttribute(forward ? ntt_multi_kernel<true> : ntt_multi_kernel<false>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(forward ? ntt_multi_kernel<false> : ntt_multi_kernel<true>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        if (dev >= 0 && dev < 64) attr_done[dev] = true;
    }
    for (uint32_t q = 0; q < 2; q++) {
        const uint32_t pi = forward ? 1u - q : q;  // forward: the upper pass first
        MultiPassArgs a;
        memset(&a, 0, sizeof(a));
        uint32_t blocks = 0;
        for (uint32_t g = 0; g < n_groups; g++) {
            if (!merge[g]) continue;
            const NttGroup &G = grp[g];
            const uint32_t total = (G.src && forward) ? G.src_log : G.log_n;
            const uint32_t r = pi == 0 ? 12u : total - 12u, wl = pi == 0 ? 0u : 12u - r;
            const uint32_t e2 = (30u * G.log_n) % 31u;
            Pass2Args &p = a.g[a.n_groups];
            p.data = G.data; p.dev_cols = nullptr; p.col_stride = G.col_stride;
            p.src = (q == 0 && G.src) ? G.src : nullptr;
            p.src_mask = G.src ? ((1ull << G.src_log) - 1ull) : ~0ull;
            p.src_stride = G.src ? (1ull << G.src_log) : 0ull;
            p.line = G.tw.line; p.circle = G.tw.circle; p.cmode = G.tw.circle_mode;
            for (int i = 0; i < 32; i++) p.off.v[i] = G.tw.off[i];
            p.s = pi == 0 ? 0u : 12u;
            p.scale = (!forward && q == 1u) ? (e2 == 0 ? 1u : (1u << e2)) : 1u;
            p.vec = ((((uintptr_t)G.data & 15u) == 0) && (G.n_cols == 1 || G.col_stride % 4u == 0) &&
                     (!G.src || ((((uintptr_t)G.src & 15u) == 0) && G.src_log >= 2))) ? 1u : 0u;
            p.hb_log = (q == 0 && G.src && forward && G.log_n > G.src_log && p.s + r == G.src_log)
                           ? G.log_n - G.src_log : 0u;
            a.R[a.n_groups] = r;
            a.tiles[a.n_groups] = (uint32_t)((1ull << G.log_n) >> 12);
            a.first[a.n_groups] = blocks;
            blocks += a.tiles[a.n_groups] * G.n_cols;
            a.n_groups++;
            (void)wl;
        }
        a.first[a.n_groups] = blocks;
        e = launch_pdl(forward ? ntt_multi_kernel<true> : ntt_multi_kernel<false>, dim3(blocks), dim3(256), smem,
                       stream, a);
        if (e != cudaSuccess) return e;
        if (launches) *launches += 1;
    }
    return cudaSuccess;
}

cudaError_t ntt_single_layer(uint32_t *data, const uint32_t *tw, uint32_t layer_idx, uint32_t log_n, bool forward,
                             cudaStream_t stream) {
    uint64_t half = (1ull << log_n) / 2;
    if (!half) return cudaSuccess;
    ntt_layer_kernel<<<blocks_for(half, 256), 256, 0, stream>>>(data, nullptr, tw, layer_idx, half, forward ? 1 : 0);
    return cudaGetLastError();
}

cudaError_t ntt_single_layer_cols(uint32_t *const *dev_cols, uint32_t n_cols, const uint32_t *tw, uint32_t layer_idx,
                                  uint32_t log_n, bool forward, cudaStream_t stream) {
    uint64_t half = (1ull << log_n) / 2;
    if (!half || !n_cols) return cudaSuccess;
    ntt_layer_kernel<<<dim3(blocks_for(half, 256), n_cols), 256, 0, stream>>>(nullptr, dev_cols, tw, layer_idx, half,
                                                                            forward ? 1 : 0);
    return cudaGetLastError();
}

}  // namespace vx
