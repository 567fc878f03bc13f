// Circle NTT passes for sm_100a (see vx_ntt.cuh for the layout).
#include "vx_ntt.cuh"
#include "vx_field.cuh"
#include "vx_common.cuh"

namespace vx {

namespace {

constexpr uint32_t kMaxPassLayers = 11;  // 2^11 rows x 8 columns x 4 B = 64 KB tile
constexpr uint32_t kMaxTileWords = (1u << kMaxPassLayers) * 8u;

struct PassOff { uint32_t v[32]; };

template <bool FWD>
__global__ void __launch_bounds__(512) ntt_pass_kernel(
    uint32_t *data, uint32_t *const *dev_cols, uint64_t col_stride,
    const uint32_t *src, uint64_t src_mask, uint64_t src_stride,
    const uint32_t *__restrict__ line, const uint32_t *__restrict__ circle, PassOff off,
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
        const uint32_t *tw = L ? line + off.v[L - 1] : circle;
        for (uint32_t b = threadIdx.x; b < nb; b += blockDim.x) {
            uint32_t c = b & (W - 1u), p = b >> wlog;
            uint32_t row0 = ((p >> j) << (j + 1)) | (p & ((1u << j) - 1u));
            uint32_t e0 = (row0 << wlog) | c, e1 = e0 + (1u << (j + wlog));
            uint64_t h = (hb << (r - 1u - j)) | (uint64_t)(row0 >> (j + 1));
            uint32_t t = __ldg(tw + h);
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

void ntt_table_offsets(uint32_t log_n, uint32_t off[32]) {
    uint64_t m = 1ull << log_n;
    for (uint32_t l = 0; l < 32; l++) off[l] = (l + 1 < log_n) ? (uint32_t)(m - (m >> l)) : 0u;
}

cudaError_t ntt_transform(uint32_t *data, uint32_t *const *dev_cols, uint64_t col_stride, uint32_t n_cols,
                          uint32_t log_n, const NttTables &tw, bool forward, const uint32_t *src,
                          uint32_t src_log, cudaStream_t stream) {
    if (log_n == 0 || n_cols == 0) return cudaSuccess;
    cudaError_t e = ensure_attrs();
    if (e != cudaSuccess) return e;
    const uint32_t top = (src ? src_log : log_n) - 1u;  // highest layer applied
    const uint32_t total = top + 1u;
    const uint32_t np = (total + kMaxPassLayers - 1u) / kMaxPassLayers;
    // pass ranges from the top down: sizes as even as possible
    uint32_t ps[32], pr[32];
    uint32_t hi = total;
    for (uint32_t i = 0; i < np; i++) {
        uint32_t r = total / np + (i < total % np ? 1u : 0u);
        pr[i] = r;
        ps[i] = hi - r;
        hi -= r;
    }
    PassOff off;
    for (int i = 0; i < 32; i++) off.v[i] = tw.off[i];
    uint32_t e2 = (30u * log_n) % 31u;
    uint32_t inv_n = e2 == 0 ? 1u : (1u << e2);
    for (uint32_t q = 0; q < np; q++) {
        uint32_t i = forward ? q : np - 1u - q;
        uint32_t s = ps[i], r = pr[i];
        uint32_t wlog = s < 3u ? s : 3u;
        uint32_t tsz = (1u << r) << wlog;
        uint32_t threads = tsz / 2 < 32u ? 32u : (tsz / 2 > 512u ? 512u : tsz / 2);
        uint64_t tiles = (1ull << log_n) / tsz;
        dim3 grid((unsigned)tiles, n_cols);
        const uint32_t *in = (q == 0 && src) ? src : nullptr;
        uint64_t mask = src ? ((1ull << src_log) - 1ull) : ~0ull;
        uint64_t src_stride = src ? (1ull << src_log) : 0ull;
        bool last_inv = !forward && q == np - 1u;
        if (forward)
            ntt_pass_kernel<true><<<grid, threads, tsz * 4, stream>>>(data, dev_cols, col_stride, in, mask, src_stride,
                                                                     tw.line, tw.circle, off, s, r, wlog, 1u);
        else
            ntt_pass_kernel<false><<<grid, threads, tsz * 4, stream>>>(data, dev_cols, col_stride, in, mask, src_stride,
                                                                      tw.line, tw.circle, off, s, r, wlog,
                                                                      last_inv ? inv_n : 1u);
        e = cudaGetLastError();
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
