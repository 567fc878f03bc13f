// Twiddle table construction (see vx_twiddles.cuh).
#include <mutex>
#include <vector>

#include "vx_common.cuh"
#include "vx_twiddles.cuh"

namespace vx {

namespace {

std::mutex g_gen_mu;
cpoint *g_gen_dev[64] = {nullptr};

__global__ void line_layer_kernel(GenTables g, uint32_t e0, uint32_t k, uint32_t l, uint32_t *out, uint64_t size) {
    uint64_t h = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= size) return;
    uint64_t e = ((uint64_t)e0 + (h << (l + 1u + 31u - k))) << l;
    out[h] = gpow(g, (uint32_t)(e & 0x7FFFFFFFull)).x;
}

__global__ void circle_layer_kernel(GenTables g, uint32_t e0, uint32_t k, uint32_t *out, uint64_t size) {
    uint64_t h = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= size) return;
    uint64_t e = (uint64_t)e0 + (h << (31u - k));
    out[h] = gpow(g, (uint32_t)(e & 0x7FFFFFFFull)).y;
}

__global__ void fold_sources_kernel(GenTables g, uint32_t e0, uint32_t k, int extract_y, uint32_t *out, uint64_t half) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= half) return;
    uint64_t idx = brev_bits((uint32_t)(i << 1), k);
    uint64_t e = (uint64_t)e0 + (idx << (31u - k));
    cpoint p = gpow(g, (uint32_t)(e & 0x7FFFFFFFull));
    out[i] = extract_y ? p.y : p.x;
}

__global__ void stwo_table_kernel(GenTables g, uint32_t log_n, uint32_t *out, uint64_t size) {
    uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= size) return;
    if (w == size - 1) { out[w] = 1u; return; }
    // level j = number of leading ones of w as a (log_n - 1)-bit number
    const uint32_t bits = log_n - 1;
    const uint32_t j = __clz(~((uint32_t)w << (32u - bits)));
    const uint64_t off = size - (size >> j);
    const uint32_t L = bits - j;                 // log size of the level's coset
    const uint64_t p = w - off;                  // < 2^(L-1)
    const uint64_t idx = L > 1 ? brev_bits((uint32_t)p, L - 1) : 0u;
    const uint32_t e0 = ecoset_half_odds_e0(L);
    const uint64_t e = (uint64_t)e0 + (idx << (31u - L));
    out[w] = gpow(g, (uint32_t)(e & 0x7FFFFFFFull)).x;
}

__global__ void stwo_fold_circle_kernel(GenTables g, uint32_t log, uint32_t *out, uint64_t half) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= half) return;
    const uint64_t idx = brev_bits((uint32_t)(i << 1), log);
    const uint64_t e = (uint64_t)ecoset_half_odds_e0(log - 1) + (idx << (31u - (log - 1)));
    out[i] = gpow(g, (uint32_t)(e & 0x7FFFFFFFull)).y;
}

// One thread per aligned chunk of 64, mirroring batch_inverse.cu:8-41
// exactly, including the zero-first-slot behaviour: prefix products that
// skip zeros, one inversion, then the backward pass.  A block of 64 threads
// stages its 64 chunks (4096 words) through shared memory, so global loads
// and stores are coalesced; chunk c's word i sits at 65 c + i, so the
// threads' per-chunk walks hit distinct banks.  The outputs overwrite the
// prefix slots (slot i is last read at step i + 1 of the backward pass).
// Every load of a block precedes its stores, and blocks own disjoint
// ranges, so it is safe in place.
constexpr uint32_t kBiChunk = 64, kBiThreads = 64, kBiWords = kBiChunk * kBiThreads;

__global__ void __launch_bounds__(kBiThreads) batch_inverse_kernel(const uint32_t *in, uint32_t *out, uint64_t n) {
    __shared__ uint32_t xv[kBiWords + kBiThreads], pre[kBiWords + kBiThreads];
    const uint32_t t = threadIdx.x;
    const uint64_t base = (uint64_t)blockIdx.x * kBiWords;
    for (uint32_t e = t; e < kBiWords; e += kBiThreads) {
        const uint64_t g = base + e;
        xv[e + e / kBiChunk] = g < n ? in[g] : 0u;
    }
    __syncthreads();
    const uint64_t s = base + (uint64_t)t * kBiChunk;
    if (s < n) {
        const uint32_t cnt = (uint32_t)((n - s) < kBiChunk ? (n - s) : kBiChunk);
        uint32_t *x = xv + t * (kBiChunk + 1), *pr = pre + t * (kBiChunk + 1);
        uint32_t acc = x[0];
        pr[0] = acc;
        for (uint32_t i = 1; i < cnt; i++) {
            const uint32_t v = x[i];
            acc = v ? mmul(acc, v) : acc;
            pr[i] = acc;
        }
        const uint32_t first = x[0];
        uint32_t inv = minv(acc);
        for (uint32_t i = cnt - 1; i > 0; i--) {
            const uint32_t v = x[i];
            if (!v) { pr[i] = 0u; continue; }
            pr[i] = mmul(inv, pr[i - 1]);
            inv = mmul(inv, v);
        }
        pr[0] = first ? inv : 0u;
    }
    __syncthreads();
    for (uint32_t e = t; e < kBiWords; e += kBiThreads) {
        const uint64_t g = base + e;
        if (g < n) out[g] = pre[e + e / kBiChunk];
    }
}

}  // namespace

cudaError_t gen_tables_get(GenTables *out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_gen_mu);
    if (!g_gen_dev[dev]) {
        std::vector<hpoint> h((1u << 16) + (1u << 15));
        hpoint p{1u, 0u};
        for (uint32_t i = 0; i < (1u << 16); i++) { h[i] = p; p = h_pmul(p, kGen); }
        hpoint g16 = h_ppow(kGen, 1ull << 16);
        p = {1u, 0u};
        for (uint32_t i = 0; i < (1u << 15); i++) { h[(1u << 16) + i] = p; p = h_pmul(p, g16); }
        cpoint *d = nullptr;
        e = cudaMalloc(&d, h.size() * sizeof(cpoint));
        if (e != cudaSuccess) return e;
        e = cudaMemcpy(d, h.data(), h.size() * sizeof(cpoint), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) { cudaFree(d); return e; }
        g_gen_dev[dev] = d;
    }
    out->lo = g_gen_dev[dev];
    out->hi = g_gen_dev[dev] + (1u << 16);
    return cudaSuccess;
}

cudaError_t batch_inverse(const uint32_t *in, uint32_t *out, uint64_t n, cudaStream_t stream) {
    if (!n) return cudaSuccess;
    batch_inverse_kernel<<<(unsigned)((n + kBiWords - 1) / kBiWords), kBiThreads, 0, stream>>>(in, out, n);
    return cudaGetLastError();
}

cudaError_t build_ntt_tables(ecoset c, bool inverse, uint32_t *line, uint32_t *circle, cudaStream_t stream) {
    GenTables g;
    cudaError_t e = gen_tables_get(&g);
    if (e != cudaSuccess) return e;
    uint64_t m = 1ull << c.k;
    uint64_t off = 0;
    for (uint32_t l = 0; l + 1 < c.k; l++) {
        uint64_t size = m >> (l + 1);
        line_layer_kernel<<<blocks_for(size, 256), 256, 0, stream>>>(g, c.e0, c.k, l, line + off, size);
        off += size;
    }
    if (m / 2) circle_layer_kernel<<<blocks_for(m / 2, 256), 256, 0, stream>>>(g, c.e0, c.k, circle, m / 2);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (inverse) {
        if (off) { e = batch_inverse(line, line, off, stream); if (e != cudaSuccess) return e; }
        if (m / 2) { e = batch_inverse(circle, circle, m / 2, stream); if (e != cudaSuccess) return e; }
    }
    return cudaSuccess;
}

cudaError_t build_fold_twiddles(ecoset c, bool extract_y, uint32_t *out, cudaStream_t stream) {
    GenTables g;
    cudaError_t e = gen_tables_get(&g);
    if (e != cudaSuccess) return e;
    uint64_t half = (1ull << c.k) / 2;
    if (!half) return cudaSuccess;
    fold_sources_kernel<<<blocks_for(half, 256), 256, 0, stream>>>(g, c.e0, c.k, extract_y ? 1 : 0, out, half);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return batch_inverse(out, out, half, stream);
}

cudaError_t build_ntt_tables_with(const GenTables &g, ecoset c, bool inverse, uint32_t *line, uint32_t *circle,
                                  cudaStream_t stream) {
    uint64_t m = 1ull << c.k;
    uint64_t off = 0;
    for (uint32_t l = 0; l + 1 < c.k; l++) {
        uint64_t size = m >> (l + 1);
        line_layer_kernel<<<blocks_for(size, 256), 256, 0, stream>>>(g, c.e0, c.k, l, line + off, size);
        off += size;
    }
    if (m / 2) circle_layer_kernel<<<blocks_for(m / 2, 256), 256, 0, stream>>>(g, c.e0, c.k, circle, m / 2);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (inverse) {
        if (off) { e = batch_inverse(line, line, off, stream); if (e != cudaSuccess) return e; }
        if (m / 2) { e = batch_inverse(circle, circle, m / 2, stream); if (e != cudaSuccess) return e; }
    }
    return cudaSuccess;
}

cudaError_t build_fold_twiddles_with(const GenTables &g, ecoset c, bool extract_y, uint32_t *out,
                                     cudaStream_t stream) {
    uint64_t half = (1ull << c.k) / 2;
    if (!half) return cudaSuccess;
    fold_sources_kernel<<<blocks_for(half, 256), 256, 0, stream>>>(g, c.e0, c.k, extract_y ? 1 : 0, out, half);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return batch_inverse(out, out, half, stream);
}

void gen_tables_host(uint32_t *w) {
    hpoint p{1u, 0u};
    for (uint32_t i = 0; i < (1u << 16); i++) { w[2 * i] = p.x; w[2 * i + 1] = p.y; p = h_pmul(p, kGen); }
    hpoint g16 = h_ppow(kGen, 1ull << 16);
    p = {1u, 0u};
    uint32_t *hi = w + 2 * (1u << 16);
    for (uint32_t i = 0; i < (1u << 15); i++) { hi[2 * i] = p.x; hi[2 * i + 1] = p.y; p = h_pmul(p, g16); }
}

cudaError_t build_stwo_table_with(const GenTables &g, uint32_t log_n, bool inverse, uint32_t *out,
                                  cudaStream_t stream) {
    if (log_n < 2 || log_n > 29) return cudaErrorInvalidValue;
    const uint64_t size = 1ull << (log_n - 1);
    stwo_table_kernel<<<blocks_for(size, 256), 256, 0, stream>>>(g, log_n, out, size);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess && inverse) e = batch_inverse(out, out, size, stream);
    return e;
}

cudaError_t build_stwo_fold_circle_with(const GenTables &g, uint32_t log, uint32_t *out, cudaStream_t stream) {
    if (log < 2 || log > 30) return cudaErrorInvalidValue;
    const uint64_t half = 1ull << (log - 1);
    stwo_fold_circle_kernel<<<blocks_for(half, 256), 256, 0, stream>>>(g, log, out, half);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = batch_inverse(out, out, half, stream);
    return e;
}

}  // namespace vx
