// Proof-of-work nonce search for the Blake2s channel (grind.cu,
// grind_m31_output.cu; host loop of crates/cuda-backend/src/grind_ops.rs).
//
// A nonce is accepted when Blake2s(prefixed_digest || nonce_le) (40 bytes,
// one compression) has at least pow_bits trailing zeros in its first 16
// bytes read as a little-endian u128 (channel.rs:140-168); the M31-output
// variant reduces those four words mod P first.  prefixed_digest =
// Blake2s(0x12345678_le || 0^12 || channel state || pow_bits_le) is the
// caller's, as in the reference.
//
// The full search visits nonces (hi << 32) | low, low < 2^20, hi = 0, 1, ...
// and returns the smallest accepted one, the order stwo's SimdBackend and the
// reference's loop use.  Warps take chunks of candidates in increasing order
// from a counter and stop at a chunk that starts beyond the best nonce found
// so far; no chunk is left half done, so the result is exactly the minimum
// of the range whatever the scheduling.  (A fixed grid-stride split wastes
// work here: the warp scheduler lets some warps run far ahead of the one
// that holds the answer.)  Launches are bounded (a fixed range each); the
// host checks the result between launches.  The reference-ABI launchers,
// which have no counter word, keep a stateless grid-stride loop.
#include <mutex>

#include "vx_blake2s.cuh"
#include "vx_common.cuh"
#include "vx_field.cuh"

namespace vx {
namespace {

struct Digest8 { uint32_t w[8]; };

// Trailing zeros of the u128 (h0 | h1 << 32 | h2 << 64 | h3 << 96).
__device__ __forceinline__ uint32_t tz128(uint32_t h0, uint32_t h1, uint32_t h2, uint32_t h3) {
    if (h0) return __ffs((int)h0) - 1u;
    if (h1) return 32u + __ffs((int)h1) - 1u;
    if (h2) return 64u + __ffs((int)h2) - 1u;
    if (h3) return 96u + __ffs((int)h3) - 1u;
    return 128u;
}

__device__ __forceinline__ uint32_t mod_p(uint32_t h) {
    const uint32_t r = (h & VX_P) + (h >> 31);
    return umin32(r, r - VX_P);
}

// Candidate w of a launch is nonce base + ((w >> lowbits) << 32) + (w & lowmask)
// (lowbits >= 63: base + w).  count candidates.  With `next` (a zeroed
// counter) warps take kWarpChunk consecutive candidates at a time; without
// it each thread walks w = its index + j * (grid threads), j = 0, 1, ...
// Both visit a thread's candidates in increasing order.  The digest comes by
// value, or from device memory when dptr is not null.
constexpr uint32_t kPerLane = 4, kWarpChunk = 32 * kPerLane;

template <bool M31OUT>
__device__ __forceinline__ void grind_one(const Digest8 &d, unsigned long long *result, uint32_t pow_bits,
                                          uint64_t nonce, uint32_t one) {
    uint32_t m[16];
#pragma unroll
    for (int i = 0; i < 8; i++) m[i] = d.w[i];
    m[8] = (uint32_t)nonce;
    m[9] = (uint32_t)(nonce >> 32);
#pragma unroll
    for (int i = 10; i < 16; i++) m[i] = 0u;
    uint32_t h[8];
    blake2s_block(h, m, 40u, one);  // one == 1: Blake2s pipe balance
    uint32_t h0 = h[0], h1 = h[1], h2 = h[2], h3 = h[3];
    if (M31OUT) { h0 = mod_p(h0); h1 = mod_p(h1); h2 = mod_p(h2); h3 = mod_p(h3); }
    if (tz128(h0, h1, h2, h3) >= pow_bits) atomicMin(result, (unsigned long long)nonce);
}

template <bool M31OUT>
__global__ void __launch_bounds__(256) grind_kernel(Digest8 d, const uint32_t *dptr, unsigned long long *result,
                                                    unsigned long long *next, uint32_t pow_bits, uint64_t base,
                                                    uint64_t count, uint32_t lowbits, uint32_t one) {
    if (dptr) {
#pragma unroll
        for (int i = 0; i < 8; i++) d.w[i] = __ldg(dptr + i);
    }
    const uint64_t lowmask = lowbits >= 63 ? ~0ull : ((1ull << lowbits) - 1ull);
    auto nonce_of = [&](uint64_t w) { return lowbits >= 63 ? base + w : base + ((w >> lowbits) << 32) + (w & lowmask); };
    if (next) {
        const uint32_t lane = threadIdx.x & 31u;
        while (true) {
            // lane 0 takes the chunk and reads the best nonce; both are
            // broadcast, so the whole warp leaves the loop together
            unsigned long long c0 = 0, best = 0;
            if (lane == 0) {
                c0 = atomicAdd(next, (unsigned long long)kWarpChunk);
                best = __ldcv(result);
            }
            c0 = __shfl_sync(0xFFFFFFFFu, c0, 0);
            best = __shfl_sync(0xFFFFFFFFu, best, 0);
            if (c0 >= count || nonce_of(c0) > best) return;
#pragma unroll 1
            for (uint32_t r = 0; r < kPerLane; r++) {
                const uint64_t w = c0 + 32u * r + lane;
                if (w < count) grind_one<M31OUT>(d, result, pow_bits, nonce_of(w), one);
            }
        }
    }
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < count; w += stride) {
        const uint64_t nonce = nonce_of(w);
        if (nonce > __ldcv(result)) return;  // a smaller nonce is already accepted
        grind_one<M31OUT>(d, result, pow_bits, nonce, one);
    }
}

// Blocks of 256 threads: every resident block with the chunk counter; two
// per SM for the grid-stride loop, which measured fastest there when the
// answer comes early (the fewer warps per SM, the less they drift apart).
unsigned grind_blocks(bool m31, bool dynamic) {
    static int cached[64][2];
    int dev = 0;
    cudaGetDevice(&dev);
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) {
        cudaGetLastError();
        sms = 148;
    }
    if (!dynamic) return (unsigned)sms * 2u;
    int *c = (dev >= 0 && dev < 64) ? &cached[dev][m31 ? 1 : 0] : nullptr;
    if (c && *c) return (unsigned)*c;
    int per_sm = 0;
    cudaError_t e = m31 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, grind_kernel<true>, 256, 0)
                        : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, grind_kernel<false>, 256, 0);
    if (e != cudaSuccess || per_sm <= 0) {
        cudaGetLastError();
        per_sm = 4;
    }
    if (c) *c = sms * per_sm;
    return (unsigned)(sms * per_sm);
}

// digest_words: 8 host words, or nullptr with dptr the device digest.
// next: a zeroed chunk counter (dynamic chunks), or null (grid-stride loop).
cudaError_t grind_launch(bool m31, const uint32_t *digest_words, const uint32_t *dptr, unsigned long long *result,
                         unsigned long long *next, uint32_t pow_bits, uint64_t base, uint64_t count, uint32_t lowbits,
                         cudaStream_t st) {
    Digest8 d{};
    if (digest_words)
        for (int i = 0; i < 8; i++) d.w[i] = digest_words[i];
    uint64_t need = (count + 255) / 256;
    unsigned blocks = grind_blocks(m31, next != nullptr);
    if (need < blocks) blocks = (unsigned)(need ? need : 1);
    if (m31)
        grind_kernel<true><<<blocks, 256, 0, st>>>(d, dptr, result, next, pow_bits, base, count, lowbits, 1u);
    else
        grind_kernel<false><<<blocks, 256, 0, st>>>(d, dptr, result, next, pow_bits, base, count, lowbits, 1u);
    return cudaGetLastError();
}

// One device result word per device for vx_grind_pow.
std::mutex g_grind_mu;
unsigned long long *g_grind_res[64] = {nullptr};

}  // namespace
}  // namespace vx

using namespace vx;

extern "C" {

// grind.cu:26-118 (cuda_grind_pow): candidates batch_offset + i, i < n_threads,
// asynchronous on the legacy stream; the caller sets *result to UINT64_MAX.
static void grind_abi(bool m31, const uint32_t *prefixed_digest, uint64_t *result, uint32_t pow_bits,
                      uint64_t batch_offset, uint32_t n_threads, const char *who) {
    if (n_threads == 0) return;
    cudaError_t e = grind_launch(m31, nullptr, prefixed_digest, (unsigned long long *)result, nullptr, pow_bits,
                                 batch_offset, n_threads, 63u, 0);
    if (e != cudaSuccess) set_last_error(VX_ERR_CUDA, "%s: %s", who, cudaGetErrorString(e));
}

void cuda_grind_pow(const uint32_t *prefixed_digest, uint64_t *result, uint32_t pow_bits, uint64_t batch_offset,
                    uint32_t n_threads) {
    grind_abi(false, prefixed_digest, result, pow_bits, batch_offset, n_threads, "cuda_grind_pow");
}

void cuda_grind_pow_m31_output(const uint32_t *prefixed_digest, uint64_t *result, uint32_t pow_bits,
                               uint64_t batch_offset, uint32_t n_threads) {
    grind_abi(true, prefixed_digest, result, pow_bits, batch_offset, n_threads, "cuda_grind_pow_m31_output");
}

}  // extern "C"

// Full search: nonces (hi << 32) | low, low < 2^20, hi = 0 .. max_batches - 1,
// in launches of up to 64 values of hi (2^26 candidates) with the result read
// back between them.
extern "C" int vx_grind_pow(const uint32_t prefixed_digest[8], uint32_t pow_bits, int m31_output,
                            uint32_t max_batches, uint64_t *nonce_out, void *stream) {
    VX_CHECK_ARG(prefixed_digest != nullptr && nonce_out != nullptr, "vx_grind_pow: null argument");
    VX_CHECK_ARG(pow_bits <= 128, "vx_grind_pow: pow_bits %u above 128", pow_bits);
    VX_CHECK_ARG(max_batches >= 1 && max_batches < (1u << 31) - 1, "vx_grind_pow: max_batches must be in [1, 2^31 - 2]");
    if (pow_bits == 0) {  // grind_ops.rs: no work below one bit
        *nonce_out = 0;
        return VX_OK;
    }
    int dev = 0;
    VX_CUDA_TRY(cudaGetDevice(&dev));
    VX_CHECK_ARG(dev >= 0 && dev < 64, "vx_grind_pow: device %d out of range", dev);
    std::lock_guard<std::mutex> lk(g_grind_mu);
    if (!g_grind_res[dev]) VX_CUDA_TRY(cudaMalloc(&g_grind_res[dev], 2 * sizeof(unsigned long long)));
    unsigned long long *res = g_grind_res[dev];  // [0] best nonce, [1] chunk counter
    cudaStream_t st = (cudaStream_t)stream;
    constexpr uint32_t kLowBits = 20, kHiPerLaunch = 64;
    for (uint32_t hi = 0; hi < max_batches; hi += kHiPerLaunch) {
        const uint32_t nh = max_batches - hi < kHiPerLaunch ? max_batches - hi : kHiPerLaunch;
        VX_CUDA_TRY(cudaMemsetAsync(res, 0xFF, sizeof(unsigned long long), st));
        VX_CUDA_TRY(cudaMemsetAsync(res + 1, 0, sizeof(unsigned long long), st));
        VX_CUDA_TRY(grind_launch(m31_output != 0, prefixed_digest, nullptr, res, res + 1, pow_bits,
                                 (uint64_t)hi << 32, (uint64_t)nh << kLowBits, kLowBits, st));
        unsigned long long found = ~0ull;
        VX_CUDA_TRY(cudaMemcpyAsync(&found, res, sizeof(found), cudaMemcpyDeviceToHost, st));
        VX_CUDA_TRY(cudaStreamSynchronize(st));
        if (found != ~0ull) {
            *nonce_out = found;
            return VX_OK;
        }
    }
    set_last_error(VX_ERR_DEVICE, "vx_grind_pow: no nonce with %u trailing zero bits in %u batches of 2^20", pow_bits,
                   max_batches);
    return VX_ERR_DEVICE;
}
