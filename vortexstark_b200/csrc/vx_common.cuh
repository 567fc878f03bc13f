// Shared host/device helpers for the vortex_b200 library.
#pragma once
#include <cstdint>
#include <cstdio>
#include <cuda_runtime.h>

#include "../../include/vortex_b200.h"

namespace vx {

// Status of the last failing call on this host thread (vx_last_error()).
void set_last_error(int code, const char *fmt, ...);

#define VX_CUDA_TRY(expr)                                                              \
    do {                                                                               \
        cudaError_t _e = (expr);                                                       \
        if (_e != cudaSuccess) {                                                       \
            ::vx::set_last_error(VX_ERR_CUDA, "%s:%d %s: %s", __FILE__, __LINE__, #expr, \
                                 cudaGetErrorString(_e));                              \
            return VX_ERR_CUDA;                                                        \
        }                                                                              \
    } while (0)

#define VX_CHECK_ARG(cond, ...)                                     \
    do {                                                            \
        if (!(cond)) {                                              \
            ::vx::set_last_error(VX_ERR_ARG, __VA_ARGS__);          \
            return VX_ERR_ARG;                                      \
        }                                                           \
    } while (0)

// Launches of the reference-compatible entry points return void, as the
// reference's do; a failed launch is recorded for vx_last_error().
#define VX_LAUNCH_CHECK()                                                                   \
    do {                                                                                    \
        cudaError_t _e = cudaGetLastError();                                                \
        if (_e != cudaSuccess)                                                              \
            ::vx::set_last_error(VX_ERR_CUDA, "%s:%d launch: %s", __FILE__, __LINE__,       \
                                 cudaGetErrorString(_e));                                   \
    } while (0)

// Programmatic dependent launch.  A kernel launched with launch_pdl may have
// its blocks scheduled while the previous kernel on the stream drains, so the
// launch latency between dependent kernels is hidden; it calls pdl_wait()
// before it touches memory that earlier work on the stream wrote.  pdl_wait()
// returns at once when the kernel was launched without the attribute.
__device__ __forceinline__ void pdl_wait() {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 900
    asm volatile("griddepcontrol.wait;" ::: "memory");
#endif
}
template <class... KArgs, class... Args>
inline cudaError_t launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                              Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, args...);
}

inline unsigned blocks_for(uint64_t n, unsigned threads) {
    return (unsigned)((n + threads - 1) / threads);
}

constexpr uint32_t kP = 0x7FFFFFFFu;

// Host-side M31 helpers (exact; used to precompute kernel constants).
inline uint32_t h_madd(uint32_t a, uint32_t b) { uint32_t r = a + b; return r >= kP ? r - kP : r; }
inline uint32_t h_msub(uint32_t a, uint32_t b) { return a >= b ? a - b : a + kP - b; }
inline uint32_t h_mmul(uint32_t a, uint32_t b) {
    uint64_t p = (uint64_t)a * b;
    uint32_t r = (uint32_t)(p & kP) + (uint32_t)(p >> 31);
    return r >= kP ? r - kP : r;
}
struct hpoint { uint32_t x, y; };
inline hpoint h_pmul(hpoint a, hpoint b) {
    return {h_msub(h_mmul(a.x, b.x), h_mmul(a.y, b.y)), h_madd(h_mmul(a.x, b.y), h_mmul(a.y, b.x))};
}
inline hpoint h_ppow(hpoint a, uint64_t k) {
    hpoint r{1u, 0u};
    while (k) { if (k & 1) r = h_pmul(r, a); a = h_pmul(a, a); k >>= 1; }
    return r;
}
inline hpoint h_rep_double(hpoint p, uint32_t n) { for (uint32_t i = 0; i < n; i++) p = h_pmul(p, p); return p; }
constexpr hpoint kGen{2u, 1268011823u};

// Cosets of src/circle.rs:101-143.
struct hcoset { hpoint initial, step; uint32_t log_size; };
inline hcoset coset_subgroup(uint32_t k) { return {{1u, 0u}, h_rep_double(kGen, 31 - k), k}; }
inline hcoset coset_half_coset(uint32_t k) { return {h_rep_double(kGen, 30 - k), h_rep_double(kGen, 31 - k), k}; }
inline hcoset coset_half_odds(uint32_t k) { return {h_rep_double(kGen, k >= 29 ? 0 : 29 - k), h_rep_double(kGen, 31 - k), k}; }
// Evaluation domain of a proof: half_coset(log) up to 30, subgroup(31) at 31
// (prover.rs:655-659, verifier.rs:161-165).
inline hcoset coset_eval_domain(uint32_t k) { return k <= 30 ? coset_half_coset(k) : coset_subgroup(k); }

}  // namespace vx
