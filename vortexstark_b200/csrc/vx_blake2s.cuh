// Blake2s-256 compression (RFC 7693) for sm_100a, register resident.
//
// The 16 message words and the 16-word working state live in registers; the
// message schedule is resolved at compile time by full unrolling, so no
// message word is ever indexed at run time.  Rotations by 16 and 8 are byte
// permutes (PRMT), by 12 and 7 funnel shifts (SHF).
//
// Pipe balance: the xors and rotations (8 per G) run on the integer ALU
// pipe, which bounds the compression rate.  a + b + m is written as
// a + (b * one + m) with `one` a runtime 1 (a kernel parameter, which ptxas
// cannot fold), so b * one + m can issue as an IMAD on the FMA pipe.
// Measured on B200 with 16-word messages (tree nodes, wide leaves): 27.5 G
// compressions/s against 22.7 G with the plain three-input add; leaves with
// mostly zero words gain ~3%.  The column step (VX_G) also writes c + d as
// d * one + c; the diagonal step (VX_GD) keeps the plain add: 2^26-leaf trees
// 4.93 -> 4.87 ms (moving every c + d instead overloads the FMA pipe: 21.7 G/s).
// Callers that pass no `one` get the literal 1, which folds back to the plain
// add.
//
// Leaves, nodes and the transcript all use the unkeyed, unpersonalised
// parameter block (h0 ^= 0x01010020), as the reference does
// (blake2s.cuh:70-136, blake2s.cu:47-60, channel.rs:256-262).
#pragma once
#include <cstdint>

namespace vx {

#define VX_IV0 0x6A09E667u
#define VX_IV1 0xBB67AE85u
#define VX_IV2 0x3C6EF372u
#define VX_IV3 0xA54FF53Au
#define VX_IV4 0x510E527Fu
#define VX_IV5 0x9B05688Cu
#define VX_IV6 0x1F83D9ABu
#define VX_IV7 0x5BE0CD19u

__device__ __forceinline__ uint32_t ror16(uint32_t x) { return __byte_perm(x, 0, 0x1032); }
__device__ __forceinline__ uint32_t ror8(uint32_t x) { return __byte_perm(x, 0, 0x0321); }
__device__ __forceinline__ uint32_t ror12(uint32_t x) { return __funnelshift_r(x, x, 12); }
__device__ __forceinline__ uint32_t ror7(uint32_t x) { return __funnelshift_r(x, x, 7); }

#define VX_G(a, b, c, d, x, y)      \
    do {                            \
        a = a + (b * one + (x));    \
        d = ror16(d ^ a);           \
        c = d * one + c;            \
        b = ror12(b ^ c);           \
        a = a + (b * one + (y));    \
        d = ror8(d ^ a);            \
        c = d * one + c;            \
        b = ror7(b ^ c);            \
    } while (0)

#define VX_GD(a, b, c, d, x, y)     \
    do {                            \
        a = a + (b * one + (x));    \
        d = ror16(d ^ a);           \
        c = c + d;                  \
        b = ror12(b ^ c);           \
        a = a + (b * one + (y));    \
        d = ror8(d ^ a);            \
        c = c + d;                  \
        b = ror7(b ^ c);            \
    } while (0)

#define VX_ROUND(s0, s1, s2, s3, s4, s5, s6, s7, s8, s9, s10, s11, s12, s13, s14, s15) \
    do {                                                                                 \
        VX_G(v0, v4, v8, v12, m[s0], m[s1]);                                             \
        VX_G(v1, v5, v9, v13, m[s2], m[s3]);                                             \
        VX_G(v2, v6, v10, v14, m[s4], m[s5]);                                            \
        VX_G(v3, v7, v11, v15, m[s6], m[s7]);                                            \
        VX_GD(v0, v5, v10, v15, m[s8], m[s9]);                                           \
        VX_GD(v1, v6, v11, v12, m[s10], m[s11]);                                         \
        VX_GD(v2, v7, v8, v13, m[s12], m[s13]);                                          \
        VX_GD(v3, v4, v9, v14, m[s14], m[s15]);                                          \
    } while (0)

// h[8] <- compress(h, m, t, last).  m is indexed only by literals.
__device__ __forceinline__ void blake2s_compress(uint32_t h[8], const uint32_t m[16], uint32_t t, bool last,
                                                 uint32_t one = 1u) {
    uint32_t v0 = h[0], v1 = h[1], v2 = h[2], v3 = h[3], v4 = h[4], v5 = h[5], v6 = h[6], v7 = h[7];
    uint32_t v8 = VX_IV0, v9 = VX_IV1, v10 = VX_IV2, v11 = VX_IV3;
    uint32_t v12 = VX_IV4 ^ t, v13 = VX_IV5, v14 = last ? ~VX_IV6 : VX_IV6, v15 = VX_IV7;
    VX_ROUND(0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15);
    VX_ROUND(14, 10, 4, 8, 9, 15, 13, 6, 1, 12, 0, 2, 11, 7, 5, 3);
    VX_ROUND(11, 8, 12, 0, 5, 2, 15, 13, 10, 14, 3, 6, 7, 1, 9, 4);
    VX_ROUND(7, 9, 3, 1, 13, 12, 11, 14, 2, 6, 5, 10, 4, 0, 15, 8);
    VX_ROUND(9, 0, 5, 7, 2, 4, 10, 15, 14, 1, 11, 12, 6, 8, 3, 13);
    VX_ROUND(2, 12, 6, 10, 0, 11, 8, 3, 4, 13, 7, 5, 15, 14, 1, 9);
    VX_ROUND(12, 5, 1, 15, 14, 13, 4, 10, 0, 7, 6, 3, 9, 2, 8, 11);
    VX_ROUND(13, 11, 7, 14, 12, 1, 3, 9, 5, 0, 15, 4, 8, 6, 2, 10);
    VX_ROUND(6, 15, 14, 9, 11, 3, 0, 8, 12, 2, 13, 7, 1, 4, 10, 5);
    VX_ROUND(10, 2, 8, 4, 7, 6, 1, 5, 15, 11, 9, 14, 3, 12, 13, 0);
    h[0] ^= v0 ^ v8;  h[1] ^= v1 ^ v9;  h[2] ^= v2 ^ v10; h[3] ^= v3 ^ v11;
    h[4] ^= v4 ^ v12; h[5] ^= v5 ^ v13; h[6] ^= v6 ^ v14; h[7] ^= v7 ^ v15;
}

__device__ __forceinline__ void blake2s_init(uint32_t h[8]) {
    h[0] = VX_IV0 ^ 0x01010020u; h[1] = VX_IV1; h[2] = VX_IV2; h[3] = VX_IV3;
    h[4] = VX_IV4; h[5] = VX_IV5; h[6] = VX_IV6; h[7] = VX_IV7;
}

// One-block hash of `nbytes` (<= 64) already laid out as 16 LE words.
__device__ __forceinline__ void blake2s_block(uint32_t out[8], const uint32_t m[16], uint32_t nbytes,
                                              uint32_t one = 1u) {
    blake2s_init(out);
    blake2s_compress(out, m, nbytes, true, one);
}

// Parent of two 8-word children (t = 64, final).
__device__ __forceinline__ void blake2s_node(uint32_t out[8], const uint32_t l[8], const uint32_t r[8],
                                             uint32_t one = 1u) {
    uint32_t m[16];
#pragma unroll
    for (int i = 0; i < 8; i++) { m[i] = l[i]; m[8 + i] = r[i]; }
    blake2s_block(out, m, 64u, one);
}

// General (multi-block) hash of a byte string held in global/shared memory
// as little-endian words; len in bytes.  Used by the transcript (mix_felts)
// and the lifted leaves.
__device__ inline void blake2s_words(uint32_t out[8], const uint32_t *w, uint32_t len) {
    blake2s_init(out);
    uint32_t off = 0;
    while (len - off > 64u) {
        uint32_t m[16];
#pragma unroll
        for (int i = 0; i < 16; i++) m[i] = w[off / 4 + i];
        off += 64u;
        blake2s_compress(out, m, off, false);
    }
    uint32_t m[16];
    uint32_t rem = len - off;  // 0..64 bytes, whole words on this path
#pragma unroll
    for (int i = 0; i < 16; i++) m[i] = (4u * i < rem) ? w[off / 4 + i] : 0u;
    blake2s_compress(out, m, len, true);
}

}  // namespace vx
