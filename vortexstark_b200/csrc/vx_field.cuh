// M31 / CM31 / QM31 arithmetic for sm_100a.
//
// Exact 32-bit integer arithmetic over P = 2^31 - 1, canonical values in
// [0, P).  Semantics match src/field/m31.rs:24-35 (reduce = lo + hi, one
// conditional subtract), cm31.rs and qm31.rs:110-155 (u^2 = 2 + i).  The
// conditional subtracts use the unsigned-min form min(r, r - P), which
// compiles to IADD3 + VIMNMX without a branch.
#pragma once
#include <cstdint>

#define VX_P 0x7FFFFFFFu

namespace vx {

__device__ __forceinline__ uint32_t umin32(uint32_t a, uint32_t b) { return a < b ? a : b; }

__device__ __forceinline__ uint32_t madd(uint32_t a, uint32_t b) {
    uint32_t r = a + b;
    return umin32(r, r - VX_P);
}
__device__ __forceinline__ uint32_t msub(uint32_t a, uint32_t b) {
    uint32_t r = a - b + VX_P;
    return umin32(r, r - VX_P);
}
__device__ __forceinline__ uint32_t mmul(uint32_t a, uint32_t b) {
    uint64_t p = (uint64_t)a * b;
    uint32_t r = ((uint32_t)p & VX_P) + (uint32_t)(p >> 31);
    return umin32(r, r - VX_P);
}
__device__ __forceinline__ uint32_t mneg(uint32_t a) { return a ? VX_P - a : 0u; }
__device__ __forceinline__ uint32_t mdbl(uint32_t a) { return madd(a, a); }
__device__ __forceinline__ uint32_t mpow(uint32_t a, uint32_t e) {
    uint32_t r = 1u;
    while (e) {
        if (e & 1u) r = mmul(r, a);
        a = mmul(a, a);
        e >>= 1;
    }
    return r;
}
// Fermat inverse; maps 0 to 0 like the reference's m31_inv.
__device__ __forceinline__ uint32_t minv(uint32_t a) { return mpow(a, VX_P - 2u); }

struct cm31 { uint32_t a, b; };
__device__ __forceinline__ cm31 cadd(cm31 x, cm31 y) { return {madd(x.a, y.a), madd(x.b, y.b)}; }
__device__ __forceinline__ cm31 csub(cm31 x, cm31 y) { return {msub(x.a, y.a), msub(x.b, y.b)}; }
__device__ __forceinline__ cm31 cmul(cm31 x, cm31 y) {
    return {msub(mmul(x.a, y.a), mmul(x.b, y.b)), madd(mmul(x.a, y.b), mmul(x.b, y.a))};
}

struct qm31 { uint32_t v[4]; };
__device__ __forceinline__ qm31 qadd(qm31 x, qm31 y) {
    return {{madd(x.v[0], y.v[0]), madd(x.v[1], y.v[1]), madd(x.v[2], y.v[2]), madd(x.v[3], y.v[3])}};
}
__device__ __forceinline__ qm31 qsub(qm31 x, qm31 y) {
    return {{msub(x.v[0], y.v[0]), msub(x.v[1], y.v[1]), msub(x.v[2], y.v[2]), msub(x.v[3], y.v[3])}};
}
__device__ __forceinline__ qm31 qmulm(qm31 x, uint32_t s) {
    return {{mmul(x.v[0], s), mmul(x.v[1], s), mmul(x.v[2], s), mmul(x.v[3], s)}};
}
// (a + b u)(c + d u) = (ac + bd (2 + i)) + (ad + bc) u
__device__ __forceinline__ qm31 qmul(qm31 x, qm31 y) {
    cm31 xa{x.v[0], x.v[1]}, xb{x.v[2], x.v[3]}, ya{y.v[0], y.v[1]}, yb{y.v[2], y.v[3]};
    cm31 ac = cmul(xa, ya), bd = cmul(xb, yb), ad = cmul(xa, yb), bc = cmul(xb, ya);
    cm31 bdu{msub(mdbl(bd.a), bd.b), madd(bd.a, mdbl(bd.b))};
    cm31 ra = cadd(ac, bdu), rb = cadd(ad, bc);
    return {{ra.a, ra.b, rb.a, rb.b}};
}

// Multiplication by a fixed QM31 a = A + B u (A = a0 + a1 i, B = a2 + a3 i):
// a z = (A Z1 + B (2 + i) Z2) + (B Z1 + A Z2) u is a 4 x 4 matrix over M31
// built from nine values.  Each output word is a dot product of four
// products of canonical words, (P - 1)^2 * 4 < 2^64, so it accumulates in
// 64 bits (four wide multiply-adds) and is reduced once: about 14
// instructions per word instead of four reduced products and three reduced
// additions.  Same values as qmul(a, z).
struct qmat { uint32_t a0, a1, na1, a2, a3, na3, c0, c1, nc1; };
__device__ __forceinline__ qmat qmat_of(qm31 a) {
    const uint32_t c0 = msub(mdbl(a.v[2]), a.v[3]), c1 = madd(a.v[2], mdbl(a.v[3]));  // B (2 + i)
    return {a.v[0], a.v[1], mneg(a.v[1]), a.v[2], a.v[3], mneg(a.v[3]), c0, c1, mneg(c1)};
}
// s mod P for any 64-bit s.
__device__ __forceinline__ uint32_t reduce64(uint64_t s) {
    const uint64_t t = (s & (uint64_t)VX_P) + (s >> 31);                    // < 2^34
    const uint32_t r = (uint32_t)(t & (uint64_t)VX_P) + (uint32_t)(t >> 31);  // < 2^31 + 8
    return umin32(r, r - VX_P);
}
__device__ __forceinline__ uint32_t dot4(uint32_t m0, uint32_t z0, uint32_t m1, uint32_t z1, uint32_t m2, uint32_t z2,
                                         uint32_t m3, uint32_t z3) {
    return reduce64((uint64_t)m0 * z0 + (uint64_t)m1 * z1 + (uint64_t)m2 * z2 + (uint64_t)m3 * z3);
}
__device__ __forceinline__ qm31 qmul_mat(const qmat &m, qm31 z) {
    const uint32_t z0 = z.v[0], z1 = z.v[1], z2 = z.v[2], z3 = z.v[3];
    return {{dot4(m.a0, z0, m.na1, z1, m.c0, z2, m.nc1, z3), dot4(m.a1, z0, m.a0, z1, m.c1, z2, m.c0, z3),
             dot4(m.a2, z0, m.na3, z1, m.a0, z2, m.na1, z3), dot4(m.a3, z0, m.a2, z1, m.a1, z2, m.a0, z3)}};
}

// Product with a doubled twiddle t2 = 2 t (t canonical, so t2 <= 2P - 2 <
// 2^32): p = a t2 < 2^63 for canonical a, a t = p / 2 = hi 2^31 + lo / 2,
// and 2^31 = 1 (mod P), so a t = hi + lo / 2 (mod P) with hi <= 2^31 - 2 and
// lo / 2 <= 2^31 - 1: one conditional subtract makes it canonical.
__device__ __forceinline__ uint32_t mmul_t2(uint32_t a, uint32_t t2) {
    const uint64_t p = (uint64_t)a * t2;
    const uint32_t r = (uint32_t)(p >> 32) + ((uint32_t)p >> 1);
    return umin32(r, r - VX_P);
}

// Circle group point (x, y) with x^2 + y^2 = 1; group law of src/circle.rs:33-39.
struct cpoint { uint32_t x, y; };
__device__ __forceinline__ cpoint pmul(cpoint a, cpoint b) {
    return {msub(mmul(a.x, b.x), mmul(a.y, b.y)), madd(mmul(a.x, b.y), mmul(a.y, b.x))};
}
__device__ __forceinline__ cpoint ppow(cpoint a, uint64_t k) {
    cpoint r{1u, 0u};
    while (k) {
        if (k & 1) r = pmul(r, a);
        a = pmul(a, a);
        k >>= 1;
    }
    return r;
}

__device__ __forceinline__ uint32_t brev_bits(uint32_t i, uint32_t bits) {
    return bits ? (__brev(i) >> (32 - bits)) : 0u;
}

}  // namespace vx
