/*
 * vx_oracle.c — CPU restatement of the VortexSTARK Fibonacci commitment
 * path.  TEST INFRASTRUCTURE ONLY (the oracle and the CPU baseline); the
 * product library never links or calls it.
 *
 * Each function follows the reference file:line cited in vx_oracle.h.
 * Parallel loops (OpenMP) only split independent elements, so outputs do
 * not depend on the thread count.
 */
#include "vx_oracle.h"
#include <stdlib.h>
#include <string.h>
#include <stdio.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define P VXO_P

/* ------------------------------------------------------------------ */
/* field: src/field/m31.rs:24-35, cm31.rs, qm31.rs:110-133            */
/* ------------------------------------------------------------------ */
static inline uint32_t m_red(uint64_t v) {
    uint32_t lo = (uint32_t)(v & P), hi = (uint32_t)(v >> 31), r = lo + hi;
    return r >= P ? r - P : r;
}
static inline uint32_t m_add(uint32_t a, uint32_t b) { uint32_t r = a + b; return r >= P ? r - P : r; }
static inline uint32_t m_sub(uint32_t a, uint32_t b) { return a >= b ? a - b : a + P - b; }
static inline uint32_t m_mul(uint32_t a, uint32_t b) { return m_red((uint64_t)a * b); }
static inline uint32_t m_neg(uint32_t a) { return a ? P - a : 0; }
static inline uint32_t m_dbl(uint32_t a) { uint32_t r = a << 1; return r >= P ? r - P : r; }
static uint32_t m_pow(uint32_t a, uint32_t e) {
    uint32_t r = 1, b = a;
    while (e) { if (e & 1) r = m_mul(r, b); b = m_mul(b, b); e >>= 1; }
    return r;
}
uint32_t vxo_m31_mul(uint32_t a, uint32_t b) { return m_mul(a, b); }
uint32_t vxo_m31_inv(uint32_t a) { return m_pow(a, P - 2); }

typedef struct { uint32_t a, b; } cm;
static inline cm cm_add(cm x, cm y) { return (cm){m_add(x.a, y.a), m_add(x.b, y.b)}; }
static inline cm cm_sub(cm x, cm y) { return (cm){m_sub(x.a, y.a), m_sub(x.b, y.b)}; }
static inline cm cm_mul(cm x, cm y) {
    return (cm){m_sub(m_mul(x.a, y.a), m_mul(x.b, y.b)), m_add(m_mul(x.a, y.b), m_mul(x.b, y.a))};
}
typedef struct { uint32_t v[4]; } qm;
static inline qm q_add(qm x, qm y) { qm r; for (int i = 0; i < 4; i++) r.v[i] = m_add(x.v[i], y.v[i]); return r; }
static inline qm q_sub(qm x, qm y) { qm r; for (int i = 0; i < 4; i++) r.v[i] = m_sub(x.v[i], y.v[i]); return r; }
static inline qm q_mulm(qm x, uint32_t s) { qm r; for (int i = 0; i < 4; i++) r.v[i] = m_mul(x.v[i], s); return r; }
/* (a + bu)(c + du) = (ac + bd(2+i)) + (ad + bc)u  — qm31.rs:138-155 */
static inline qm q_mul(qm x, qm y) {
    cm xa = {x.v[0], x.v[1]}, xb = {x.v[2], x.v[3]}, ya = {y.v[0], y.v[1]}, yb = {y.v[2], y.v[3]};
    cm ac = cm_mul(xa, ya), bd = cm_mul(xb, yb), ad = cm_mul(xa, yb), bc = cm_mul(xb, ya);
    cm bdu = {m_sub(m_dbl(bd.a), bd.b), m_add(bd.a, m_dbl(bd.b))};
    cm ra = cm_add(ac, bdu), rb = cm_add(ad, bc);
    qm r = {{ra.a, ra.b, rb.a, rb.b}};
    return r;
}
void vxo_qm31_mul(const uint32_t a[4], const uint32_t b[4], uint32_t out[4]) {
    qm x, y; memcpy(x.v, a, 16); memcpy(y.v, b, 16);
    qm r = q_mul(x, y); memcpy(out, r.v, 16);
}

/* ------------------------------------------------------------------ */
/* circle group: src/circle.rs:10-185                                 */
/* ------------------------------------------------------------------ */
static const vxo_point GEN = {2u, 1268011823u};
static const vxo_point IDENT = {1u, 0u};
vxo_point vxo_point_mul(vxo_point a, vxo_point b) {
    vxo_point r = {m_sub(m_mul(a.x, b.x), m_mul(a.y, b.y)), m_add(m_mul(a.x, b.y), m_mul(a.y, b.x))};
    return r;
}
vxo_point vxo_point_pow(vxo_point a, uint64_t k) {
    vxo_point r = IDENT, b = a;
    while (k) { if (k & 1) r = vxo_point_mul(r, b); b = vxo_point_mul(b, b); k >>= 1; }
    return r;
}
static vxo_point rep_double(vxo_point p, uint32_t n) { for (uint32_t i = 0; i < n; i++) p = vxo_point_mul(p, p); return p; }
vxo_coset vxo_coset_subgroup(uint32_t k) {
    vxo_coset c = {IDENT, rep_double(GEN, 31 - k), k}; return c;
}
vxo_coset vxo_coset_half_coset(uint32_t k) {
    vxo_coset c = {rep_double(GEN, 30 - k), rep_double(GEN, 31 - k), k}; return c;
}
vxo_coset vxo_coset_half_odds(uint32_t k) {
    vxo_coset c = {rep_double(GEN, k >= 29 ? 0 : 29 - k), rep_double(GEN, 31 - k), k}; return c;
}
vxo_point vxo_coset_at(const vxo_coset *c, uint64_t i) {
    return vxo_point_mul(c->initial, vxo_point_pow(c->step, (uint32_t)i));
}

/* all points p_j = initial * step^j, j < m (exact, so any evaluation order
 * gives the reference's coset_points values — twiddles.cu:80-105) */
static void coset_points(const vxo_coset *c, uint32_t *xs, uint32_t *ys) {
    uint64_t m = 1ull << c->log_size;
    const uint64_t CH = 4096;
    int64_t nch = (int64_t)((m + CH - 1) / CH);
    #pragma omp parallel for schedule(static)
    for (int64_t ci = 0; ci < nch; ci++) {
        uint64_t j0 = (uint64_t)ci * CH, j1 = j0 + CH < m ? j0 + CH : m;
        vxo_point p = vxo_coset_at(c, j0);
        for (uint64_t j = j0; j < j1; j++) {
            if (xs) xs[j] = p.x;
            if (ys) ys[j] = p.y;
            p = vxo_point_mul(p, c->step);
        }
    }
}

/* Montgomery batch inverse over aligned chunks of 64, exactly as the
 * reference kernel (batch_inverse.cu:8-41): a zero input maps to zero, and
 * the running prefix starts from the chunk's first element itself, so a zero
 * at a chunk's first slot makes the whole chunk's product (and hence every
 * output of that chunk) zero.  Reached only by the circle-fold twiddles of
 * subgroup(31), whose point 0 is the identity (y = 0). */
void vxo_batch_inverse(const uint32_t *in, uint32_t *out, size_t n) {
    const size_t CH = 64;
    int64_t nch = (int64_t)((n + CH - 1) / CH);
    #pragma omp parallel for schedule(static)
    for (int64_t ci = 0; ci < nch; ci++) {
        size_t s = (size_t)ci * CH, e = s + CH < n ? s + CH : n;
        uint32_t pre[64], val[64];
        for (size_t i = s; i < e; i++) val[i - s] = in[i];
        pre[0] = val[0];
        for (size_t i = 1; i < e - s; i++) pre[i] = val[i] ? m_mul(pre[i - 1], val[i]) : pre[i - 1];
        uint32_t inv = m_pow(pre[e - s - 1], P - 2);
        for (size_t i = e - s - 1; i > 0; i--) {
            if (!val[i]) { out[s + i] = 0; continue; }
            out[s + i] = m_mul(inv, pre[i - 1]);
            inv = m_mul(inv, val[i]);
        }
        out[s] = val[0] ? inv : 0;
    }
}

/* circle.rs:357-435 (compute_twiddles / compute_itwiddles) */
void vxo_twiddles(const vxo_coset *c, int inverse, uint32_t *line, uint32_t *circle, uint32_t *offsets) {
    uint32_t k = c->log_size;
    uint64_t m = 1ull << k;
    uint32_t *xs = (uint32_t *)malloc(m * 4), *ys = (uint32_t *)malloc(m * 4);
    coset_points(c, xs, ys);
    memcpy(circle, ys, (m / 2) * 4);
    uint32_t n_line = k > 0 ? k - 1 : 0;
    uint64_t cur_n = m, off = 0;
    uint32_t *cur = xs, *nxt = ys; /* ys no longer needed: reuse as scratch */
    for (uint32_t l = 0; l < n_line; l++) {
        uint64_t ls = cur_n / 2;
        offsets[l] = (uint32_t)off;
        #pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < (int64_t)ls; i++) {
            uint32_t x = cur[2 * i];
            line[off + i] = x;
            uint32_t x2 = m_mul(x, x);
            nxt[i] = m_sub(m_add(x2, x2), 1);
        }
        off += ls; cur_n = ls;
        uint32_t *t = cur; cur = nxt; nxt = t;
    }
    free(xs); free(ys);
    if (inverse) {
        if (off) vxo_batch_inverse(line, line, off);
        vxo_batch_inverse(circle, circle, m / 2);
    }
}

/* ------------------------------------------------------------------ */
/* circle NTT: circle_ntt.cu:74-117 (butterflies), 248-312 (order)    */
/* ------------------------------------------------------------------ */
void vxo_ntt_layer(uint32_t *d, const uint32_t *tw, uint32_t L, uint64_t n, int fwd) {
    int64_t half = (int64_t)(n / 2);
    uint64_t stride = 1ull << L;
    #pragma omp parallel for schedule(static)
    for (int64_t tid = 0; tid < half; tid++) {
        uint64_t h = (uint64_t)tid >> L, l = (uint64_t)tid & (stride - 1);
        uint64_t i0 = (h << (L + 1)) + l, i1 = i0 + stride;
        uint32_t v0 = d[i0], v1 = d[i1], t = tw[h];
        if (fwd) { uint32_t tmp = m_mul(v1, t); d[i1] = m_sub(v0, tmp); d[i0] = m_add(v0, tmp); }
        else { d[i0] = m_add(v0, v1); d[i1] = m_mul(m_sub(v0, v1), t); }
    }
}
void vxo_ntt_evaluate(uint32_t *d, const uint32_t *line, const uint32_t *circle, const uint32_t *offsets, uint32_t k) {
    uint64_t n = 1ull << k;
    uint32_t n_line = k > 0 ? k - 1 : 0;
    for (int l = (int)n_line - 1; l >= 0; l--) vxo_ntt_layer(d, line + offsets[l], (uint32_t)l + 1, n, 1);
    if (k > 0) vxo_ntt_layer(d, circle, 0, n, 1);
}
void vxo_ntt_interpolate(uint32_t *d, const uint32_t *iline, const uint32_t *icircle, const uint32_t *offsets, uint32_t k) {
    uint64_t n = 1ull << k;
    uint32_t n_line = k > 0 ? k - 1 : 0;
    if (k > 0) vxo_ntt_layer(d, icircle, 0, n, 0);
    for (uint32_t l = 0; l < n_line; l++) vxo_ntt_layer(d, iline + offsets[l], l + 1, n, 0);
    uint32_t e = (30u * k) % 31u;
    uint32_t inv_n = e == 0 ? 1u : (1u << e);
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; i++) d[i] = m_mul(d[i], inv_n);
}
static void with_tables(uint32_t *d, const vxo_coset *c, int inverse) {
    uint64_t m = 1ull << c->log_size;
    uint32_t *line = (uint32_t *)malloc((m > 1 ? m - 1 : 1) * 4), *circ = (uint32_t *)malloc((m / 2 + 1) * 4);
    uint32_t offs[32];
    vxo_twiddles(c, inverse, line, circ, offs);
    if (inverse) vxo_ntt_interpolate(d, line, circ, offs, c->log_size);
    else vxo_ntt_evaluate(d, line, circ, offs, c->log_size);
    free(line); free(circ);
}
void vxo_evaluate_on(uint32_t *d, const vxo_coset *c) { with_tables(d, c, 0); }
void vxo_interpolate_on(uint32_t *d, const vxo_coset *c) { with_tables(d, c, 1); }

static inline uint64_t brev(uint64_t i, uint32_t bits) {
    if (!bits) return 0;
    uint64_t r = 0;
    for (uint32_t b = 0; b < bits; b++) { r = (r << 1) | (i & 1); i >>= 1; }
    return r;
}
void vxo_bit_reverse(uint32_t *d, uint32_t log_n) {
    int64_t n = (int64_t)1 << log_n;
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) {
        uint64_t j = brev((uint64_t)i, log_n);
        if ((uint64_t)i < j) { uint32_t t = d[i]; d[i] = d[j]; d[j] = t; }
    }
}
static inline uint64_t hc_to_brt(uint64_t k, uint32_t log_n) {
    uint64_t n = 1ull << log_n;
    uint64_t cn = (k & 1) ? n - 1 - k / 2 : k / 2;
    return brev(cn, log_n);
}
void vxo_permute_hc_to_canonic_brt(const uint32_t *src, uint32_t *dst, uint32_t log_n) {
    int64_t n = (int64_t)1 << log_n;
    #pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < n; k++) dst[hc_to_brt((uint64_t)k, log_n)] = src[k];
}
void vxo_permute_canonic_brt_to_hc(const uint32_t *src, uint32_t *dst, uint32_t log_n) {
    int64_t n = (int64_t)1 << log_n;
    #pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < n; k++) dst[k] = src[hc_to_brt((uint64_t)k, log_n)];
}

/* ------------------------------------------------------------------ */
/* trace + quotient: air.rs:85-189, constraint.cu:10-64               */
/* ------------------------------------------------------------------ */
/* (F(k), F(k+1)) by 2x2 matrix power — air.rs:85-131 */
static void fib_at(uint32_t a, uint32_t b, uint64_t k, uint32_t *fk, uint32_t *fk1) {
    uint32_t m00 = 1, m01 = 0, m10 = 0, m11 = 1, b00 = 1, b01 = 1, b10 = 1, b11 = 0;
    while (k) {
        if (k & 1) {
            uint32_t t00 = m_add(m_mul(m00, b00), m_mul(m01, b10)), t01 = m_add(m_mul(m00, b01), m_mul(m01, b11));
            uint32_t t10 = m_add(m_mul(m10, b00), m_mul(m11, b10)), t11 = m_add(m_mul(m10, b01), m_mul(m11, b11));
            m00 = t00; m01 = t01; m10 = t10; m11 = t11;
        }
        uint32_t t00 = m_add(m_mul(b00, b00), m_mul(b01, b10)), t01 = m_add(m_mul(b00, b01), m_mul(b01, b11));
        uint32_t t10 = m_add(m_mul(b10, b00), m_mul(b11, b10)), t11 = m_add(m_mul(b10, b01), m_mul(b11, b11));
        b00 = t00; b01 = t01; b10 = t10; b11 = t11;
        k >>= 1;
    }
    *fk = m_add(m_mul(m10, b), m_mul(m11, a));
    *fk1 = m_add(m_mul(m00, b), m_mul(m01, a));
}
void vxo_fibonacci_trace(uint32_t a, uint32_t b, uint32_t log_n, uint32_t *out) {
    uint64_t n = 1ull << log_n;
    const uint64_t CH = 1ull << 16;
    int64_t nch = (int64_t)((n + CH - 1) / CH);
    #pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < nch; c++) {
        uint64_t s = (uint64_t)c * CH, e = s + CH < n ? s + CH : n;
        uint32_t f0, f1;
        fib_at(a, b, s, &f0, &f1);
        out[s] = f0;
        if (s + 1 < e) out[s + 1] = f1;
        for (uint64_t i = s + 2; i < e; i++) out[i] = m_add(out[i - 1], out[i - 2]);
    }
}
void vxo_fibonacci_quotient(const uint32_t *t, uint64_t n, const uint32_t alpha[4],
                            uint32_t *q0, uint32_t *q1, uint32_t *q2, uint32_t *q3) {
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; i++) {
        uint32_t c = m_sub(t[(i + 2) % n], m_add(t[(i + 1) % n], t[i]));
        q0[i] = m_mul(alpha[0], c); q1[i] = m_mul(alpha[1], c);
        q2[i] = m_mul(alpha[2], c); q3[i] = m_mul(alpha[3], c);
    }
}

/* ------------------------------------------------------------------ */
/* Blake2s-256 (RFC 7693; channel.rs:216-298, blake2s.cuh:55-136)      */
/* ------------------------------------------------------------------ */
static const uint32_t IV[8] = {0x6A09E667u, 0xBB67AE85u, 0x3C6EF372u, 0xA54FF53Au,
                               0x510E527Fu, 0x9B05688Cu, 0x1F83D9ABu, 0x5BE0CD19u};
static const uint8_t SIG[10][16] = {
    {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15}, {14, 10, 4, 8, 9, 15, 13, 6, 1, 12, 0, 2, 11, 7, 5, 3},
    {11, 8, 12, 0, 5, 2, 15, 13, 10, 14, 3, 6, 7, 1, 9, 4}, {7, 9, 3, 1, 13, 12, 11, 14, 2, 6, 5, 10, 4, 0, 15, 8},
    {9, 0, 5, 7, 2, 4, 10, 15, 14, 1, 11, 12, 6, 8, 3, 13}, {2, 12, 6, 10, 0, 11, 8, 3, 4, 13, 7, 5, 15, 14, 1, 9},
    {12, 5, 1, 15, 14, 13, 4, 10, 0, 7, 6, 3, 9, 2, 8, 11}, {13, 11, 7, 14, 12, 1, 3, 9, 5, 0, 15, 4, 8, 6, 2, 10},
    {6, 15, 14, 9, 11, 3, 0, 8, 12, 2, 13, 7, 1, 4, 10, 5}, {10, 2, 8, 4, 7, 6, 1, 5, 15, 11, 9, 14, 3, 12, 13, 0}};
static inline uint32_t rotr(uint32_t x, int n) { return (x >> n) | (x << (32 - n)); }
#define GM(a, b, c, d, x, y) do { \
    v[a] = v[a] + v[b] + (x); v[d] = rotr(v[d] ^ v[a], 16); v[c] = v[c] + v[d]; v[b] = rotr(v[b] ^ v[c], 12); \
    v[a] = v[a] + v[b] + (y); v[d] = rotr(v[d] ^ v[a], 8); v[c] = v[c] + v[d]; v[b] = rotr(v[b] ^ v[c], 7); } while (0)
void vxo_blake2s_compress_words(uint32_t h[8], const uint32_t m[16], uint32_t t, uint32_t f) {
    uint32_t v[16];
    for (int i = 0; i < 8; i++) { v[i] = h[i]; v[i + 8] = IV[i]; }
    v[12] ^= t; v[14] ^= f;
    for (int r = 0; r < 10; r++) {
        const uint8_t *s = SIG[r];
        GM(0, 4, 8, 12, m[s[0]], m[s[1]]); GM(1, 5, 9, 13, m[s[2]], m[s[3]]);
        GM(2, 6, 10, 14, m[s[4]], m[s[5]]); GM(3, 7, 11, 15, m[s[6]], m[s[7]]);
        GM(0, 5, 10, 15, m[s[8]], m[s[9]]); GM(1, 6, 11, 12, m[s[10]], m[s[11]]);
        GM(2, 7, 8, 13, m[s[12]], m[s[13]]); GM(3, 4, 9, 14, m[s[14]], m[s[15]]);
    }
    for (int i = 0; i < 8; i++) h[i] ^= v[i] ^ v[i + 8];
}
static inline uint32_t ld32(const uint8_t *p) { return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24); }
static inline void st32(uint8_t *p, uint32_t v) { p[0] = (uint8_t)v; p[1] = (uint8_t)(v >> 8); p[2] = (uint8_t)(v >> 16); p[3] = (uint8_t)(v >> 24); }
void vxo_blake2s(const uint8_t *in, size_t len, uint8_t out[32]) {
    uint32_t h[8];
    for (int i = 0; i < 8; i++) h[i] = IV[i];
    h[0] ^= 0x01010020u;
    uint32_t m[16];
    size_t off = 0;
    while (len - off > 64) {
        for (int i = 0; i < 16; i++) m[i] = ld32(in + off + 4 * i);
        off += 64;
        vxo_blake2s_compress_words(h, m, (uint32_t)off, 0);
    }
    uint8_t blk[64] = {0};
    memcpy(blk, in + off, len - off);
    for (int i = 0; i < 16; i++) m[i] = ld32(blk + 4 * i);
    vxo_blake2s_compress_words(h, m, (uint32_t)len, 0xFFFFFFFFu);
    for (int i = 0; i < 8; i++) st32(out + 4 * i, h[i]);
}
/* single-block word hash: t = 4*n (n <= 16), the GPU leaf convention */
static inline void hash_words16(const uint32_t *w, uint32_t n, uint32_t out[8]) {
    uint32_t m[16] = {0};
    if (n > 16) n = 16;
    for (uint32_t i = 0; i < n; i++) m[i] = w[i];
    for (int i = 0; i < 8; i++) out[i] = IV[i];
    out[0] ^= 0x01010020u;
    vxo_blake2s_compress_words(out, m, 4 * n, 0xFFFFFFFFu);
}
void vxo_hash_leaf(const uint32_t *w, uint32_t n, uint32_t out[8]) { hash_words16(w, n, out); }
void vxo_hash_pair(const uint32_t l[8], const uint32_t r[8], uint32_t out[8]) {
    uint32_t m[16];
    memcpy(m, l, 32); memcpy(m + 8, r, 32);
    hash_words16(m, 16, out);
}

/* ------------------------------------------------------------------ */
/* Merkle: merkle.rs:28-130 (layout), 455-497 (paths), 520-566        */
/* ------------------------------------------------------------------ */
void vxo_tree_build(vxo_tree *t, const uint32_t *const *cols, uint32_t n_cols, uint32_t log_n) {
    t->log_n = log_n;
    t->levels = (uint32_t **)calloc(log_n + 1, sizeof(uint32_t *));
    uint64_t n = 1ull << log_n;
    uint32_t *lv = (uint32_t *)malloc(n * 32);
    uint32_t nc = n_cols > 16 ? 16 : n_cols;
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; i++) {
        uint32_t w[16];
        for (uint32_t c = 0; c < nc; c++) w[c] = cols[c][i];
        hash_words16(w, nc, lv + 8 * i);
    }
    t->levels[0] = lv;
    for (uint32_t l = 1; l <= log_n; l++) {
        uint64_t m = n >> l;
        uint32_t *up = (uint32_t *)malloc(m * 32), *dn = t->levels[l - 1];
        #pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < (int64_t)m; i++) vxo_hash_pair(dn + 16 * i, dn + 16 * i + 8, up + 8 * i);
        t->levels[l] = up;
    }
}
void vxo_tree_free(vxo_tree *t) {
    if (!t->levels) return;
    for (uint32_t l = 0; l <= t->log_n; l++) free(t->levels[l]);
    free(t->levels); t->levels = NULL;
}
void vxo_tree_root(const vxo_tree *t, uint32_t out[8]) { memcpy(out, t->levels[t->log_n], 32); }
void vxo_tree_path(const vxo_tree *t, uint64_t idx, uint32_t *out) {
    for (uint32_t l = 0; l < t->log_n; l++) {
        memcpy(out + 8 * l, t->levels[l] + 8 * (idx ^ 1), 32);
        idx >>= 1;
    }
}
void vxo_merkle_root(const uint32_t *const *cols, uint32_t n_cols, uint32_t log_n, uint32_t out[8]) {
    vxo_tree t; vxo_tree_build(&t, cols, n_cols, log_n); vxo_tree_root(&t, out); vxo_tree_free(&t);
}
int vxo_verify_path(const uint32_t root[8], const uint32_t leaf[8], uint64_t idx, const uint32_t *path, uint32_t depth) {
    uint32_t cur[8];
    memcpy(cur, leaf, 32);
    for (uint32_t l = 0; l < depth; l++) {
        uint32_t nx[8];
        if (idx & 1) vxo_hash_pair(path + 8 * l, cur, nx); else vxo_hash_pair(cur, path + 8 * l, nx);
        memcpy(cur, nx, 32);
        idx >>= 1;
    }
    return memcmp(cur, root, 32) == 0;
}
void vxo_lifted_leaves(const uint32_t *const *cols, const uint32_t *log_sizes, uint32_t n_cols,
                       uint32_t S, uint32_t *out) {
    uint64_t n = 1ull << S;
    #pragma omp parallel for schedule(static)
    for (int64_t idx = 0; idx < (int64_t)n; idx++) {
        uint8_t *buf = (uint8_t *)malloc(4 * (size_t)n_cols + 1);
        for (uint32_t c = 0; c < n_cols; c++) {
            uint32_t L = log_sizes[c];
            uint64_t row = (L == S) ? (uint64_t)idx : ((((uint64_t)idx >> (S - L + 1)) << 1) | ((uint64_t)idx & 1));
            st32(buf + 4 * c, cols[c][row]);
        }
        uint8_t dg[32];
        vxo_blake2s(buf, 4 * (size_t)n_cols, dg);
        for (int i = 0; i < 8; i++) out[8 * idx + i] = ld32(dg + 4 * i);
        free(buf);
    }
}

/* ------------------------------------------------------------------ */
/* FRI: fri.rs:73-224 (twiddles, folds), twiddles.cu:23-52            */
/* ------------------------------------------------------------------ */
void vxo_fold_twiddles(const vxo_coset *dom, int extract_y, uint32_t *out) {
    uint32_t k = dom->log_size;
    int64_t half = (int64_t)1 << (k - 1);
    uint32_t *src = (uint32_t *)malloc((size_t)half * 4);
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < half; i++) {
        vxo_point p = vxo_coset_at(dom, brev((uint64_t)i << 1, k));
        src[i] = extract_y ? p.y : p.x;
    }
    vxo_batch_inverse(src, out, (size_t)half);
    free(src);
}
void vxo_fold_line(const uint32_t *const in[4], const uint32_t *tw, const uint32_t alpha[4],
                   uint32_t *const out[4], uint64_t half_n) {
    qm al; memcpy(al.v, alpha, 16);
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)half_n; i++) {
        qm f0, f1;
        for (int c = 0; c < 4; c++) { f0.v[c] = in[c][2 * i]; f1.v[c] = in[c][2 * i + 1]; }
        qm r = q_add(q_add(f0, f1), q_mul(al, q_mulm(q_sub(f0, f1), tw[i])));
        for (int c = 0; c < 4; c++) out[c][i] = r.v[c];
    }
}
void vxo_fold_circle_into_line(uint32_t *const dst[4], const uint32_t *const src[4], const uint32_t *tw,
                               const uint32_t alpha[4], const uint32_t alpha_sq[4], uint64_t half_n) {
    qm al, al2; memcpy(al.v, alpha, 16); memcpy(al2.v, alpha_sq, 16);
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)half_n; i++) {
        qm f0, f1, prev;
        for (int c = 0; c < 4; c++) { f0.v[c] = src[c][2 * i]; f1.v[c] = src[c][2 * i + 1]; prev.v[c] = dst[c][i]; }
        qm fp = q_add(q_add(f0, f1), q_mul(al, q_mulm(q_sub(f0, f1), tw[i])));
        qm r = q_add(q_mul(prev, al2), fp);
        for (int c = 0; c < 4; c++) dst[c][i] = r.v[c];
    }
}

/* ------------------------------------------------------------------ */
/* channel: channel.rs:15-185                                         */
/* ------------------------------------------------------------------ */
void vxo_channel_init(vxo_channel *ch) { memset(ch->state, 0, 32); ch->n_draws = 0; }
void vxo_channel_mix_digest(vxo_channel *ch, const uint32_t d[8]) {
    uint8_t in[64];
    memcpy(in, ch->state, 32);
    for (int i = 0; i < 8; i++) st32(in + 32 + 4 * i, d[i]);
    vxo_blake2s(in, 64, ch->state);
    ch->n_draws = 0;
}
void vxo_channel_mix_felts(vxo_channel *ch, const uint32_t *f, size_t nf) {
    if (!nf) return;
    size_t len = 32 + 16 * nf;
    uint8_t *in = (uint8_t *)malloc(len);
    memcpy(in, ch->state, 32);
    for (size_t i = 0; i < 4 * nf; i++) st32(in + 32 + 4 * i, f[i]);
    vxo_blake2s(in, len, ch->state);
    free(in);
    ch->n_draws = 0;
}
static void squeeze(vxo_channel *ch, uint8_t out[32]) {
    uint8_t in[37];
    memcpy(in, ch->state, 32);
    st32(in + 32, ch->n_draws);
    in[36] = 0;
    ch->n_draws++;
    vxo_blake2s(in, 37, out);
}
void vxo_channel_draw_felt(vxo_channel *ch, uint32_t out[4]) {
    for (;;) {
        uint8_t b[32];
        squeeze(ch, b);
        uint32_t w[8];
        int ok = 1;
        for (int i = 0; i < 8; i++) { w[i] = ld32(b + 4 * i); if (w[i] >= 2 * P) ok = 0; }
        if (ok) { for (int i = 0; i < 4; i++) out[i] = w[i] % P; return; }
    }
}
uint64_t vxo_channel_draw_number(vxo_channel *ch, uint64_t bound) {
    uint8_t b[32];
    squeeze(ch, b);
    uint64_t raw = (uint64_t)ld32(b) | ((uint64_t)ld32(b + 4) << 32);
    return raw % bound;
}
void vxo_channel_draw_query_indices(vxo_channel *ch, uint32_t log_domain, uint32_t n, uint32_t *out) {
    uint32_t mask = (uint32_t)((1ull << log_domain) - 1), got = 0;
    while (got < n) {
        uint8_t b[32];
        squeeze(ch, b);
        for (int i = 0; i < 8 && got < n; i++) out[got++] = ld32(b + 4 * i) & mask;
    }
}

/* ------------------------------------------------------------------ */
/* whole proof: prover.rs:264-619, bytes: stark_cli.rs:1051-1123      */
/* ------------------------------------------------------------------ */
typedef struct { uint8_t *p; size_t n, cap; } wbuf;
static void wr(wbuf *w, uint32_t v) {
    if (w->n + 4 > w->cap) { w->cap = w->cap * 2 + 4096; w->p = (uint8_t *)realloc(w->p, w->cap); }
    st32(w->p + w->n, v); w->n += 4;
}
static void wrs(wbuf *w, const uint32_t *s, size_t k) { for (size_t i = 0; i < k; i++) wr(w, s[i]); }

size_t vxo_proof_size(uint32_t log_n, uint32_t B, uint32_t nq) {
    uint32_t le = log_n + B, nfri = le - 3;
    size_t s = 4 * (5 + 8 + 8 + 1 + 8 * (size_t)nfri + 1 + 4 * 8 + 1 + nq);
    s += 4 + 8 * (size_t)nq + 2 * (size_t)nq * (4 + 32 * (size_t)le);
    s += 4 + 32 * (size_t)nq + 2 * (size_t)nq * (4 + 32 * (size_t)le);
    s += 4;
    for (uint32_t k = 0; k < nfri; k++) {
        uint32_t d = le - 1 - k;
        s += 4 + 32 * (size_t)nq + 2 * (size_t)nq * (4 + 32 * (size_t)d);
    }
    return s;
}

/* one decommitment block: n, values, sibling values, paths, sibling paths */
static void write_decom(wbuf *w, const vxo_tree *t, const uint32_t *const *cols, uint32_t nc,
                        const uint64_t *idx, uint32_t nq) {
    wr(w, nq);
    for (uint32_t q = 0; q < nq; q++) for (uint32_t c = 0; c < nc; c++) wr(w, cols[c][idx[q]]);
    for (uint32_t q = 0; q < nq; q++) for (uint32_t c = 0; c < nc; c++) wr(w, cols[c][idx[q] ^ 1]);
    uint32_t *path = (uint32_t *)malloc(((size_t)t->log_n + 1) * 32);
    for (int s = 0; s < 2; s++)
        for (uint32_t q = 0; q < nq; q++) {
            vxo_tree_path(t, idx[q] ^ (uint64_t)s, path);
            wr(w, t->log_n);
            wrs(w, path, 8 * (size_t)t->log_n);
        }
    free(path);
}

static vxo_coset eval_domain(uint32_t le) { return le <= 30 ? vxo_coset_half_coset(le) : vxo_coset_subgroup(le); }

static int prove_impl(uint32_t a, uint32_t b, uint32_t log_n, uint32_t B, uint32_t nq,
                      uint8_t **out, size_t *out_len, uint32_t *roots_out) {
    if (log_n < 4 || log_n + B > 31 || a >= P || b >= P) return 1;
    uint32_t le = log_n + B;
    uint64_t n = 1ull << log_n, N = 1ull << le;
    /* trace -> interpolate on half_coset(log_n) */
    uint32_t *eval = (uint32_t *)calloc(N, 4);
    vxo_fibonacci_trace(a, b, log_n, eval);
    vxo_coset tdom = vxo_coset_half_coset(log_n);
    vxo_interpolate_on(eval, &tdom);
    /* zero pad (already zero) -> evaluate on the eval domain */
    vxo_coset edom = eval_domain(le);
    vxo_evaluate_on(eval, &edom);
    (void)n;
    /* trace commitment */
    vxo_tree ttree;
    const uint32_t *tcols[1] = {eval};
    vxo_tree_build(&ttree, tcols, 1, le);
    uint32_t troot[8]; vxo_tree_root(&ttree, troot);
    vxo_channel ch; vxo_channel_init(&ch);
    vxo_channel_mix_digest(&ch, troot);
    uint32_t alpha[4]; vxo_channel_draw_felt(&ch, alpha);
    /* quotient + commitment */
    uint32_t *q[4];
    for (int c = 0; c < 4; c++) q[c] = (uint32_t *)malloc(N * 4);
    vxo_fibonacci_quotient(eval, N, alpha, q[0], q[1], q[2], q[3]);
    vxo_tree qtree;
    vxo_tree_build(&qtree, (const uint32_t *const *)q, 4, le);
    uint32_t qroot[8]; vxo_tree_root(&qtree, qroot);
    vxo_channel_mix_digest(&ch, qroot);
    /* FRI */
    uint32_t nfri = le - 3;
    uint32_t **lay = (uint32_t **)calloc((size_t)nfri * 4, sizeof(uint32_t *));
    vxo_tree *ftree = (vxo_tree *)calloc(nfri, sizeof(vxo_tree));
    uint32_t *froots = (uint32_t *)malloc((size_t)nfri * 32);
    uint32_t fa[4]; vxo_channel_draw_felt(&ch, fa);
    uint32_t fa2[4]; vxo_qm31_mul(fa, fa, fa2);
    uint32_t *tw = (uint32_t *)malloc((N / 2) * 4);
    vxo_fold_twiddles(&edom, 1, tw);
    for (int c = 0; c < 4; c++) lay[c] = (uint32_t *)calloc(N / 2, 4);
    vxo_fold_circle_into_line(lay, (const uint32_t *const *)q, tw, fa, fa2, N / 2);
    uint32_t cur = le - 1;
    vxo_tree_build(&ftree[0], (const uint32_t *const *)lay, 4, cur);
    vxo_tree_root(&ftree[0], froots);
    vxo_channel_mix_digest(&ch, froots);
    for (uint32_t k = 1; k < nfri; k++) {
        uint32_t al[4]; vxo_channel_draw_felt(&ch, al);
        vxo_coset dom = vxo_coset_half_odds(cur);
        uint64_t half = 1ull << (cur - 1);
        vxo_fold_twiddles(&dom, 0, tw);
        for (int c = 0; c < 4; c++) lay[4 * k + c] = (uint32_t *)malloc(half * 4);
        vxo_fold_line((const uint32_t *const *)(lay + 4 * (k - 1)), tw, al, lay + 4 * k, half);
        cur--;
        vxo_tree_build(&ftree[k], (const uint32_t *const *)(lay + 4 * k), 4, cur);
        vxo_tree_root(&ftree[k], froots + 8 * k);
        vxo_channel_mix_digest(&ch, froots + 8 * k);
    }
    free(tw);
    /* last layer (8 QM31) -> mix_felts -> queries */
    uint32_t last[32];
    for (int i = 0; i < 8; i++) for (int c = 0; c < 4; c++) last[4 * i + c] = lay[4 * (nfri - 1) + c][i];
    vxo_channel_mix_felts(&ch, last, 8);
    uint64_t *qi = (uint64_t *)malloc(sizeof(uint64_t) * (nq ? nq : 1));
    for (uint32_t j = 0; j < nq; j++) qi[j] = vxo_channel_draw_number(&ch, N);

    if (roots_out) {
        memcpy(roots_out, troot, 32); memcpy(roots_out + 8, qroot, 32);
        memcpy(roots_out + 16, froots, (size_t)nfri * 32);
    }
    if (out) {
        wbuf w = {NULL, 0, 0};
        w.cap = vxo_proof_size(log_n, B, nq); w.p = (uint8_t *)malloc(w.cap);
        wr(&w, 0x4B52414Bu); wr(&w, 1); wr(&w, log_n); wr(&w, a); wr(&w, b);
        wrs(&w, troot, 8); wrs(&w, qroot, 8);
        wr(&w, nfri); wrs(&w, froots, 8 * (size_t)nfri);
        wr(&w, 8); wrs(&w, last, 32);
        wr(&w, nq); for (uint32_t j = 0; j < nq; j++) wr(&w, (uint32_t)qi[j]);
        write_decom(&w, &ttree, tcols, 1, qi, nq);
        write_decom(&w, &qtree, (const uint32_t *const *)q, 4, qi, nq);
        wr(&w, nfri);
        uint64_t *fi = (uint64_t *)malloc(sizeof(uint64_t) * (nq ? nq : 1));
        for (uint32_t j = 0; j < nq; j++) fi[j] = qi[j] >> 1;
        for (uint32_t k = 0; k < nfri; k++) {
            write_decom(&w, &ftree[k], (const uint32_t *const *)(lay + 4 * k), 4, fi, nq);
            for (uint32_t j = 0; j < nq; j++) fi[j] >>= 1;
        }
        free(fi);
        *out = w.p; *out_len = w.n;
    }
    free(qi);
    for (uint32_t k = 0; k < nfri; k++) { vxo_tree_free(&ftree[k]); for (int c = 0; c < 4; c++) free(lay[4 * k + c]); }
    free(ftree); free(lay); free(froots);
    vxo_tree_free(&qtree); for (int c = 0; c < 4; c++) free(q[c]);
    vxo_tree_free(&ttree); free(eval);
    return 0;
}
int vxo_prove(uint32_t a, uint32_t b, uint32_t log_n, uint32_t B, uint32_t nq, uint8_t **out, size_t *out_len) {
    return prove_impl(a, b, log_n, B, nq, out, out_len, NULL);
}

/* ------------------------------------------------------------------ */
/* the same proof in bounded host memory (for 2^30- and 2^31-point     */
/* proofs): prover.rs:264-619 computes the same values; only what is    */
/* kept in memory differs.                                              */
/*  - The quotient q = alpha (t[i+2] - t[i+1] - t[i]) is never stored:  */
/*    its leaves, its circle fold and its openings recompute it from    */
/*    the evaluation (constraint.cu:10-64; prover.rs:1522-1530 does the */
/*    same on the host).                                                */
/*  - A tree keeps its levels from height K up; an authentication path */
/*    re-hashes the 2^K-leaf subtree of its leaf (merkle.rs:455-497     */
/*    reads the same siblings from a full tree).                        */
/* At log_n = 30 / blowup 1 the peak is the evaluation (8 GiB), the FRI */
/* layers (32 GiB) and the fold twiddles (4 GiB).                       */
/* ------------------------------------------------------------------ */
enum { LSRC_TRACE = 0, LSRC_QUOT = 1, LSRC_COLS4 = 2 };
typedef struct {
    int kind;
    const uint32_t *t;        /* trace evaluation (TRACE, QUOT) */
    uint64_t n;               /* leaves */
    uint32_t alpha[4];        /* QUOT */
    const uint32_t *c[4];     /* COLS4 */
} lsrc;

static inline uint32_t quot_c(const uint32_t *t, uint64_t n, uint64_t i) {
    return m_sub(t[(i + 2) % n], m_add(t[(i + 1) % n], t[i]));
}
static inline uint32_t lsrc_words(const lsrc *s, uint64_t i, uint32_t w[4]) {
    switch (s->kind) {
    case LSRC_TRACE: w[0] = s->t[i]; return 1;
    case LSRC_QUOT: {
        uint32_t c = quot_c(s->t, s->n, i);
        for (int k = 0; k < 4; k++) w[k] = m_mul(s->alpha[k], c);
        return 4;
    }
    default:
        for (int k = 0; k < 4; k++) w[k] = s->c[k][i];
        return 4;
    }
}

typedef struct { uint32_t log_n, K; uint32_t **levels; lsrc src; } ltree;

/* 2^K leaves of subtree j hashed and reduced in place; levels (if non-NULL)
 * receives every level of the subtree, leaves first (2^(K+1) - 1 hashes). */
static void lsub(const lsrc *s, uint32_t K, uint64_t j, uint32_t *levels, uint32_t out[8]) {
    uint64_t m = 1ull << K;
    uint32_t *buf = levels ? levels : (uint32_t *)malloc(m * 32);
    for (uint64_t i = 0; i < m; i++) {
        uint32_t w[4];
        uint32_t nw = lsrc_words(s, (j << K) + i, w);
        hash_words16(w, nw, buf + 8 * i);
    }
    uint32_t *dn = buf;
    for (uint32_t l = 1; l <= K; l++) {
        uint64_t cnt = m >> l;
        uint32_t *up = levels ? dn + 8 * (cnt * 2) : buf;
        for (uint64_t i = 0; i < cnt; i++) vxo_hash_pair(dn + 16 * i, dn + 16 * i + 8, up + 8 * i);
        dn = up;
    }
    memcpy(out, dn, 32);
    if (!levels) free(buf);
}

static void ltree_build(ltree *t, const lsrc *s, uint32_t log_n) {
    t->log_n = log_n;
    t->K = log_n < 8 ? log_n : 8;
    t->src = *s;
    t->levels = (uint32_t **)calloc(log_n + 1, sizeof(uint32_t *));
    uint64_t nk = 1ull << (log_n - t->K);
    uint32_t *lk = (uint32_t *)malloc(nk * 32);
    #pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < (int64_t)nk; j++) lsub(&t->src, t->K, (uint64_t)j, NULL, lk + 8 * j);
    t->levels[t->K] = lk;
    for (uint32_t l = t->K + 1; l <= log_n; l++) {
        uint64_t m = 1ull << (log_n - l);
        uint32_t *up = (uint32_t *)malloc(m * 32), *dn = t->levels[l - 1];
        #pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < (int64_t)m; i++) vxo_hash_pair(dn + 16 * i, dn + 16 * i + 8, up + 8 * i);
        t->levels[l] = up;
    }
}
static void ltree_free(ltree *t) {
    if (!t->levels) return;
    for (uint32_t l = t->K; l <= t->log_n; l++) free(t->levels[l]);
    free(t->levels); t->levels = NULL;
}
static void ltree_path(const ltree *t, uint64_t idx, uint32_t *out) {
    uint32_t K = t->K;
    uint64_t m = 1ull << K;
    uint32_t *sub = (uint32_t *)malloc((2 * m) * 32), root[8];
    lsub(&t->src, K, idx >> K, sub, root);
    uint64_t off = 0, cnt = m, li = idx & (m - 1);
    for (uint32_t l = 0; l < K; l++) {
        memcpy(out + 8 * l, sub + 8 * (off + (li ^ 1)), 32);
        off += cnt; cnt >>= 1; li >>= 1;
    }
    uint64_t hi = idx >> K;
    for (uint32_t l = K; l < t->log_n; l++) {
        memcpy(out + 8 * l, t->levels[l] + 8 * (hi ^ 1), 32);
        hi >>= 1;
    }
    free(sub);
}
static void write_ldecom(wbuf *w, const ltree *t, const uint64_t *idx, uint32_t nq) {
    uint32_t v[4];
    wr(w, nq);
    for (int s = 0; s < 2; s++)
        for (uint32_t q = 0; q < nq; q++) {
            uint32_t nw = lsrc_words(&t->src, idx[q] ^ (uint64_t)s, v);
            wrs(w, v, nw);
        }
    uint32_t *path = (uint32_t *)malloc(((size_t)t->log_n + 1) * 32);
    for (int s = 0; s < 2; s++)
        for (uint32_t q = 0; q < nq; q++) {
            ltree_path(t, idx[q] ^ (uint64_t)s, path);
            wr(w, t->log_n);
            wrs(w, path, 8 * (size_t)t->log_n);
        }
    free(path);
}

int vxo_prove_lean(uint32_t a, uint32_t b, uint32_t log_n, uint32_t B, uint32_t nq, uint8_t **out, size_t *out_len) {
    if (log_n < 4 || log_n + B > 31 || a >= P || b >= P || !out || !out_len) return 1;
    uint32_t le = log_n + B;
    uint64_t N = 1ull << le;
    uint32_t *eval = (uint32_t *)calloc(N, 4);
    if (!eval) return 2;
    vxo_fibonacci_trace(a, b, log_n, eval);
    vxo_coset tdom = vxo_coset_half_coset(log_n);
    vxo_interpolate_on(eval, &tdom);
    vxo_coset edom = eval_domain(le);
    vxo_evaluate_on(eval, &edom);
    lsrc ts = {LSRC_TRACE, eval, N, {0, 0, 0, 0}, {NULL, NULL, NULL, NULL}};
    ltree ttree;
    ltree_build(&ttree, &ts, le);
    uint32_t troot[8]; memcpy(troot, ttree.levels[le], 32);
    vxo_channel ch; vxo_channel_init(&ch);
    vxo_channel_mix_digest(&ch, troot);
    lsrc qs = {LSRC_QUOT, eval, N, {0, 0, 0, 0}, {NULL, NULL, NULL, NULL}};
    vxo_channel_draw_felt(&ch, qs.alpha);
    ltree qtree;
    ltree_build(&qtree, &qs, le);
    uint32_t qroot[8]; memcpy(qroot, qtree.levels[le], 32);
    vxo_channel_mix_digest(&ch, qroot);
    uint32_t nfri = le - 3;
    uint32_t **lay = (uint32_t **)calloc((size_t)nfri * 4, sizeof(uint32_t *));
    ltree *ftree = (ltree *)calloc(nfri, sizeof(ltree));
    uint32_t *froots = (uint32_t *)malloc((size_t)nfri * 32);
    uint32_t fa[4]; vxo_channel_draw_felt(&ch, fa);
    uint32_t fa2[4]; vxo_qm31_mul(fa, fa, fa2);
    uint32_t *tw = (uint32_t *)malloc((N / 2) * 4);
    vxo_fold_twiddles(&edom, 1, tw);
    for (int c = 0; c < 4; c++) lay[c] = (uint32_t *)malloc((N / 2) * 4);
    {   /* circle fold of the recomputed quotient into a zero accumulator (fri.rs:163-191) */
        qm al, al2; memcpy(al.v, fa, 16); memcpy(al2.v, fa2, 16);
        #pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < (int64_t)(N / 2); i++) {
            qm f0 = {{0, 0, 0, 0}}, f1 = {{0, 0, 0, 0}}, prev = {{0, 0, 0, 0}};
            lsrc_words(&qs, 2 * (uint64_t)i, f0.v);
            lsrc_words(&qs, 2 * (uint64_t)i + 1, f1.v);
            qm fp = q_add(q_add(f0, f1), q_mul(al, q_mulm(q_sub(f0, f1), tw[i])));
            qm r = q_add(q_mul(prev, al2), fp);
            for (int c = 0; c < 4; c++) lay[c][i] = r.v[c];
        }
    }
    uint32_t cur = le - 1;
    lsrc fs = {LSRC_COLS4, NULL, 1ull << cur, {0, 0, 0, 0}, {lay[0], lay[1], lay[2], lay[3]}};
    ltree_build(&ftree[0], &fs, cur);
    memcpy(froots, ftree[0].levels[cur], 32);
    vxo_channel_mix_digest(&ch, froots);
    for (uint32_t k = 1; k < nfri; k++) {
        uint32_t al[4]; vxo_channel_draw_felt(&ch, al);
        vxo_coset dom = vxo_coset_half_odds(cur);
        uint64_t half = 1ull << (cur - 1);
        vxo_fold_twiddles(&dom, 0, tw);
        for (int c = 0; c < 4; c++) lay[4 * k + c] = (uint32_t *)malloc(half * 4);
        vxo_fold_line((const uint32_t *const *)(lay + 4 * (k - 1)), tw, al, lay + 4 * k, half);
        cur--;
        lsrc ks = {LSRC_COLS4, NULL, 1ull << cur, {0, 0, 0, 0},
                   {lay[4 * k], lay[4 * k + 1], lay[4 * k + 2], lay[4 * k + 3]}};
        ltree_build(&ftree[k], &ks, cur);
        memcpy(froots + 8 * k, ftree[k].levels[cur], 32);
        vxo_channel_mix_digest(&ch, froots + 8 * k);
    }
    free(tw);
    uint32_t last[32];
    for (int i = 0; i < 8; i++) for (int c = 0; c < 4; c++) last[4 * i + c] = lay[4 * (nfri - 1) + c][i];
    vxo_channel_mix_felts(&ch, last, 8);
    uint64_t *qi = (uint64_t *)malloc(sizeof(uint64_t) * (nq ? nq : 1));
    for (uint32_t j = 0; j < nq; j++) qi[j] = vxo_channel_draw_number(&ch, N);
    wbuf w = {NULL, 0, 0};
    w.cap = vxo_proof_size(log_n, B, nq); w.p = (uint8_t *)malloc(w.cap);
    wr(&w, 0x4B52414Bu); wr(&w, 1); wr(&w, log_n); wr(&w, a); wr(&w, b);
    wrs(&w, troot, 8); wrs(&w, qroot, 8);
    wr(&w, nfri); wrs(&w, froots, 8 * (size_t)nfri);
    wr(&w, 8); wrs(&w, last, 32);
    wr(&w, nq); for (uint32_t j = 0; j < nq; j++) wr(&w, (uint32_t)qi[j]);
    write_ldecom(&w, &ttree, qi, nq);
    write_ldecom(&w, &qtree, qi, nq);
    wr(&w, nfri);
    uint64_t *fi = (uint64_t *)malloc(sizeof(uint64_t) * (nq ? nq : 1));
    for (uint32_t j = 0; j < nq; j++) fi[j] = qi[j] >> 1;
    for (uint32_t k = 0; k < nfri; k++) {
        write_ldecom(&w, &ftree[k], fi, nq);
        for (uint32_t j = 0; j < nq; j++) fi[j] >>= 1;
    }
    free(fi); free(qi);
    *out = w.p; *out_len = w.n;
    for (uint32_t k = 0; k < nfri; k++) { ltree_free(&ftree[k]); for (int c = 0; c < 4; c++) free(lay[4 * k + c]); }
    free(ftree); free(lay); free(froots);
    ltree_free(&qtree); ltree_free(&ttree); free(eval);
    return 0;
}
int vxo_prove_roots(uint32_t a, uint32_t b, uint32_t log_n, uint32_t B,
                    uint32_t *tr, uint32_t *qr, uint32_t *fr) {
    uint32_t le = log_n + B;
    uint32_t *r = (uint32_t *)malloc((size_t)(2 + le) * 32);
    int rc = prove_impl(a, b, log_n, B, 0, NULL, NULL, r);
    if (!rc) { memcpy(tr, r, 32); memcpy(qr, r + 8, 32); memcpy(fr, r + 16, (size_t)(le - 3) * 32); }
    free(r);
    return rc;
}
void vxo_free(void *p) { free(p); }
void vxo_set_threads(int n) {
#ifdef _OPENMP
    omp_set_num_threads(n);
#else
    (void)n;
#endif
}
int vxo_get_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------------ */
/* verifier.rs:39-310 over the byte layout                             */
/* ------------------------------------------------------------------ */
typedef struct { const uint8_t *p; size_t n, off; int bad; } rbuf;
static uint32_t rd(rbuf *r) {
    if (r->off + 4 > r->n) { r->bad = 1; return 0; }
    uint32_t v = ld32(r->p + r->off); r->off += 4; return v;
}
#define FAIL(code, ...) do { if (msg) snprintf(msg, msg_len, __VA_ARGS__); rc = code; goto done; } while (0)

typedef struct { uint32_t n; uint32_t *vals, *svals; uint32_t *paths, *spaths; uint32_t depth_ok; } decom_t;
static int read_decom(rbuf *r, decom_t *d, uint32_t width, uint32_t depth) {
    d->n = rd(r);
    if (r->bad || d->n > (1u << 20)) return 0;
    d->vals = (uint32_t *)malloc((size_t)d->n * width * 4 + 4);
    d->svals = (uint32_t *)malloc((size_t)d->n * width * 4 + 4);
    d->paths = (uint32_t *)malloc((size_t)d->n * depth * 32 + 4);
    d->spaths = (uint32_t *)malloc((size_t)d->n * depth * 32 + 4);
    d->depth_ok = 1;
    for (size_t i = 0; i < (size_t)d->n * width; i++) d->vals[i] = rd(r);
    for (size_t i = 0; i < (size_t)d->n * width; i++) d->svals[i] = rd(r);
    for (int s = 0; s < 2; s++)
        for (uint32_t q = 0; q < d->n; q++) {
            uint32_t dep = rd(r);
            if (dep != depth) { d->depth_ok = 0; r->bad = 1; return 0; }
            uint32_t *dst = (s ? d->spaths : d->paths) + (size_t)q * depth * 8;
            for (uint32_t i = 0; i < depth * 8; i++) dst[i] = rd(r);
        }
    return !r->bad;
}
static void free_decom(decom_t *d) { free(d->vals); free(d->svals); free(d->paths); free(d->spaths); }
static int check_decom(const decom_t *d, const uint32_t root[8], const uint64_t *idx, uint32_t width, uint32_t depth, uint32_t nq) {
    if (d->n != nq) return 0;
    for (uint32_t q = 0; q < nq; q++) {
        uint32_t h[8];
        hash_words16(d->vals + (size_t)q * width, width, h);
        if (!vxo_verify_path(root, h, idx[q], d->paths + (size_t)q * depth * 8, depth)) return 0;
        hash_words16(d->svals + (size_t)q * width, width, h);
        if (!vxo_verify_path(root, h, idx[q] ^ 1, d->spaths + (size_t)q * depth * 8, depth)) return 0;
    }
    return 1;
}
static qm fold_pair(qm f0, qm f1, qm al, uint32_t tw) {
    return q_add(q_add(f0, f1), q_mul(al, q_mulm(q_sub(f0, f1), tw)));
}
static uint32_t fold_tw_at(const vxo_coset *dom, uint64_t fi, int circle) {
    vxo_point p = vxo_coset_at(dom, brev(fi << 1, dom->log_size));
    return vxo_m31_inv(circle ? p.y : p.x);
}
int vxo_verify(const uint8_t *proof, size_t len, uint32_t B, uint32_t nq, char *msg, size_t msg_len) {
    int rc = 0;
    rbuf r = {proof, len, 0, 0};
    decom_t td = {0}, qd = {0}, *fd = NULL;
    uint32_t nfd = 0, nfri = 0, *froots = NULL, *fal = NULL;
    uint64_t *qi = NULL, *fi = NULL;
    if (rd(&r) != 0x4B52414Bu) FAIL(1, "bad magic");
    if (rd(&r) != 1) FAIL(1, "bad version");
    uint32_t log_n = rd(&r), a = rd(&r), b = rd(&r);
    if (r.bad || log_n < 1 || log_n + B > 31) FAIL(1, "bad log_n");
    uint32_t le = log_n + B;
    uint64_t N = 1ull << le;
    if (a >= P || b >= P) FAIL(2, "public inputs out of M31 range");
    uint32_t troot[8], qroot[8];
    for (int i = 0; i < 8; i++) troot[i] = rd(&r);
    for (int i = 0; i < 8; i++) qroot[i] = rd(&r);
    nfri = rd(&r);
    if (r.bad || nfri > 64) FAIL(1, "bad fri count");
    froots = (uint32_t *)malloc((size_t)nfri * 32 + 4);
    for (uint32_t i = 0; i < 8 * nfri; i++) froots[i] = rd(&r);
    uint32_t nlast = rd(&r);
    if (r.bad || nlast > 64) FAIL(1, "bad last layer count");
    uint32_t last[256];
    for (uint32_t i = 0; i < 4 * nlast; i++) last[i] = rd(&r);
    uint32_t nqp = rd(&r);
    if (r.bad || nqp > (1u << 20)) FAIL(1, "bad query count");
    qi = (uint64_t *)malloc(sizeof(uint64_t) * (nqp + 1));
    for (uint32_t j = 0; j < nqp; j++) qi[j] = rd(&r);
    if (nqp != nq) FAIL(3, "expected %u queries, got %u", nq, nqp);
    if (!read_decom(&r, &td, 1, le)) FAIL(1, "truncated trace decommitment");
    if (!read_decom(&r, &qd, 4, le)) FAIL(1, "truncated quotient decommitment");
    nfd = rd(&r);
    if (r.bad || nfd != nfri) FAIL(1, "bad fri decommitment count");
    fd = (decom_t *)calloc(nfd + 1, sizeof(decom_t));
    for (uint32_t k = 0; k < nfd; k++)
        if (!read_decom(&r, &fd[k], 4, le - 1 - k)) FAIL(1, "truncated fri decommitment %u", k);
    if (r.off != len) FAIL(1, "trailing bytes");

    /* replay transcript — verifier.rs:56-96 */
    vxo_channel ch; vxo_channel_init(&ch);
    vxo_channel_mix_digest(&ch, troot);
    uint32_t tmp[4]; vxo_channel_draw_felt(&ch, tmp);
    vxo_channel_mix_digest(&ch, qroot);
    fal = (uint32_t *)malloc(((size_t)nfri + 1) * 16);
    vxo_channel_draw_felt(&ch, fal);
    for (uint32_t k = 0; k < nfri; k++) { vxo_channel_mix_digest(&ch, froots + 8 * k); vxo_channel_draw_felt(&ch, fal + 4 * (k + 1)); }
    if (nfri != le - 3) FAIL(4, "expected %u FRI layers, got %u", le - 3, nfri);
    if (nlast != 8) FAIL(4, "expected 8 last-layer values, got %u", nlast);
    vxo_channel_mix_felts(&ch, last, nlast);
    for (uint32_t j = 0; j < nq; j++) if (vxo_channel_draw_number(&ch, N) != qi[j]) FAIL(5, "query indices don't match Fiat-Shamir derivation");
    static const uint32_t Z[8] = {0};
    if (!memcmp(troot, Z, 32)) FAIL(6, "trace commitment is zero");
    if (!memcmp(qroot, Z, 32)) FAIL(6, "quotient commitment is zero");
    if (!check_decom(&td, troot, qi, 1, le, nq)) FAIL(7, "trace auth path invalid");
    if (!check_decom(&qd, qroot, qi, 4, le, nq)) FAIL(7, "quotient auth path invalid");
    fi = (uint64_t *)malloc(sizeof(uint64_t) * (nq + 1));
    for (uint32_t j = 0; j < nq; j++) fi[j] = qi[j] >> 1;
    for (uint32_t k = 0; k < nfd; k++) {
        if (!check_decom(&fd[k], froots + 8 * k, fi, 4, le - 1 - k, nq)) FAIL(7, "FRI layer %u auth path invalid", k);
        for (uint32_t j = 0; j < nq; j++) fi[j] >>= 1;
    }
    /* fold equations — verifier.rs:153-233 */
    for (uint32_t j = 0; j < nq; j++) {
        uint64_t ci = qi[j];
        uint32_t cl = le;
        vxo_coset dom = eval_domain(cl);
        qm v, s, f0, f1, al, exp, act;
        memcpy(v.v, qd.vals + 4 * j, 16); memcpy(s.v, qd.svals + 4 * j, 16);
        if (ci & 1) { f0 = s; f1 = v; } else { f0 = v; f1 = s; }
        memcpy(al.v, fal, 16);
        exp = fold_pair(f0, f1, al, fold_tw_at(&dom, ci >> 1, 1));
        memcpy(act.v, fd[0].vals + 4 * j, 16);
        if (memcmp(exp.v, act.v, 16)) FAIL(8, "circle fold mismatch at query %u", j);
        ci >>= 1; cl--;
        for (uint32_t k = 0; k + 1 < nfd; k++) {
            vxo_coset ld = vxo_coset_half_odds(cl);
            memcpy(v.v, fd[k].vals + 4 * j, 16); memcpy(s.v, fd[k].svals + 4 * j, 16);
            if (ci & 1) { f0 = s; f1 = v; } else { f0 = v; f1 = s; }
            memcpy(al.v, fal + 4 * (k + 1), 16);
            exp = fold_pair(f0, f1, al, fold_tw_at(&ld, ci >> 1, 0));
            memcpy(act.v, fd[k + 1].vals + 4 * j, 16);
            if (memcmp(exp.v, act.v, 16)) FAIL(8, "line fold mismatch at query %u layer %u", j, k);
            ci >>= 1; cl--;
        }
        if (nfd > 0) {
            if (ci >= nlast) FAIL(9, "last layer index out of bounds");
            if (memcmp(fd[nfd - 1].vals + 4 * j, last + 4 * ci, 16)) FAIL(9, "last layer mismatch at query %u", j);
        }
    }
done:
    free_decom(&td); free_decom(&qd);
    if (fd) { for (uint32_t k = 0; k < nfd; k++) free_decom(&fd[k]); free(fd); }
    free(froots); free(fal); free(qi); free(fi);
    return rc;
}

/* ------------------------------------------------------------------ */
/* stwo-format NTT: ntt.rs:300-379, circle_ntt_stwo.cu:15-404          */
/* ------------------------------------------------------------------ */
void vxo_stwo_twiddles(uint32_t log_n, int inverse, uint32_t *out) {
    /* StwoNttCache::new (ntt.rs:300-341): levels of half_odds(log_n - 1),
     * x-coordinates of each level's first half in bit-reversed order, the
     * coset doubled between levels, then a 1; 2^(log_n-1) words. */
    uint64_t tc = 1ull << (log_n - 1), w = 0;
    vxo_coset cur = vxo_coset_half_odds(log_n - 1);
    uint32_t levels = cur.log_size;
    for (uint32_t lv = 0; lv < levels; lv++) {
        uint64_t half = (1ull << cur.log_size) / 2;
        uint32_t ll = 0;
        while ((1ull << ll) < half) ll++;
        vxo_point pt = cur.initial;
        for (uint64_t j = 0; j < half; j++) {
            uint64_t bj = ll ? brev(j, ll) : 0;
            out[w + bj] = pt.x;
            pt = vxo_point_mul(pt, cur.step);
        }
        w += half;
        cur.initial = vxo_point_mul(cur.initial, cur.initial);
        cur.step = vxo_point_mul(cur.step, cur.step);
        cur.log_size--;
    }
    if (w < tc) out[w++] = 1u;
    while (w < tc) out[w++] = 0u;
    if (inverse) vxo_batch_inverse(out, out, (size_t)tc);
}

/* one butterfly layer of the stwo kernels (circle_ntt_stwo.cu:31-57) */
static void stwo_line_layer(uint32_t *d, const uint32_t *tw, uint32_t layer_idx, uint64_t half_n, int fwd) {
    #pragma omp parallel for schedule(static)
    for (int64_t tid = 0; tid < (int64_t)half_n; tid++) {
        uint64_t stride = 1ull << layer_idx, h = (uint64_t)tid >> layer_idx;
        uint64_t i0 = (h << (layer_idx + 1)) + ((uint64_t)tid & (stride - 1)), i1 = i0 + stride;
        uint32_t v0 = d[i0], v1 = d[i1], t = tw[h];
        if (fwd) { uint32_t x = m_mul(v1, t); d[i1] = m_sub(v0, x); d[i0] = m_add(v0, x); }
        else { d[i0] = m_add(v0, v1); d[i1] = m_mul(m_sub(v0, v1), t); }
    }
}
/* circle layer: twiddle [y, -y, -x, x][tid % 4] of the pair
 * (x, y) = (tw[2 (tid / 4)], tw[2 (tid / 4) + 1]) (circle_ntt_stwo.cu:202-249) */
static void stwo_circle_layer(uint32_t *d, const uint32_t *tw, uint64_t half_n, int fwd) {
    #pragma omp parallel for schedule(static)
    for (int64_t tid = 0; tid < (int64_t)half_n; tid++) {
        uint64_t pr = (uint64_t)tid / 4;
        uint32_t x = tw[2 * pr], y = tw[2 * pr + 1], t;
        switch (tid % 4) { case 0: t = y; break; case 1: t = m_neg(y); break; case 2: t = m_neg(x); break; default: t = x; }
        uint32_t v0 = d[2 * tid], v1 = d[2 * tid + 1];
        if (fwd) { uint32_t x2 = m_mul(v1, t); d[2 * tid + 1] = m_sub(v0, x2); d[2 * tid] = m_add(v0, x2); }
        else { d[2 * tid] = m_add(v0, v1); d[2 * tid + 1] = m_mul(m_sub(v0, v1), t); }
    }
}
void vxo_stwo_ntt_evaluate(uint32_t *d, const uint32_t *tw, uint32_t log_n) {
    uint64_t half_n = 1ull << (log_n - 1);
    uint32_t nl = log_n - 1;
    for (int k = (int)nl - 1; k >= 0; k--)
        stwo_line_layer(d, tw + (half_n - (1ull << (nl - (uint32_t)k))), (uint32_t)k + 1, half_n, 1);
    stwo_circle_layer(d, tw, half_n, 1);
}
void vxo_stwo_ntt_interpolate(uint32_t *d, const uint32_t *itw, uint32_t log_n) {
    uint64_t half_n = 1ull << (log_n - 1), n = 1ull << log_n;
    uint32_t nl = log_n - 1;
    stwo_circle_layer(d, itw, half_n, 0);
    for (uint32_t k = 0; k < nl; k++) stwo_line_layer(d, itw + (half_n - (1ull << (nl - k))), k + 1, half_n, 0);
    uint32_t e = (30u * log_n) % 31u, s = e ? (1u << e) : 1u;
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; i++) d[i] = m_mul(d[i], s);
}

void vxo_bit_reverse_qm31(const uint32_t *in, uint32_t *out, uint32_t log_n) {
    uint64_t n = 1ull << log_n;
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; i++) {
        uint64_t j = brev((uint64_t)i, log_n);
        for (int c = 0; c < 4; c++) out[4 * j + c] = in[4 * i + c];
    }
}
void vxo_accumulate_lift(uint32_t *col, const uint32_t *curr, uint64_t col_n, uint32_t log_ratio) {
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)col_n; i++) {
        uint64_t src = (((uint64_t)i >> (log_ratio + 1)) << 1) | ((uint64_t)i & 1);
        col[i] = m_add(col[i], curr[src]);
    }
}
void vxo_pack_leaves(const uint32_t *const in[4], uint32_t *const out[64], uint64_t n) {
    for (uint32_t c = 0; c < 4; c++)
        for (uint64_t i = 0; i < n; i++) out[c * 16 + (i % 16)][i / 16] = in[c][i];
}

/* CircleDomain(half_odds(log-1)).at(k): the half coset for k < n/2, its
 * conjugate after (ntt.rs:539, 585) */
static vxo_point stwo_domain_at(uint32_t log, uint64_t k) {
    vxo_coset hc = vxo_coset_half_odds(log - 1);
    uint64_t half = 1ull << (log - 1);
    if (k < half) return vxo_coset_at(&hc, k);
    vxo_point p = vxo_coset_at(&hc, k - half);
    p.y = m_neg(p.y);
    return p;
}
void vxo_stwo_fold_circle_twiddles(uint32_t log, uint32_t *out) {
    /* fri_ops.rs:44-66: 1 / y(domain.at(bit_reverse_index(i << 1, log))) */
    int64_t half = (int64_t)1 << (log - 1);
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < half; i++) out[i] = vxo_m31_inv(stwo_domain_at(log, brev((uint64_t)i << 1, log)).y);
}

/* ------------------------------------------------------------------ */
/* Batched lifted commitment ("LIFT" v1): stwo-format LDE of every     */
/* column, one lifted tree, a random QM31 combination of the lifted    */
/* columns, FRI with stwo twiddles, queries by draw_query_indices.     */
/* ------------------------------------------------------------------ */
static int lifted_check(const uint32_t *logs, uint32_t n_cols, uint32_t B, uint32_t nq) {
    if (n_cols < 1 || n_cols > 64 || B < 1 || B > 4 || nq < 1 || nq > 1024) return 0;
    for (uint32_t c = 0; c < n_cols; c++) {
        if (logs[c] < 2 || logs[c] + B > 28) return 0;
        if (c && logs[c] < logs[c - 1]) return 0;
    }
    return logs[n_cols - 1] + B >= 4;
}
size_t vxo_lifted_size(uint32_t n_cols, const uint32_t *logs, uint32_t B, uint32_t nq) {
    if (!lifted_check(logs, n_cols, B, nq)) return 0;
    uint32_t S = logs[n_cols - 1] + B, nfri = S - 3;
    size_t w = 5 + n_cols + 8 + 8 + 1 + 8 * (size_t)nfri + 1 + 32 + 1 + nq;
    w += 1 + 2 * (size_t)nq * n_cols + 2 * (size_t)nq * (1 + 8 * (size_t)S);
    w += 1 + 2 * (size_t)nq * 4 + 2 * (size_t)nq * (1 + 8 * (size_t)S);
    w += 1;
    for (uint32_t k = 0; k < nfri; k++) w += 1 + 2 * (size_t)nq * 4 + 2 * (size_t)nq * (1 + 8 * (size_t)(S - 1 - k));
    return 4 * w;
}
static inline uint64_t lift_row(uint64_t idx, uint32_t S, uint32_t L) {
    return L == S ? idx : (((idx >> (S - L + 1)) << 1) | (idx & 1));
}
static void tree_from_leaves(vxo_tree *t, uint32_t *leaves, uint32_t log_n) {
    t->log_n = log_n;
    t->levels = (uint32_t **)calloc(log_n + 1, sizeof(uint32_t *));
    t->levels[0] = leaves;
    for (uint32_t l = 1; l <= log_n; l++) {
        uint64_t m = (1ull << log_n) >> l;
        uint32_t *up = (uint32_t *)malloc(m * 32), *dn = t->levels[l - 1];
        #pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < (int64_t)m; i++) vxo_hash_pair(dn + 16 * i, dn + 16 * i + 8, up + 8 * i);
        t->levels[l] = up;
    }
}
static int lifted_impl(const uint32_t *const *cols, const uint32_t *logs, uint32_t n_cols, uint32_t B,
                       uint32_t nq, uint8_t **out, size_t *out_len, uint32_t **lde_out) {
    if (!lifted_check(logs, n_cols, B, nq)) return 1;
    const uint32_t S = logs[n_cols - 1] + B, nfri = S - 3;
    const uint64_t NS = 1ull << S;
    /* 1. LDE of every column: stwo interpolate at 2^L, zero pad, stwo evaluate at 2^(L+B) */
    uint32_t **lde = (uint32_t **)calloc(n_cols, sizeof(uint32_t *));
    uint32_t *lde_logs = (uint32_t *)malloc(n_cols * 4);
    for (uint32_t c = 0; c < n_cols; c++) {
        uint32_t L = logs[c], LE = L + B;
        lde_logs[c] = LE;
        lde[c] = (uint32_t *)calloc(1ull << LE, 4);
        memcpy(lde[c], cols[c], (1ull << L) * 4);
        uint32_t *itw = (uint32_t *)malloc((1ull << (L - 1)) * 4);
        vxo_stwo_twiddles(L, 1, itw);
        vxo_stwo_ntt_interpolate(lde[c], itw, L);
        free(itw);
        uint32_t *tw = (uint32_t *)malloc((1ull << (LE - 1)) * 4);
        vxo_stwo_twiddles(LE, 0, tw);
        vxo_stwo_ntt_evaluate(lde[c], tw, LE);
        free(tw);
    }
    /* 2. lifted tree */
    uint32_t *leaves = (uint32_t *)malloc(NS * 32);
    vxo_lifted_leaves((const uint32_t *const *)lde, lde_logs, n_cols, S, leaves);
    vxo_tree t0;
    tree_from_leaves(&t0, leaves, S);
    uint32_t r0[8]; vxo_tree_root(&t0, r0);
    vxo_channel ch; vxo_channel_init(&ch);
    vxo_channel_mix_digest(&ch, r0);
    uint32_t alpha[4]; vxo_channel_draw_felt(&ch, alpha);
    /* 3. C = sum_c alpha^c * lift(lde_c) */
    qm pw[64];
    pw[0].v[0] = 1; pw[0].v[1] = pw[0].v[2] = pw[0].v[3] = 0;
    qm al; memcpy(al.v, alpha, 16);
    for (uint32_t c = 1; c < n_cols; c++) pw[c] = q_mul(pw[c - 1], al);
    uint32_t *C[4];
    for (int k = 0; k < 4; k++) C[k] = (uint32_t *)malloc(NS * 4);
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)NS; i++) {
        qm acc = {{0, 0, 0, 0}};
        for (uint32_t c = 0; c < n_cols; c++) acc = q_add(acc, q_mulm(pw[c], lde[c][lift_row((uint64_t)i, S, lde_logs[c])]));
        for (int k = 0; k < 4; k++) C[k][i] = acc.v[k];
    }
    vxo_tree t1;
    vxo_tree_build(&t1, (const uint32_t *const *)C, 4, S);
    uint32_t r1[8]; vxo_tree_root(&t1, r1);
    vxo_channel_mix_digest(&ch, r1);
    /* 4. FRI: circle fold with the stwo twiddles, then line folds (fri_ops.rs) */
    uint32_t **lay = (uint32_t **)calloc((size_t)nfri * 4, sizeof(uint32_t *));
    vxo_tree *ft = (vxo_tree *)calloc(nfri, sizeof(vxo_tree));
    uint32_t *froots = (uint32_t *)malloc((size_t)nfri * 32);
    uint32_t fa[4], fa2[4];
    vxo_channel_draw_felt(&ch, fa);
    vxo_qm31_mul(fa, fa, fa2);
    uint32_t *tw = (uint32_t *)malloc((NS / 2) * 4);
    vxo_stwo_fold_circle_twiddles(S, tw);
    for (int k = 0; k < 4; k++) lay[k] = (uint32_t *)calloc(NS / 2, 4);
    vxo_fold_circle_into_line(lay, (const uint32_t *const *)C, tw, fa, fa2, NS / 2);
    uint32_t cur = S - 1;
    vxo_tree_build(&ft[0], (const uint32_t *const *)lay, 4, cur);
    vxo_tree_root(&ft[0], froots);
    vxo_channel_mix_digest(&ch, froots);
    for (uint32_t k = 1; k < nfri; k++) {
        uint32_t a2[4]; vxo_channel_draw_felt(&ch, a2);
        vxo_coset dom = vxo_coset_half_odds(cur);
        uint64_t half = 1ull << (cur - 1);
        vxo_fold_twiddles(&dom, 0, tw);
        for (int c = 0; c < 4; c++) lay[4 * k + c] = (uint32_t *)malloc(half * 4);
        vxo_fold_line((const uint32_t *const *)(lay + 4 * (k - 1)), tw, a2, lay + 4 * k, half);
        cur--;
        vxo_tree_build(&ft[k], (const uint32_t *const *)(lay + 4 * k), 4, cur);
        vxo_tree_root(&ft[k], froots + 8 * k);
        vxo_channel_mix_digest(&ch, froots + 8 * k);
    }
    free(tw);
    uint32_t last[32];
    for (int i = 0; i < 8; i++) for (int c = 0; c < 4; c++) last[4 * i + c] = lay[4 * (nfri - 1) + c][i];
    vxo_channel_mix_felts(&ch, last, 8);
    uint32_t *qi = (uint32_t *)malloc(4 * (size_t)nq);
    vxo_channel_draw_query_indices(&ch, S, nq, qi);
    /* 5. bytes */
    if (out) {
        wbuf w = {NULL, 0, 0};
        w.cap = vxo_lifted_size(n_cols, logs, B, nq); w.p = (uint8_t *)malloc(w.cap);
        wr(&w, 0x5446494Cu); wr(&w, 1); wr(&w, n_cols); wr(&w, B); wr(&w, S);
        wrs(&w, logs, n_cols);
        wrs(&w, r0, 8); wrs(&w, r1, 8);
        wr(&w, nfri); wrs(&w, froots, 8 * (size_t)nfri);
        wr(&w, 8); wrs(&w, last, 32);
        wr(&w, nq); wrs(&w, qi, nq);
        uint64_t *idx = (uint64_t *)malloc(8 * (size_t)nq);
        for (uint32_t j = 0; j < nq; j++) idx[j] = qi[j];
        /* lifted tree: the row of every column at q and at q ^ 1, then paths */
        wr(&w, nq);
        for (int s = 0; s < 2; s++)
            for (uint32_t j = 0; j < nq; j++)
                for (uint32_t c = 0; c < n_cols; c++) wr(&w, lde[c][lift_row(idx[j] ^ (uint64_t)s, S, lde_logs[c])]);
        uint32_t *path = (uint32_t *)malloc(((size_t)S + 1) * 32);
        for (int s = 0; s < 2; s++)
            for (uint32_t j = 0; j < nq; j++) {
                vxo_tree_path(&t0, idx[j] ^ (uint64_t)s, path);
                wr(&w, S);
                wrs(&w, path, 8 * (size_t)S);
            }
        free(path);
        write_decom(&w, &t1, (const uint32_t *const *)C, 4, idx, nq);
        wr(&w, nfri);
        for (uint32_t j = 0; j < nq; j++) idx[j] >>= 1;
        for (uint32_t k = 0; k < nfri; k++) {
            write_decom(&w, &ft[k], (const uint32_t *const *)(lay + 4 * k), 4, idx, nq);
            for (uint32_t j = 0; j < nq; j++) idx[j] >>= 1;
        }
        free(idx);
        *out = w.p; *out_len = w.n;
    }
    free(qi);
    for (uint32_t k = 0; k < nfri; k++) { vxo_tree_free(&ft[k]); for (int c = 0; c < 4; c++) free(lay[4 * k + c]); }
    free(ft); free(lay); free(froots);
    vxo_tree_free(&t1); for (int k = 0; k < 4; k++) free(C[k]);
    vxo_tree_free(&t0);
    if (lde_out) for (uint32_t c = 0; c < n_cols; c++) lde_out[c] = lde[c];
    else for (uint32_t c = 0; c < n_cols; c++) free(lde[c]);
    free(lde); free(lde_logs);
    return 0;
}
int vxo_commit_lifted(const uint32_t *const *cols, const uint32_t *log_sizes, uint32_t n_cols, uint32_t blowup,
                      uint32_t n_queries, uint8_t **out, size_t *out_len) {
    return lifted_impl(cols, log_sizes, n_cols, blowup, n_queries, out, out_len, NULL);
}
int vxo_lifted_lde(const uint32_t *const *cols, const uint32_t *log_sizes, uint32_t n_cols, uint32_t blowup,
                   uint32_t **lde_out) {
    return lifted_impl(cols, log_sizes, n_cols, blowup, 1, NULL, NULL, lde_out);
}

/* ------------------------------------------------------------------ */
/* proof of work: channel.rs:140-168, grind.cu:26-90, grind_ops.rs     */
/* ------------------------------------------------------------------ */
void vxo_pow_prefix(const uint32_t state[8], uint32_t pow_bits, uint32_t out[8]) {
    uint8_t in[52];
    memset(in, 0, sizeof(in));
    st32(in, 0x12345678u);
    for (int i = 0; i < 8; i++) st32(in + 16 + 4 * i, state[i]);
    st32(in + 48, pow_bits);
    uint8_t dg[32];
    vxo_blake2s(in, 52, dg);
    for (int i = 0; i < 8; i++) out[i] = ld32(dg + 4 * i);
}
static uint32_t pow_tz(const uint32_t prefix[8], uint64_t nonce, int m31) {
    uint32_t m[16] = {0}, h[8];
    for (int i = 0; i < 8; i++) m[i] = prefix[i];
    m[8] = (uint32_t)nonce;
    m[9] = (uint32_t)(nonce >> 32);
    for (int i = 0; i < 8; i++) h[i] = IV[i];
    h[0] ^= 0x01010020u;
    vxo_blake2s_compress_words(h, m, 40, 0xFFFFFFFFu);
    uint32_t w[4];
    for (int i = 0; i < 4; i++) w[i] = m31 ? m_red((uint64_t)h[i]) : h[i];
    for (int i = 0; i < 4; i++)
        if (w[i]) return 32u * (uint32_t)i + (uint32_t)__builtin_ctz(w[i]);
    return 128u;
}
int vxo_verify_pow_nonce(const uint32_t prefix[8], uint32_t pow_bits, uint64_t nonce, int m31) {
    return pow_tz(prefix, nonce, m31) >= pow_bits;
}
int vxo_grind_pow(const uint32_t prefix[8], uint32_t pow_bits, int m31, uint32_t max_batches, uint64_t *nonce) {
    if (pow_bits == 0) { *nonce = 0; return 0; }
    for (uint64_t hi = 0; hi < max_batches; hi++) {
        /* each thread scans one contiguous run of lows in order: its first hit
         * is its smallest, and the smallest over threads is the batch's */
        int64_t found = -1;
        #pragma omp parallel if (pow_bits > 8)
        {
            int64_t mine = -1;
            #pragma omp for schedule(static)
            for (int64_t low = 0; low < (int64_t)(1 << 20); low++) {
                if (mine >= 0) continue;
                if (pow_tz(prefix, (hi << 32) | (uint64_t)low, m31) >= pow_bits) mine = low;
            }
            #pragma omp critical
            { if (mine >= 0 && (found < 0 || mine < found)) found = mine; }
        }
        if (found >= 0) { *nonce = (hi << 32) | (uint64_t)found; return 0; }
    }
    return 1;
}

/* ------------------------------------------------------------------ */
/* FRI chain of a QM31 codeword with per-layer commitments: the FRI    */
/* item of the log_n = 24 configuration, composed from the pieces of   */
/* the proof's FRI (prover.rs:860-926, fri.rs:163-224):                */
/*  alpha_0 = draw_felt(state); layer 0 = circle fold of the codeword  */
/*  on half_coset(L) (dst zero); then for k >= 1: mix(root_{k-1}),     */
/*  alpha_k = draw_felt, layer k = line fold of layer k-1 with the     */
/*  half_odds(l) twiddles; every layer committed as a 4-word-leaf tree  */
/*  (the last, of 2 values, too) and its root mixed.                   */
/* ------------------------------------------------------------------ */
void vxo_fri_chain(const uint32_t *const src[4], uint32_t log_size, const uint32_t state[8], uint32_t *roots,
                   uint32_t *alphas, uint32_t last[8]) {
    const uint32_t L = log_size, nl = L - 1;
    vxo_channel ch;
    for (int i = 0; i < 8; i++) st32(ch.state + 4 * i, state[i]);
    ch.n_draws = 0;
    uint64_t m = 1ull << (L - 1);
    uint32_t *cur[4], *nxt[4];
    for (int c = 0; c < 4; c++) {
        cur[c] = (uint32_t *)calloc(m, 4);
        nxt[c] = (uint32_t *)calloc(m / 2 ? m / 2 : 1, 4);
    }
    uint32_t *tw = (uint32_t *)malloc(m * 4);
    vxo_coset dom = vxo_coset_half_coset(L);
    vxo_fold_twiddles(&dom, 1, tw);
    static const uint32_t zero4[4] = {0, 0, 0, 0};
    vxo_channel_draw_felt(&ch, alphas);
    vxo_fold_circle_into_line(cur, src, tw, alphas, zero4, m);
    vxo_merkle_root((const uint32_t *const *)cur, 4, L - 1, roots);
    vxo_channel_mix_digest(&ch, roots);
    for (uint32_t k = 1; k < nl; k++) {
        const uint32_t l = L - k;  /* log size of the layer being folded */
        const uint64_t half = 1ull << (l - 1);
        vxo_channel_draw_felt(&ch, alphas + 4 * k);
        vxo_coset od = vxo_coset_half_odds(l);
        vxo_fold_twiddles(&od, 0, tw);
        vxo_fold_line((const uint32_t *const *)cur, tw, alphas + 4 * k, nxt, half);
        vxo_merkle_root((const uint32_t *const *)nxt, 4, l - 1, roots + 8 * k);
        vxo_channel_mix_digest(&ch, roots + 8 * k);
        for (int c = 0; c < 4; c++) { uint32_t *t = cur[c]; cur[c] = nxt[c]; nxt[c] = t; }
    }
    for (int i = 0; i < 2; i++)
        for (int c = 0; c < 4; c++) last[4 * i + c] = cur[c][i];
    for (int c = 0; c < 4; c++) { free(cur[c]); free(nxt[c]); }
    free(tw);
}

/* ------------------------------------------------------------------ */
/* PolyOps on the device path of the stwo backend                      */
/* ------------------------------------------------------------------ */
/* eval_at_point by folding, level by level (circle_ntt.cu:186-231,
 * 429-468): level 0 combines v[t] + f_0 v[t + n/2] with the coefficients as
 * QM31 of one M31 word; level l uses factor l on the half-length result. */
void vxo_eval_at_point(const uint32_t *coeffs, const uint32_t *factors, uint32_t log_n, uint32_t out[4]) {
    const uint64_t n = 1ull << log_n;
    qm *v = (qm *)malloc(sizeof(qm) * (n ? n : 1));
    for (uint64_t i = 0; i < n; i++) { v[i].v[0] = coeffs[i]; v[i].v[1] = v[i].v[2] = v[i].v[3] = 0; }
    uint64_t cur = n;
    for (uint32_t l = 0; l < log_n; l++) {
        qm f; memcpy(f.v, factors + 4 * l, 16);
        const uint64_t half = cur / 2;
        for (uint64_t t = 0; t < half; t++) v[t] = q_add(v[t], q_mul(v[t + half], f));
        cur = half;
    }
    memcpy(out, v[0].v, 16);
    free(v);
}
/* barycentric_eval_kernel partial sums (barycentric_eval.cu:44-94): block b of
 * a grid-stride loop over n_blocks x 256 threads. */
void vxo_barycentric_partials(const uint32_t *evals, const uint32_t *weights, uint32_t n, uint32_t n_blocks,
                              uint32_t *out) {
    memset(out, 0, 16ull * n_blocks);
    const uint64_t stride = 256ull * n_blocks;
    for (uint64_t i = 0; i < n; i++) {
        const uint64_t b = (i % stride) / 256;
        qm w; memcpy(w.v, weights + 4 * i, 16);
        qm acc; memcpy(acc.v, out + 4 * b, 16);
        acc = q_add(acc, q_mulm(w, evals[i]));
        memcpy(out + 4 * b, acc.v, 16);
    }
}
