"""Pure-Python restatement of the Fibonacci commitment path, for small sizes.

TEST INFRASTRUCTURE ONLY.  A second, independently written statement of the
reference's arithmetic used to cross-check the C oracle (vx_oracle.c) and to
generate the committed golden fixtures under tests/golden/.  Hashing uses
Python's hashlib.blake2s (standard Blake2s-256), which is what the reference's
single-block ``blake2s_hash`` (src/channel.rs:216-298) and the ``blake2`` crate
in ``mix_felts`` (src/channel.rs:46-59) compute for the input lengths used.

Twiddles are derived here from their closed form rather than the reference's
extract-and-squash iteration (src/circle.rs:357-435):
  line layer l, index h: x(initial^(2^l) * step^(2^(2l+1) * h))
  circle index h:        y(initial * step^h)
so agreement with the C oracle also checks that derivation.
"""
from __future__ import annotations

import hashlib
import struct

P = (1 << 31) - 1
G = (2, 1268011823)  # src/circle.rs:26-29
IDENT = (1, 0)


def madd(a, b):
    return (a + b) % P


def msub(a, b):
    return (a - b) % P


def mmul(a, b):
    return (a * b) % P


def minv(a):
    return pow(a, P - 2, P)  # 0 -> 0, as M31::inverse (src/field/m31.rs:32-35)


# QM31 = (a0 + a1 i) + (a2 + a3 i) u, u^2 = 2 + i  (src/field/qm31.rs)
def qadd(x, y):
    return tuple((a + b) % P for a, b in zip(x, y))


def qsub(x, y):
    return tuple((a - b) % P for a, b in zip(x, y))


def qmulm(x, s):
    return tuple(a * s % P for a in x)


def qmul(x, y):
    def cmul(a, b):
        return ((a[0] * b[0] - a[1] * b[1]) % P, (a[0] * b[1] + a[1] * b[0]) % P)

    xa, xb, ya, yb = (x[0], x[1]), (x[2], x[3]), (y[0], y[1]), (y[2], y[3])
    ac, bd, ad, bc = cmul(xa, ya), cmul(xb, yb), cmul(xa, yb), cmul(xb, ya)
    bdu = ((2 * bd[0] - bd[1]) % P, (bd[0] + 2 * bd[1]) % P)
    return ((ac[0] + bdu[0]) % P, (ac[1] + bdu[1]) % P, (ad[0] + bc[0]) % P, (ad[1] + bc[1]) % P)


def pmul(p, q):
    return ((p[0] * q[0] - p[1] * q[1]) % P, (p[0] * q[1] + p[1] * q[0]) % P)


def ppow(p, k):
    r = IDENT
    while k:
        if k & 1:
            r = pmul(r, p)
        p = pmul(p, p)
        k >>= 1
    return r


def rep_double(p, n):
    return ppow(p, 1 << n)


def subgroup(k):
    return (IDENT, rep_double(G, 31 - k), k)


def half_coset(k):
    return (rep_double(G, 30 - k), rep_double(G, 31 - k), k)


def half_odds(k):
    return (rep_double(G, max(29 - k, 0)), rep_double(G, 31 - k), k)


def at(cs, i):
    return pmul(cs[0], ppow(cs[1], i))


def brev(i, bits):
    return int(format(i, f"0{bits}b")[::-1], 2) if bits else 0


def fwd_tables(cs):
    init, step, k = cs
    m = 1 << k
    circle = [at(cs, h)[1] for h in range(m // 2)]
    line = []
    for l in range(k - 1):
        a = ppow(init, 1 << l)
        b = ppow(step, 1 << (2 * l + 1))
        line.append([pmul(a, ppow(b, h))[0] for h in range(m >> (l + 1))])
    return line, circle


def chunk_inverse(vals):
    """Element inverses over aligned chunks of 64 with the reference kernel's
    zero handling (cuda/batch_inverse.cu:8-41)."""
    out = []
    for s in range(0, len(vals), 64):
        ch = vals[s:s + 64]
        if ch[0] == 0:
            out.extend([0] * len(ch))
        else:
            out.extend(minv(v) if v else 0 for v in ch)
    return out


def ntt_layer(d, tw, L, fwd):
    n = len(d)
    s = 1 << L
    for tid in range(n // 2):
        h = tid >> L
        i0 = (h << (L + 1)) + (tid & (s - 1))
        i1 = i0 + s
        v0, v1, t = d[i0], d[i1], tw[h]
        if fwd:
            tmp = v1 * t % P
            d[i0], d[i1] = (v0 + tmp) % P, (v0 - tmp) % P
        else:
            d[i0], d[i1] = (v0 + v1) % P, (v0 - v1) * t % P


def evaluate(d, cs):
    line, circle = fwd_tables(cs)
    k = cs[2]
    for L in range(k - 1, 0, -1):
        ntt_layer(d, line[L - 1], L, True)
    ntt_layer(d, circle, 0, True)


def interpolate(d, cs):
    line, circle = fwd_tables(cs)
    k = cs[2]
    flat = [x for layer in line for x in layer]
    iflat = chunk_inverse(flat)
    iline, off = [], 0
    for layer in line:
        iline.append(iflat[off:off + len(layer)])
        off += len(layer)
    ntt_layer(d, chunk_inverse(circle), 0, False)
    for L in range(1, k):
        ntt_layer(d, iline[L - 1], L, False)
    inv_n = minv(1 << k)
    for i in range(len(d)):
        d[i] = d[i] * inv_n % P


def b2s(data: bytes) -> bytes:
    return hashlib.blake2s(data, digest_size=32).digest()


def words(b: bytes):
    return list(struct.unpack(f"<{len(b) // 4}I", b))


def wbytes(ws):
    return struct.pack(f"<{len(ws)}I", *ws)


def leaf(ws):
    return words(b2s(wbytes(ws[:16])))


def node(l, r):
    return words(b2s(wbytes(l) + wbytes(r)))


def tree(rows):
    levels = [[leaf(r) for r in rows]]
    while len(levels[-1]) > 1:
        lv = levels[-1]
        levels.append([node(lv[2 * i], lv[2 * i + 1]) for i in range(len(lv) // 2)])
    return levels


def path(levels, idx):
    out = []
    for lv in levels[:-1]:
        out.append(lv[idx ^ 1])
        idx >>= 1
    return out


class Channel:
    """src/channel.rs:15-185"""

    def __init__(self):
        self.state = bytes(32)
        self.n_draws = 0

    def mix_digest(self, d):
        self.state = b2s(self.state + wbytes(d))
        self.n_draws = 0

    def mix_felts(self, felts):
        self.state = b2s(self.state + b"".join(wbytes(f) for f in felts))
        self.n_draws = 0

    def squeeze(self):
        out = b2s(self.state + struct.pack("<I", self.n_draws) + b"\x00")
        self.n_draws += 1
        return out

    def draw_felt(self):
        while True:
            w = words(self.squeeze())
            if all(x < 2 * P for x in w):
                return tuple(x % P for x in w[:4])

    def draw_number(self, bound):
        return struct.unpack("<Q", self.squeeze()[:8])[0] % bound


def fib_trace(a, b, n):
    t = [a, b]
    while len(t) < n:
        t.append((t[-1] + t[-2]) % P)
    return t[:n]


def fold_tw(cs, circle):
    k = cs[2]
    src = []
    for i in range(1 << (k - 1)):
        p = at(cs, brev(i << 1, k))
        src.append(p[1] if circle else p[0])
    return chunk_inverse(src)


def fold(vals, tw, alpha):
    out = []
    for i in range(len(vals) // 2):
        f0, f1 = vals[2 * i], vals[2 * i + 1]
        out.append(qadd(qadd(f0, f1), qmul(alpha, qmulm(qsub(f0, f1), tw[i]))))
    return out


def prove(a, b, log_n, blowup_bits=2, n_queries=80):
    """src/prover.rs:264-619, serialized as src/bin/stark_cli.rs:1092-1123."""
    le = log_n + blowup_bits
    n, N = 1 << log_n, 1 << le
    d = fib_trace(a, b, n)
    interpolate(d, half_coset(log_n))
    e = d + [0] * (N - n)
    edom = half_coset(le) if le <= 30 else subgroup(le)
    evaluate(e, edom)
    ttree = tree([[v] for v in e])
    troot = ttree[-1][0]
    ch = Channel()
    ch.mix_digest(troot)
    alpha = ch.draw_felt()
    q = []
    for i in range(N):
        c = (e[(i + 2) % N] - (e[(i + 1) % N] + e[i])) % P
        q.append(qmulm(alpha, c))
    qtree = tree([list(v) for v in q])
    qroot = qtree[-1][0]
    ch.mix_digest(qroot)
    fa = ch.draw_felt()
    layers = [fold(q, fold_tw(edom, True), fa)]
    ftrees = [tree([list(v) for v in layers[0]])]
    ch.mix_digest(ftrees[0][-1][0])
    cur = le - 1
    while cur > 3:
        al = ch.draw_felt()
        layers.append(fold(layers[-1], fold_tw(half_odds(cur), False), al))
        cur -= 1
        ftrees.append(tree([list(v) for v in layers[-1]]))
        ch.mix_digest(ftrees[-1][-1][0])
    last = layers[-1]
    ch.mix_felts(last)
    qi = [ch.draw_number(N) for _ in range(n_queries)]

    w = [0x4B52414B, 1, log_n, a, b] + troot + qroot + [len(ftrees)]
    for t in ftrees:
        w += t[-1][0]
    w += [len(last)]
    for v in last:
        w += list(v)
    w += [n_queries] + qi

    def decom(levels, vals, idx):
        out = [len(idx)]
        for i in idx:
            out += list(vals[i])
        for i in idx:
            out += list(vals[i ^ 1])
        for s in (0, 1):
            for i in idx:
                pth = path(levels, i ^ s)
                out.append(len(pth))
                for h in pth:
                    out += h
        return out

    w += decom(ttree, [[v] for v in e], qi)
    w += decom(qtree, q, qi)
    w += [len(ftrees)]
    fi = [i >> 1 for i in qi]
    for t, lay in zip(ftrees, layers):
        w += decom(t, lay, fi)
        fi = [i >> 1 for i in fi]
    return wbytes(w)


def prove_roots(a, b, log_n, blowup_bits=2):
    """Trace, quotient and FRI roots only (same transcript as prove)."""
    blob = prove(a, b, log_n, blowup_bits, n_queries=0)
    w = words(blob)
    tr, qr = w[5:13], w[13:21]
    nf = w[21]
    fr = [w[22 + 8 * k:30 + 8 * k] for k in range(nf)]
    return tr, qr, fr


def last_layer_poly_coeffs(evals):
    """src/fri.rs:276-323: BRT evals on half_odds(log n) -> natural-order
    line-poly coefficients, truncated to 8."""
    n = len(evals)
    log_n = n.bit_length() - 1
    e = [evals[brev(i, log_n)] for i in range(n)]
    chunk, dom_log = n, log_n
    while chunk > 1:
        dom = half_odds(dom_log)
        half = chunk // 2
        for s in range(0, n, chunk):
            for i in range(half):
                xi = minv(at(dom, i)[0])
                l, r = e[s + i], e[s + half + i]
                e[s + i] = qadd(l, r)
                e[s + half + i] = qmulm(qsub(l, r), xi)
        dom_log -= 1
        chunk = half
    ninv = minv(n)
    e = [qmulm(v, ninv) for v in e]
    e = [e[brev(i, log_n)] for i in range(n)]
    return e[:8]


def eval_last_layer_poly(coeffs, last_idx, log_size):
    """src/fri.rs:350-382"""
    dom = half_odds(log_size)
    x = at(dom, brev(last_idx, log_size))[0]
    n = len(coeffs)
    if n == 1:
        return coeffs[0]
    log_c = n.bit_length() - 1
    dbl = []
    xi = x
    for _ in range(log_c):
        dbl.append(xi)
        xi = (2 * xi * xi - 1) % P
    brt = [None] * n
    for i in range(n):
        brt[brev(i, log_c)] = coeffs[i]

    def fe(c, d):
        if len(c) == 1:
            return c[0]
        h = len(c) // 2
        return qadd(fe(c[:h], d[1:]), qmulm(fe(c[h:], d[1:]), d[0]))

    return fe(brt, dbl)
