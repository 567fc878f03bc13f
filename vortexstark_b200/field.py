"""Host-side M31 / CM31 / QM31 arithmetic (src/field/m31.rs, cm31.rs, qm31.rs).

QM31 elements are 4-tuples (a0, a1, a2, a3) = (a0 + a1 i) + (a2 + a3 i) u with
i^2 = -1 and u^2 = 2 + i.  Used for the small host-side quantities of the
protocol (alpha^2 of the circle fold, the verifier's fold checks).
"""
from __future__ import annotations

P = 0x7FFFFFFF


def m31_inv(a: int) -> int:
    """Fermat inverse; 0 -> 0 (m31.rs:32-35)."""
    return pow(a, P - 2, P)


def qm31_add(x, y):
    return tuple((a + b) % P for a, b in zip(x, y))


def qm31_sub(x, y):
    return tuple((a - b) % P for a, b in zip(x, y))


def qm31_mul_m31(x, s: int):
    return tuple(a * s % P for a in x)


def qm31_mul(x, y):
    """(a + b u)(c + d u) = (ac + bd (2 + i)) + (ad + bc) u  (qm31.rs:138-155)"""
    def cm(p, q):
        return ((p[0] * q[0] - p[1] * q[1]) % P, (p[0] * q[1] + p[1] * q[0]) % P)

    xa, xb, ya, yb = (x[0], x[1]), (x[2], x[3]), (y[0], y[1]), (y[2], y[3])
    ac, bd, ad, bc = cm(xa, ya), cm(xb, yb), cm(xa, yb), cm(xb, ya)
    bdu = ((2 * bd[0] - bd[1]) % P, (bd[0] + 2 * bd[1]) % P)
    return ((ac[0] + bdu[0]) % P, (ac[1] + bdu[1]) % P, (ad[0] + bc[0]) % P, (ad[1] + bc[1]) % P)
