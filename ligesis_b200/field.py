"""Scalar Goldilocks / F_{p^2} helpers for host-side bookkeeping (O(k) work such as
`MlPoly::eval_eq`).  Bulk arithmetic always runs in liblgs.so on the GPU."""
from __future__ import annotations

P = 0xFFFFFFFF00000001
W = 7  # EF = F_p[x] / (x^2 - 7)


def add(a: int, b: int) -> int:
    return (a + b) % P


def sub(a: int, b: int) -> int:
    return (a - b) % P


def mul(a: int, b: int) -> int:
    return (a * b) % P


def ef(x) -> tuple[int, int]:
    """Coerce a BF int, an EF pair or a length-2 array to an EF tuple."""
    if isinstance(x, (int,)):
        return (x % P, 0)
    a, b = x
    return (int(a) % P, int(b) % P)


def ef_add(a, b):
    return ((a[0] + b[0]) % P, (a[1] + b[1]) % P)


def ef_sub(a, b):
    return ((a[0] - b[0]) % P, (a[1] - b[1]) % P)


def ef_mul(a, b):
    return ((a[0] * b[0] + W * a[1] * b[1]) % P, (a[0] * b[1] + a[1] * b[0]) % P)


def ef_pow(a, e: int):
    r = (1, 0)
    while e:
        if e & 1:
            r = ef_mul(r, a)
        a = ef_mul(a, a)
        e >>= 1
    return r


def ef_inv(a):
    norm = (a[0] * a[0] - W * a[1] * a[1]) % P
    ni = pow(norm, P - 2, P)
    return (a[0] * ni % P, (-a[1]) * ni % P)


ONE = (1, 0)
ZERO = (0, 0)


def eval_eq(p1, p2):
    """`MlPoly::eval_eq` (utils/src/poly.rs:55-61): prod_i (a_i b_i + (1 - a_i)(1 - b_i))."""
    res = ONE
    for a, b in zip(p1, p2):
        a, b = ef(a), ef(b)
        res = ef_mul(res, ef_add(ef_mul(a, b), ef_mul(ef_sub(ONE, a), ef_sub(ONE, b))))
    return res
