"""Exact float32 building blocks for the oracle (numpy has no fused multiply-add)."""
from __future__ import annotations

import numpy as np
from scipy.special import erf as _erf64

F32 = np.float32
F64 = np.float64


def f32(x):
    return np.asarray(x, np.float32)


def fma(a, b, c):
    """float32 fused multiply-add a * b + c rounded once.

    The float64 product of two float32 values is exact; the float64 sum can round, and rounding that sum to float32
    is wrong only when it lands exactly on a float32 rounding midpoint while the exact sum does not. That case is
    detected with the TwoSum error term and resolved towards the exact value."""
    a = np.asarray(a, F64)
    b = np.asarray(b, F64)
    c = np.asarray(c, F64)
    p = a * b
    s = p + c
    bb = s - p
    err = (p - (s - bb)) + (c - bb)
    r = s.astype(F32)
    r64 = r.astype(F64)
    # neighbours of r in the direction of s
    up = np.nextafter(r, F32(np.inf)).astype(F64)
    dn = np.nextafter(r, F32(-np.inf)).astype(F64)
    mid_up = 0.5 * (r64 + up)
    mid_dn = 0.5 * (r64 + dn)
    fix_up = (s == mid_up) & (err > 0)     # tie resolved downwards to r, exact value above the midpoint
    fix_dn = (s == mid_dn) & (err < 0)
    r = np.where(fix_up, up.astype(F32), r)
    r = np.where(fix_dn, dn.astype(F32), r)
    return r.astype(F32)


def norm3(v):
    """|v| of float32 3-vectors (..., 3): sqrt(fma(z, z, fma(y, y, x * x)))."""
    v = f32(v)
    x, y, z = v[..., 0], v[..., 1], v[..., 2]
    return np.sqrt(fma(z, z, fma(y, y, x * x))).astype(F32)


def cross3(a, b):
    """float32 cross product, each component fma(a_i, b_j, -(a_j * b_i))."""
    a = f32(a)
    b = f32(b)
    c0 = fma(a[..., 1], b[..., 2], -(a[..., 2] * b[..., 1]))
    c1 = fma(a[..., 2], b[..., 0], -(a[..., 0] * b[..., 2]))
    c2 = fma(a[..., 0], b[..., 1], -(a[..., 1] * b[..., 0]))
    return np.stack([c0, c1, c2], -1).astype(F32)


def dot3_fma(d, e):
    """float32 dot product of (..., 3) with a 3-vector: fma(d2, e2, fma(d1, e1, d0 * e0))."""
    d = f32(d)
    e = f32(e)
    return fma(d[..., 2], e[2], fma(d[..., 1], e[1], d[..., 0] * e[0]))


def dot3_seq(d, e):
    """float32 dot product, sequential products and sums: (d0 e0 + d1 e1) + d2 e2."""
    d = f32(d)
    e = f32(e)
    return ((d[..., 0] * e[0] + d[..., 1] * e[1]) + d[..., 2] * e[2]).astype(F32)


def erf32(x):
    return _erf64(np.asarray(x, F64)).astype(F32)


def exp32(x):
    return np.exp(np.asarray(x, F64)).astype(F32)


def expm1_32(x):
    return np.expm1(np.asarray(x, F64)).astype(F32)


def sum32(x, axis=None):
    """float64 accumulation rounded to float32."""
    return np.asarray(np.sum(np.asarray(x, F64), axis=axis), F64).astype(F32)


def sum64(x, axis=None):
    return np.sum(np.asarray(x, F64), axis=axis)
