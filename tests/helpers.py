"""Test helpers: per-order comparison and the oracle replay of a case."""
from __future__ import annotations

import numpy as np


def order_slices(N: int):
    """Column slices of each order k = 1..N in a (.., 2 + 18N) series array."""
    return [slice(2 + 18 * (k - 1), 2 + 18 * k) for k in range(1, N + 1)]


def per_order_rel(a: np.ndarray, b: np.ndarray, N: int):
    """max|a-b| / max|b| for every order (b is the checker's value)."""
    a = np.asarray(a).reshape(-1, 2 + 18 * N)
    b = np.asarray(b).reshape(-1, 2 + 18 * N)
    out = []
    for sl in order_slices(N):
        den = np.abs(b[:, sl]).max()
        num = np.abs(a[:, sl] - b[:, sl]).max()
        out.append(num / den if den > 0 else num)
    return np.array(out)


def flag_diff(a: np.ndarray, b: np.ndarray, N: int) -> float:
    a = np.asarray(a).reshape(-1, 2 + 18 * N)
    b = np.asarray(b).reshape(-1, 2 + 18 * N)
    return float(np.abs(a[:, :2] - b[:, :2]).max())


def rel_scale(a, b, scale=None) -> float:
    """max|a-b| relative to max|b| (or to a given scale)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    s = np.abs(b).max() if scale is None else scale
    d = np.abs(a - b).max()
    return float(d / s) if s > 0 else float(d)


def obs_close(a, b, tol, floor=1e-2):
    """Per-order observables (leading axis = order): |a_k - b_k| <= tol * s_k
    with s_k = max(max|b_k|, floor * max|b|).  Orders whose value is tiny
    compared with the leading one -- the order-1 plaquette and all imaginary
    parts vanish in exact arithmetic and carry only rounding noise -- are
    held to an absolute bound of tol * floor * max|b| instead."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    lead = np.abs(b).max()
    worst = 0.0
    for k in range(a.shape[0]):
        s = max(np.abs(b[k]).max(), floor * lead)
        d = np.abs(a[k] - b[k]).max()
        worst = max(worst, d / s if s > 0 else d)
    return worst <= tol, worst
