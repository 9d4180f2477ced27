"""Shared helpers of the test suite: seeded inputs, padding, device runs."""

import numpy as np


def make_system(dims, solvedim, dtype=np.float64, seed=0, margin=None):
    """Seeded batch in the reference layout (flat, x fastest).

    a, c ~ U(-0.5, 0.5) with a = 0 on the first and c = 0 on the last row of
    every system along `solvedim`; b = 1 + |a| + |c| + U(0, 1), or, when
    `margin` (array or scalar) is given, b = |a| + |c| + margin; d ~ N(0, 1).
    """
    rng = np.random.default_rng(seed)
    shape = tuple(reversed(dims))  # C-order view: x is the last axis
    a = rng.uniform(-0.5, 0.5, shape)
    c = rng.uniform(-0.5, 0.5, shape)
    ax = len(dims) - 1 - solvedim
    idx0 = [slice(None)] * len(dims)
    idx0[ax] = 0
    a[tuple(idx0)] = 0.0
    idxl = [slice(None)] * len(dims)
    idxl[ax] = -1
    c[tuple(idxl)] = 0.0
    if margin is None:
        b = 1.0 + np.abs(a) + np.abs(c) + rng.uniform(0.0, 1.0, shape)
    else:  # diagonal-dominance margin b - |a| - |c|
        b = np.abs(a) + np.abs(c) + margin
    d = rng.standard_normal(shape)
    out = [np.ascontiguousarray(v.reshape(-1), dtype=dtype) for v in (a, b, c, d)]
    return out


def pad_offset(pads):
    """Offset of element (1,1,...) in a padded array (scalar/test/test_cpu.cpp:109-114)."""
    off = 1
    acc = 1
    for p in pads[:-1]:
        acc *= p
        off += acc
    return off


def padded_index(dims, pads):
    """Index into a padded array (dims = pads) of every element of a compact
    x-fastest array of `dims`, with the interior starting at pad_offset(pads)."""
    strides = [1]
    for p in pads[:-1]:
        strides.append(strides[-1] * p)
    nd = len(dims)
    lin = np.zeros(tuple(reversed(dims)), dtype=np.int64)
    for k, (n, s) in enumerate(zip(dims, strides)):
        shape = [1] * nd
        shape[nd - 1 - k] = n
        lin = lin + (np.arange(n, dtype=np.int64) * s).reshape(shape)
    return lin.reshape(-1) + pad_offset(pads)


def to_padded(x, dims, pads, fill=np.nan):
    """Copy a compact x-fastest array into the interior of a padded one (grown
    past prod(pads) when a dimension has no padding to hold the offset)."""
    idx = padded_index(dims, pads)
    size = max(int(np.prod(pads)), int(idx.max()) + 1 if idx.size else 0)
    full = np.full(size, fill, dtype=x.dtype)
    full[idx] = x
    return full


def from_padded(full, dims, pads):
    return np.ascontiguousarray(full[padded_index(dims, pads)])


def normwise(x, ref):
    x = np.asarray(x, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    den = np.max(np.abs(ref))
    return float(np.max(np.abs(x - ref)) / (den if den > 0 else 1.0))
