"""Shared helpers for the parity tests (inputs, tolerances, device transfer)."""

import numpy as np

try:
    import torch
except ImportError:  # pragma: no cover
    torch = None

# Parity bars (relative max-norm ||x - x_ref||_inf / ||x_ref||_inf).
RTOL = {np.float64: 1e-12, np.float32: 1e-5}


def rel_err(x, ref):
    x, ref = np.asarray(x), np.asarray(ref)
    t = np.complex128 if np.iscomplexobj(x) or np.iscomplexobj(ref) else np.float64
    x, ref = x.astype(t), ref.astype(t)
    return float(np.abs(x - ref).max() / max(np.abs(ref).max(), 1e-300))


def rand_coeffs(rng, size, dtype=np.float64):
    """The benchmark distribution: a, c ~ U(-1,1), b = |a|+|c|+U(1,2), d ~ N(0,1)."""
    a = rng.uniform(-1, 1, size)
    c = rng.uniform(-1, 1, size)
    b = np.abs(a) + np.abs(c) + rng.uniform(1, 2, size)
    d = rng.standard_normal(size)
    return [x.astype(dtype) for x in (a, b, c, d)]


def rand_complex_coeffs(rng, size, dtype=np.complex128):
    """Complex rows diagonally dominant in modulus: a, c with components
    U(-1,1), b = (|a|+|c|+U(1,2)) e^{i phi} with phi ~ U(0, 2 pi), d with
    N(0,1) components."""
    a = rng.uniform(-1, 1, size) + 1j * rng.uniform(-1, 1, size)
    c = rng.uniform(-1, 1, size) + 1j * rng.uniform(-1, 1, size)
    b = (np.abs(a) + np.abs(c) + rng.uniform(1, 2, size)) * np.exp(1j * rng.uniform(0, 2 * np.pi, size))
    d = rng.standard_normal(size) + 1j * rng.standard_normal(size)
    return [x.astype(dtype) for x in (a, b, c, d)]


def dev(x):
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def overlapping_varlen_problem(seed, ngood=600, npairs=400, extra=8192):
    """A variable-length batch whose offsets stop increasing: ngood ordinary
    systems packed in rows [0, G), then npairs of systems alternating between
    [G, G + extra] (valid-looking, every one overlapping the others) and
    [G + extra, G] (decreasing).  The decreasing ones must be flagged (bit 4)
    and skipped, the valid-looking ones must not drive any work table past
    its size (a layout of 256-row block items would need about
    npairs * extra / 256 entries), and the ngood systems must stay solved.
    Returns the FP64 arrays, the offsets and G."""
    rng = np.random.default_rng(seed)
    lens = np.floor(np.exp(rng.uniform(np.log(8), np.log(2048), ngood))).astype(np.int64)
    good = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    G = int(good[-1])
    tail = np.array([G + extra if k % 2 == 0 else G for k in range(2 * npairs)], dtype=np.int64)
    off = np.concatenate([good, tail])
    a, b, c, d = rand_coeffs(rng, G + extra)
    return (a, b, c, d), off, G
