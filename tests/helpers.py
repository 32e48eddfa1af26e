"""Shared helpers for the parity tests (inputs, tolerances, device transfer)."""

import numpy as np

try:
    import torch
except ImportError:  # pragma: no cover
    torch = None

# Parity bars (relative max-norm ||x - x_ref||_inf / ||x_ref||_inf).
RTOL = {np.float64: 1e-12, np.float32: 1e-5}


def rel_err(x, ref):
    x = np.asarray(x, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    return float(np.abs(x - ref).max() / max(np.abs(ref).max(), 1e-300))


def rand_coeffs(rng, size, dtype=np.float64):
    """The benchmark distribution: a, c ~ U(-1,1), b = |a|+|c|+U(1,2), d ~ N(0,1)."""
    a = rng.uniform(-1, 1, size)
    c = rng.uniform(-1, 1, size)
    b = np.abs(a) + np.abs(c) + rng.uniform(1, 2, size)
    d = rng.standard_normal(size)
    return [x.astype(dtype) for x in (a, b, c, d)]


def dev(x):
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()
