"""Helpers shared by the parity tests: oracle <-> library buffer conversion."""

import math

import numpy as np

import pencil_oracle as po


def oracle_pencil(p):
    """Oracle Pencil from a pencil_b200.Pencil."""
    return po.Pencil(po.Topology(p.topology.dims), p.global_shape, p.decomposition, p.permutation)


def to_device(arr, dtype):
    import torch
    return torch.from_numpy(np.ascontiguousarray(arr)).to(device="cuda", dtype=dtype)


def to_host(t):
    return t.detach().cpu().numpy()


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.complex128).ravel()
    b = np.asarray(b, dtype=np.complex128).ravel()
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))


def fft_bound(real_dtype_bytes, n_total):
    """rel-L2 tolerance: 1e-6*log2(N) (f32) or 1e-14*log2(N) (f64)."""
    lg = max(1.0, math.log2(max(2, n_total)))
    return (1e-6 if real_dtype_bytes == 4 else 1e-14) * lg


def value_3d_global(shape, extra):
    """Integer encoding of crates/pencil-array/tests/alltoallv_transpose.rs:18-20."""
    idx = np.indices(shape)
    v = idx[0] * 10000 + idx[1] * 100 + idx[2]
    return np.stack([v + 1_000_000 * e for e in range(extra)]).astype(np.int64)
