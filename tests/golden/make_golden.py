"""Generate the golden known-answer fixtures from the reference's own tests.

The reference (nogaki/pencil-rs, Rust) cannot be built in this environment
(no cargo/rustc, no MPI, crates not vendored), and its external FFTW fixtures
are generated on the fly by Julia and never checked in.  Its unit and
integration tests pin results with closed-form inputs and O(n^2) direct-sum
oracles instead; this script restates exactly those formulas (each function
names its source) and stores inputs and expected outputs, so the oracle and
the CUDA library are checked against the reference tests' own known answers.

Run ``python tests/golden/make_golden.py`` to regenerate
``tests/golden/reference_known_answers.npz``.  It imports nothing from the
oracle or the product.
"""

from __future__ import annotations

import math
import os

import numpy as np

TAU = 2.0 * math.pi
HERE = os.path.dirname(os.path.abspath(__file__))

KINDS = ("DctI", "DctII", "DctIII", "DctIV", "DstI", "DstII", "DstIII", "DstIV")


def c2c_sample_input(line_len, batches):
    """crates/pencil-fft/src/lib.rs:762-772 (sample_input)."""
    x = np.arange(line_len * batches, dtype=np.float64) + 1.0
    return np.sin(0.37 * x) + 0.07 * x + 1j * (np.cos(0.19 * x) - 0.11 * x)


def dft_direct(values, line_len, sign, scale):
    """crates/pencil-fft/src/lib.rs:774-799 (dft_oracle)."""
    lines = values.reshape(-1, line_len)
    out = np.zeros_like(lines)
    for k in range(line_len):
        acc = np.zeros(lines.shape[0], dtype=np.complex128)
        for j in range(line_len):
            ang = sign * TAU * j * k / line_len
            acc += lines[:, j] * complex(math.cos(ang), math.sin(ang))
        out[:, k] = acc * scale
    return out.reshape(-1)


def r2c_real_input(real_len, batches):
    """crates/pencil-fft/src/r2c.rs:1033-1040 (real_input)."""
    x = np.arange(real_len * batches, dtype=np.float64) + 1.0
    return np.sin(0.31 * x) + 0.09 * x - np.cos(0.11 * x)


def r2r_input(n, batches):
    """crates/pencil-fft/src/r2r.rs:1114-1121 (input)."""
    x = np.arange(n * batches, dtype=np.float64) + 1.0
    return np.sin(0.19 * x) + 0.07 * x + 1j * (np.cos(0.23 * x) - 0.11 * x)


def r2r_direct(kind, line):
    """crates/pencil-fft/src/r2r.rs:1064-1112 (direct)."""
    n = len(line)
    out = np.zeros(n, dtype=np.complex128)
    for k in range(n):
        acc = 0.0 + 0.0j
        for j, v in enumerate(line):
            if kind == "DctI":
                if j == 0 or j == n - 1:
                    c = -1.0 if (j == n - 1 and k % 2 == 1) else 1.0
                else:
                    c = 2.0 * math.cos(math.pi * j * k / (n - 1))
            elif kind == "DctII":
                c = 2.0 * math.cos(math.pi * (j + 0.5) * k / n)
            elif kind == "DctIII":
                c = 1.0 if j == 0 else 2.0 * math.cos(math.pi * j * (k + 0.5) / n)
            elif kind == "DctIV":
                c = 2.0 * math.cos(math.pi * (j + 0.5) * (k + 0.5) / n)
            elif kind == "DstI":
                c = 2.0 * math.sin(math.pi * (j + 1.0) * (k + 1.0) / (n + 1))
            elif kind == "DstII":
                c = 2.0 * math.sin(math.pi * (j + 0.5) * (k + 1.0) / n)
            elif kind == "DstIII":
                if j == n - 1:
                    c = 1.0 if k % 2 == 0 else -1.0
                else:
                    c = 2.0 * math.sin(math.pi * (j + 1.0) * (k + 0.5) / n)
            else:
                c = 2.0 * math.sin(math.pi * (j + 0.5) * (k + 0.5) / n)
            acc += v * c
        out[k] = acc
    return out


def dht_input(line_len, batches):
    """crates/pencil-fft/src/dht.rs:421-428 (input)."""
    x = np.arange(line_len * batches, dtype=np.float64) + 0.37
    return np.cos(0.17 * x) - 0.04 * x + 1j * (np.sin(0.23 * x) + 0.06 * x)


def dht_direct(line):
    """crates/pencil-fft/src/dht.rs:434-449 (direct)."""
    n = len(line)
    out = np.zeros(n, dtype=np.complex128)
    for k in range(n):
        for j, v in enumerate(line):
            ang = TAU * j * k / n
            out[k] += v * (math.cos(ang) + math.sin(ang))
    return out


def input_value(extra, spatial, seed):
    """crates/pencil-fft/tests/distributed_c2c.rs:2853-2874 (input_value)."""
    re = 0.13 + seed * 0.017
    im = -0.27 - seed * 0.011
    for i, v in enumerate(extra):
        re += (i + 2) * (v + 1) * 0.071
        im -= (i + 3) * (v + 1) * 0.043
    for a, v in enumerate(spatial):
        re += (a + 1) * (v + 1) * 0.19 + math.sin(v + 1 + a) * 0.013
        im += (a + 2) * (v + 1) * 0.11 + math.cos(v + 2 + a) * 0.017
    return complex(re, im)


def spectrum_value(extra, wave, seed):
    """crates/pencil-fft/tests/distributed_c2c.rs:2876-2896 (spectrum_value)."""
    re = 0.41 + seed * 0.009
    im = -0.18 - seed * 0.007
    for i, v in enumerate(extra):
        re += (i + 1) * (v + 2) * 0.037
        im += (i + 4) * (v + 1) * 0.029
    for a, v in enumerate(wave):
        re += (a + 2) * (v + 1) * 0.083
        im -= (a + 1) * (v + 2) * 0.047
    return complex(re, im)


def nd_dft(field, inverse, normalize):
    """crates/pencil-fft/tests/distributed_c2c.rs:2813-2851 (dft_value), all targets."""
    shape = field.shape
    idx = np.stack(np.meshgrid(*[np.arange(s) for s in shape], indexing="ij"), -1).reshape(-1, len(shape))
    sign = 1.0 if inverse else -1.0
    flat = field.reshape(-1)
    out = np.zeros(len(idx), dtype=np.complex128)
    for t, target in enumerate(idx):
        phase = sign * TAU * np.sum(idx * target[None, :] / np.array(shape)[None, :], axis=1)
        out[t] = np.sum(flat * (np.cos(phase) + 1j * np.sin(phase)))
    if inverse and normalize:
        out /= flat.size
    return out.reshape(shape)


def main():
    data = {}
    # local C2C, lengths of lib.rs:903-914, three batches
    for n in (1, 2, 3, 4, 5, 7, 8, 9, 11, 12, 13):
        src = c2c_sample_input(n, 3)
        data[f"c2c_in_{n}"] = src
        data[f"c2c_fwd_{n}"] = dft_direct(src, n, -1.0, 1.0)
        data[f"c2c_bwd_{n}"] = dft_direct(src, n, 1.0, 1.0)
    # local R2C: forward = first n/2+1 bins of the DFT of the real input
    for n in (1, 2, 3, 4, 5, 6, 7, 8, 9, 12, 13, 16):
        src = r2c_real_input(n, 3)
        data[f"r2c_in_{n}"] = src
        full = dft_direct(src.astype(np.complex128), n, -1.0, 1.0).reshape(3, n)
        data[f"r2c_fwd_{n}"] = full[:, : n // 2 + 1].reshape(-1)
    # the eight DCT/DST kinds, lengths 1..13, real and complex input
    for kind in KINDS:
        for n in range(1, 14):
            if kind == "DctI" and n == 1:
                continue
            src = r2r_input(n, 2)
            data[f"r2r_in_{kind}_{n}"] = src
            data[f"r2r_out_{kind}_{n}"] = np.concatenate(
                [r2r_direct(kind, src[b * n:(b + 1) * n]) for b in range(2)])
    # (model length, normalisation factor) for n = 1, 2, 5, 8 (r2r.rs:1449-1458)
    table = {
        "DctI": [(0, 0), (2, 2), (8, 8), (14, 14)],
        "DctII": [(4, 2), (8, 4), (20, 10), (32, 16)],
        "DctIII": [(4, 2), (8, 4), (20, 10), (32, 16)],
        "DctIV": [(8, 2), (16, 4), (40, 10), (64, 16)],
        "DstI": [(4, 4), (6, 6), (12, 12), (18, 18)],
        "DstII": [(4, 2), (8, 4), (20, 10), (32, 16)],
        "DstIII": [(4, 2), (8, 4), (20, 10), (32, 16)],
        "DstIV": [(8, 2), (16, 4), (40, 10), (64, 16)],
    }
    data["r2r_table_n"] = np.array([1, 2, 5, 8])
    for kind, rows in table.items():
        data[f"r2r_table_{kind}"] = np.array(rows, dtype=np.int64)
    # DHT, lengths 1..13
    for n in range(1, 14):
        src = dht_input(n, 2)
        data[f"dht_in_{n}"] = src
        data[f"dht_out_{n}"] = np.concatenate([dht_direct(src[b * n:(b + 1) * n]) for b in range(2)])
    # distributed C2C analytic fields (distributed_c2c.rs), shape [4,6,5], extra [2]
    shape = (4, 6, 5)
    seed = 1.0
    for e in range(2):
        fld = np.zeros(shape, dtype=np.complex128)
        spec = np.zeros(shape, dtype=np.complex128)
        for g in np.ndindex(*shape):
            fld[g] = input_value([e], list(g), seed)
            spec[g] = spectrum_value([e], list(g), seed)
        data[f"nd_in_{e}"] = fld
        data[f"nd_fwd_{e}"] = nd_dft(fld, False, False)
        data[f"nd_spec_{e}"] = spec
        data[f"nd_inv_{e}"] = nd_dft(spec, True, True)
        data[f"nd_bwd_{e}"] = nd_dft(spec, True, False)
    path = os.path.join(HERE, "reference_known_answers.npz")
    np.savez_compressed(path, **data)
    print(f"wrote {path} ({len(data)} arrays)")


if __name__ == "__main__":
    main()
