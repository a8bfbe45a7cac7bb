"""Shapes of the synthetic benchmark workloads (no data, no device work).

The reference publishes no benchmark inputs, so its benchmark configurations
are restated as seeded synthetic shapes; ``bench.py`` and the GPU tests draw
them from here so both run the same grids.
"""

from __future__ import annotations

from typing import List, Tuple


def smooth_lengths(lo: int = 32, hi: int = 256) -> List[int]:
    """The lengths 2^a 3^b 5^c 7^d in [lo, hi], ascending (55 numbers for [32, 256])."""
    out = set()
    p2 = 1
    while p2 <= hi:
        p3 = p2
        while p3 <= hi:
            p5 = p3
            while p5 <= hi:
                p7 = p5
                while p7 <= hi:
                    if p7 >= lo:
                        out.add(p7)
                    p7 *= 7
                p5 *= 5
            p3 *= 3
        p2 *= 2
    return sorted(out)


def ragged_batch(seed: int = 4, count: int = 64, with_extra: int = 16) -> List[Tuple[Tuple[int, int, int], Tuple[int, ...]]]:
    """The ragged batch of 3-D C2C grids: each axis length drawn with numpy
    ``default_rng(seed)`` from ``smooth_lengths(32, 256)``, then ``with_extra``
    distinct grids (25% of 64) chosen to carry an extra dimension of 2.
    Returns ``[(shape, extra_shape), ...]``."""
    import numpy as np
    smooth = smooth_lengths(32, 256)
    rng = np.random.default_rng(seed)
    shapes = [tuple(int(v) for v in rng.choice(smooth, 3)) for _ in range(count)]
    extra = set(int(i) for i in rng.choice(count, with_extra, replace=False))
    return [(s, (2,) if i in extra else ()) for i, s in enumerate(shapes)]
