"""Generates smem_layout.hpp: the shared-memory sequence layout (padding shift
and sequence stride) of the power-of-two and mixed-radix pass kernels, per
line length and precision.

Element i of a sequence sits at s*SEQ + i + (i >> SH) (SH = 0: no padding).
For every candidate (SH, SEQ) this script replays each shared-memory access of
a tile -- the Stockham exchanges, the twiddle reads, the natural-order writes
and the transposed or R2C-split reads of the store, for every pass kind and
store mode (and the real-to-real kernel's), with the kernels' thread mappings
-- warp by warp, and counts wavefronts with the bank model

    wavefronts(access) = sum over phases of max(1 if a lane is active,
                                                max over bank groups of distinct elements)

A phase is 128 bytes of lanes (16 lanes of 8-byte elements, 8 lanes of
16-byte elements); bank group = element mod 16 or mod 8; lanes reading the
same element share it.  This per-phase rule reproduces the shared-memory
wavefronts ncu counts for the register kernel (1280 per 512-point tile, where
balancing bank groups over the whole warp predicts 1024).  The layout with
the fewest wavefronts summed over all kinds wins (the smaller SEQ on a tie).

Run from this directory: ``python gen_smem_layout.py`` (a few minutes).
The thread/sequence mappings replayed here are those of pow2_kernel.cu and
mr_kernel.cuh; a change to either kernel's indexing needs a rerun.
"""

from __future__ import annotations

import os
from multiprocessing import get_context

import numpy as np

THREADS = 256
POW2 = [32, 64, 128, 256, 512, 1024, 2048]
MR = [35, 36, 40, 42, 45, 48, 49, 50, 54, 56, 60, 63, 70, 72, 75, 80, 81, 84, 90, 96, 98, 100, 105, 108, 112, 120,
      125, 126, 135, 140, 144, 147, 150, 160, 162, 168, 175, 180, 189, 192, 196, 200, 210, 216, 224, 225, 240, 243,
      245, 250, 252, 270, 280, 288, 294, 300, 315, 320, 324, 336, 343, 350, 360, 375, 378, 384, 392, 400, 405, 420,
      432, 441, 448, 450, 480, 486, 490, 500, 504, 525, 540, 560, 567, 576, 588, 600, 625, 630, 640, 648, 672,
      675, 686, 700, 720, 729, 735, 750, 756, 768, 784, 800, 810, 840, 864, 875, 882, 896, 900, 945, 960, 972,
      980, 1000, 1008]
# the mixed-radix kernel also runs the real-to-real kinds on powers of two and
# on 770 (mr_lengths.hpp, kMrR2rLengths)
MR_ALL = sorted(MR + [32, 64, 128, 256, 512, 770])
SHIFTS = [0, 2, 3, 4, 5]
KINDS = [("c2c", False), ("r2c", False), ("c2r", False), ("c2c", True), ("r2c", True), ("c2r", True)]


def wavefronts(idx: np.ndarray, E: int) -> int:
    """idx: (M, 32) element indices of M warp accesses, -1 for idle lanes."""
    M = idx.shape[0]
    G = 128 // E
    P = 128 // E  # lanes per phase
    sub = idx.reshape(M * (32 // P), P)
    R = sub.shape[0]
    s = np.sort(sub, axis=1)
    valid = s >= 0
    uniq = valid.copy()
    uniq[:, 1:] &= s[:, 1:] != s[:, :-1]
    cnt = np.zeros((R, G), dtype=np.int64)
    rows = np.broadcast_to(np.arange(R)[:, None], (R, P))
    np.add.at(cnt, (rows[uniq], s[uniq] % G), 1)
    return int(np.maximum(cnt.max(axis=1), valid.any(axis=1)).sum())


def loop_lanes(count: int) -> np.ndarray:
    """Work indices of each warp instruction of ``for (i = tid; i < count; i += 256)``."""
    iters = -(-count // THREADS)
    b = np.arange(iters * THREADS).reshape(-1, 32)
    return np.where(b < count, b, -1)


def padded(i, sh):
    return i if sh == 0 else i + (i >> sh)


# ---------------------------------------------------------------- pow2 kernel
def p2_geom(N, rb):
    T = N // 8
    slots = THREADS // T
    lpt = 2 if (rb == 4 and 64 <= N <= 512) else 1
    return T, slots, lpt, slots * lpt


def p2_cost(N, rb, sh, SEQ, kind, direct):
    E = 2 * rb
    T, slots, lpt, nseq = p2_geom(N, rb)
    log = N.bit_length() - 1
    lead = 8 if log % 3 == 0 else (2 if log % 3 == 1 else 4)
    nst = log // 3 if log % 3 == 0 else log // 3 + 1
    tid = np.arange(THREADS).reshape(-1, 32)
    # thread mappings of pow2_kernel.cu: (sequence, butterfly) of each value set
    last = "x" if (not direct and kind == "c2c") else ("r" if (not direct and kind == "r2c" and lpt == 2) else "m")
    first_h = kind == "c2r" and lpt == 2

    def mapping(which):
        if which == "x":
            g, b = tid % slots, tid // slots
            return [(lpt * g + i, b) for i in range(lpt)]
        if which in ("r", "h"):
            if which == "r":
                s, c = tid % nseq, tid // nseq
            else:
                s, c = tid // (T // 2), tid % (T // 2)
            return [(s, c), (s, np.where(c == 0, T // 2, T - c))]
        slot, t = tid // T, tid % T
        return [(slot + slots * i, t) for i in range(lpt)]

    tot = 0
    for st in range(nst - 1):  # exchange after stage st
        R = lead if st == 0 else 8
        NS = 1 if st == 0 else lead * 8 ** (st - 1)
        for sq, bf in mapping("h" if (st == 0 and first_h) else "m"):
            for q in range(8):
                u, r = divmod(q, R)
                jb = bf + u * T
                k = jb & (NS - 1)
                tot += wavefronts(sq * SEQ + padded((jb - k) * R + k + r * NS, sh), E)
        for sq, bf in mapping(last if st + 1 == nst - 1 else "m"):
            for m in range(8):
                tot += wavefronts(sq * SEQ + padded(bf + T * m, sh), E)
    H = N // 2 + 1
    # register stores (direct C2C/C2R, transposed C2C, transposed R2C at two
    # sequences per thread) touch no shared memory after the last stage
    if (direct and kind != "r2c") or last != "m":
        return tot
    slot, t = tid // T, tid % T
    for i in range(lpt):
        base = (slot + slots * i) * SEQ
        for r in range(8):
            tot += wavefronts(base + padded(t + T * r, sh), E)
    if direct:  # R2C split store from shared memory
        for i in range(lpt):
            s = slot + slots * i
            for k0 in range(0, H, T):
                k = k0 + t
                act = k < H
                kk = np.where(act, k, 0)
                tot += wavefronts(np.where(act, s * SEQ + padded(kk, sh), -1), E)
                tot += wavefronts(np.where(act, s * SEQ + padded((N - kk) & (N - 1), sh), -1), E)
        return tot
    lmax = nseq if kind == "c2c" else 2 * nseq
    pairs = max(lmax // 2, 1)
    nout = H if kind == "r2c" else N
    I = loop_lanes(pairs * nout)
    act = I >= 0
    Ia = np.where(act, I, 0)
    j = 2 * (Ia & (pairs - 1))
    k = Ia // pairs
    tot += wavefronts(np.where(act, (j >> 1) * SEQ + padded(k, sh), -1), E)
    if kind == "r2c":
        tot += wavefronts(np.where(act, (j >> 1) * SEQ + padded((N - k) & (N - 1), sh), -1), E)
    return tot


# ---------------------------------------------------------- mixed-radix kernel
RADICES = [16, 15, 14, 12, 11, 10, 9, 8, 7, 6, 5, 4, 3, 2]


def mr_factor(N, max_radix=16):
    """Stage radices of mr_kernel.cuh (up to max_radix; 11 always allowed):
    fewest stages, then smallest largest radix."""
    inf = 1 << 20
    st, mx, ch = {}, {}, {}
    for m in range(2, N + 1):
        if N % m:
            continue
        st[m], mx[m], ch[m] = inf, inf, 0
        for r in RADICES:
            if m % r or (r > max_radix and r != 11):
                continue
            rest = m // r
            if rest > 1 and st[rest] >= inf:
                continue
            sx = (0 if rest == 1 else st[rest]) + 1
            xx = r if (rest == 1 or mx[rest] < r) else mx[rest]
            if sx < st[m] or (sx == st[m] and xx < mx[m]):
                st[m], mx[m], ch[m] = sx, xx, r
    out, m = [], N
    while m > 1 and ch[m] > 0:
        out.append(ch[m])
        m //= ch[m]
    return out


def mr_nseq(N, rb):
    fit = (3072 if rb == 4 else 1536) // N
    if fit >= 64:
        return 64
    if rb == 4 and N > 512:
        return 4
    if fit < 2:
        return 2
    p = 1
    while p * 2 <= fit:
        p *= 2
    return p


def mr_max_radix(N, nseq, rb):
    """Radix cap of mr_kernel.cuh (MRGeom::MAX_RADIX)."""
    return 16 if (rb == 4 and N & (N - 1)) else 8


def mr_sched(N, nseq, rb):
    r = mr_factor(N, mr_max_radix(N, nseq, rb))
    best, best_cost = 0, 1 << 30
    for i, R in enumerate(r):
        c = ((nseq * (N // R) + THREADS - 1) // THREADS) * R
        if c < best_cost or (c == best_cost and R > r[best]):
            best, best_cost = i, c
    return [r[best]] + r[:best] + r[best + 1:]


def mr_cost(N, rb, sh, SEQ, kind, direct):
    if kind == "r2r":
        return mr_r2r_cost(N, rb, sh, SEQ, direct)
    E = 2 * rb
    nseq = mr_nseq(N, rb)
    rad = mr_sched(N, nseq, rb)
    tot = 0
    ns = 1
    for st, R in enumerate(rad):
        NB = N // R
        B = loop_lanes(nseq * NB)
        act = B >= 0
        last_to_hbm = st == len(rad) - 1 and direct and kind != "r2c"
        if st == 0 or last_to_hbm:  # butterfly-fastest (coalesced HBM side)
            s, jb = np.divmod(np.where(act, B, 0), NB)
        else:  # shared-memory stages: sequence-fastest
            jb, s = np.divmod(np.where(act, B, 0), nseq)
        k = jb % ns
        if st == len(rad) - 1 and not direct and kind == "c2c":
            # register store: item (g, jb) reads butterfly jb of sequences 2g, 2g+1
            P = nseq // 2
            I = loop_lanes(P * NB)
            act = I >= 0
            Ia = np.where(act, I, 0)
            g, jb = Ia % P, Ia // P
            for r in range(R):
                for i in range(2):
                    tot += wavefronts(np.where(act, (2 * g + i) * SEQ + padded(jb + r * NB, sh), -1), E)
                if r > 0:
                    tot += wavefronts(np.where(act, (r - 1) * ns + jb, -1), E)
            return tot
        for r in range(R):
            if st > 0:
                tot += wavefronts(np.where(act, s * SEQ + padded(jb + r * NB, sh), -1), E)
                if r > 0:  # per-stage twiddle table: entry (r-1)*NS + k
                    tot += wavefronts(np.where(act, (r - 1) * ns + k, -1), E)
            if not last_to_hbm:
                base = (jb - k) * R + k
                tot += wavefronts(np.where(act, s * SEQ + padded(base + r * ns, sh), -1), E)
        ns *= R
    H = N // 2 + 1
    if direct:
        if kind == "r2c":
            I = loop_lanes(2 * nseq * H)
            act = I >= 0
            Ia = np.where(act, I, 0)
            l, k = Ia // H, Ia % H
            tot += wavefronts(np.where(act, (l >> 1) * SEQ + padded(k, sh), -1), E)
            tot += wavefronts(np.where(act, (l >> 1) * SEQ + padded((N - k) % N, sh), -1), E)
        return tot
    if kind == "c2c":
        P = nseq // 2
        I = loop_lanes(P * N)
        act = I >= 0
        Ia = np.where(act, I, 0)
        p, k = Ia % P, Ia // P
        tot += wavefronts(np.where(act, 2 * p * SEQ + padded(k, sh), -1), E)
        tot += wavefronts(np.where(act, (2 * p + 1) * SEQ + padded(k, sh), -1), E)
    else:
        I = loop_lanes(nseq * (H if kind == "r2c" else N))
        act = I >= 0
        Ia = np.where(act, I, 0)
        p, k = Ia % nseq, Ia // nseq
        tot += wavefronts(np.where(act, p * SEQ + padded(k, sh), -1), E)
        if kind == "r2c":
            tot += wavefronts(np.where(act, p * SEQ + padded((N - k) % N, sh), -1), E)
    return tot


def mr_r2r_cost(N, rb, sh, SEQ, direct):
    """The real-to-real kernel on the same layout: every stage after stage 0 in
    shared memory (sequence-fastest), then the store's reads, modelled on the
    DHT's pair k, n - k (lanes over sequences for a transposed store, along k
    for a direct one)."""
    E = 2 * rb
    nseq = mr_nseq(N, rb)
    rad = mr_sched(N, nseq, rb)
    tot = 0
    ns = 1
    for st, R in enumerate(rad):
        NB = N // R
        B = loop_lanes(nseq * NB)
        act = B >= 0
        if st == 0:
            s, jb = np.divmod(np.where(act, B, 0), NB)
        else:
            jb, s = np.divmod(np.where(act, B, 0), nseq)
        k = jb % ns
        for r in range(R):
            if st > 0:
                tot += wavefronts(np.where(act, s * SEQ + padded(jb + r * NB, sh), -1), E)
                if r > 0:
                    tot += wavefronts(np.where(act, (r - 1) * ns + k, -1), E)
            base = (jb - k) * R + k
            tot += wavefronts(np.where(act, s * SEQ + padded(base + r * ns, sh), -1), E)
        ns *= R
    I = loop_lanes(nseq * N)
    act = I >= 0
    Ia = np.where(act, I, 0)
    if direct:
        p, k = Ia // N, Ia % N
    else:
        p, k = Ia % nseq, Ia // nseq
    tot += wavefronts(np.where(act, p * SEQ + padded(k, sh), -1), E)
    tot += wavefronts(np.where(act, p * SEQ + padded((N - k) % N, sh), -1), E)
    return tot


def best_layout(args):
    family, N, rb = args
    cost = p2_cost if family == "pow2" else mr_cost
    kinds = KINDS if family == "pow2" else KINDS + [("r2r", False), ("r2r", True)]
    best = None
    for sh in SHIFTS:
        lo = padded(N - 1, sh) + 1
        for SEQ in range(lo, lo + 16):
            c = sum(cost(N, rb, sh, SEQ, kind, direct) for kind, direct in kinds)
            key = (c, SEQ, sh)
            if best is None or key < best:
                best = key
    return family, N, rb, best[2], best[1], best[0]


def main():
    jobs = [("pow2", N, rb) for N in POW2 for rb in (4, 8)] + [("mr", N, rb) for N in MR_ALL for rb in (4, 8)]
    with get_context("spawn").Pool(os.cpu_count() or 1) as pool:
        res = pool.map(best_layout, jobs)
    table = {(f, N, rb): (sh, seq) for f, N, rb, sh, seq, _ in res}
    out = ["// Generated by gen_smem_layout.py: shared-memory sequence layout (padding",
           "// shift SH, sequence stride SEQ) of the pass kernels, chosen per length and",
           "// precision by replaying the kernels' shared-memory accesses through a bank",
           "// model.  Element i of sequence s sits at s*SEQ + i + (SH ? i >> SH : 0).",
           "#pragma once", "", "namespace pb {", "", "struct SmemLayout {", "  int sh;", "  int seq;", "};", ""]
    for family, lengths in (("pow2", POW2), ("mr", MR_ALL)):
        out.append(f"// {family}: {{f32}}, {{f64}} per length")
        out.append(f"__host__ __device__ constexpr SmemLayout {family}_layout(int N, int real_bytes) {{")
        out.append("  switch (N) {")
        for N in lengths:
            a, b = table[(family, N, 4)], table[(family, N, 8)]
            out.append(f"    case {N}: return real_bytes == 4 ? SmemLayout{{{a[0]}, {a[1]}}} : SmemLayout{{{b[0]}, {b[1]}}};")
        out.append("    default: return SmemLayout{3, N + N / 8 + 1};")
        out.append("  }")
        out.append("}")
        out.append("")
    out.append("}  // namespace pb")
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "smem_layout.hpp")
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")
    for f, N, rb, sh, seq, c in sorted(res):
        print(f, N, rb, sh, seq, c)


if __name__ == "__main__":
    main()
