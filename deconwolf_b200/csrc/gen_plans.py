"""Generate the per-length kernel instantiations of the FFT passes.

Writes, next to this file:
  plans_gen.h         the table of supported line lengths with their radix
                      lists and launch shapes (lines: T lines per CTA;
                      x pass: R rows per CTA)
  inst_lines_<k>.cu   explicit instantiations of k_lines, k_xpass and
  inst_x_<k>.cu       k_ypass, split for parallel compilation (the y files
  inst_y_<k>.cu       keep scalar complex adds: DW_PAIRED_ADDS 0)

A length N is supported when it factors into at most three radices <= 16
(7-smooth).  Candidate 0 of a length is the radix list that minimises the
threads per line (N / smallest radix), then the number of stages, then the
spread; the other candidates (alternate radix lists, a narrower column
tile) are for the engine's autotuner, which times them at first use.
Run: python gen_plans.py [--max 4096] [--parts 16]  (the committed files use 16 parts)
"""
from __future__ import annotations

import argparse
import itertools
import os

HERE = os.path.dirname(os.path.abspath(__file__))


def factors(n):
    out = []
    for p in (2, 3, 5, 7):
        while n % p == 0:
            out.append(p)
            n //= p
    return out, n


def smooth(n):
    return factors(n)[1] == 1


RADS = [r for r in range(2, 17) if smooth(r)]


def tpl_of(n, s):
    return max(n // s[0], n // s[1], n // s[2] if s[2] > 1 else 0)


def best_split(n):
    """(RA, RB, RC) with RA*RB*RC == n, radices in RADS (RB, RC may be 1)."""
    if n == 1:
        return (1, 1, 1)  # identity; the z pass of a 2-D job still multiplies by the OTF
    cands = []
    if n in RADS:
        cands.append((n, 1, 1))
    for a in RADS:
        if n % a:
            continue
        b = n // a
        if b in RADS:
            cands.append((a, b, 1))
        for c in RADS:
            if b % c == 0 and (b // c) in RADS:
                cands.append((a, c, b // c))
    if not cands:
        return None

    def key(s):
        rs = [r for r in s if r > 1]
        stages = 3 if s[2] > 1 else 2
        if len(rs) == 1:
            stages = 1
        tpl = tpl_of(n, s)
        # prefer a large first radix (it reads global memory with the most
        # independent loads per thread) and a moderate last one
        return (tpl, stages, max(rs) - min(rs), -s[0])

    return min(cands, key=key)


def lines_T(n, split):
    """Lines per CTA for the strided passes: as many as fit 1024 threads and
    ~100 KB of shared memory, at most 16 (128-byte segments)."""
    a, b, c = split
    rev = (c, b, a) if c > 1 else (b, a, 1)
    tpl = max(tpl_of(n, split), tpl_of(n, rev))
    padn = n + n // min(a, rev[0]) + 1
    T = 16
    while T > 1 and (T * tpl > 1024 or T * padn * 8 > 100 * 1024):
        T //= 2
    return T, tpl


SMEM_MAX = 220 * 1024
KB = 4


def padn(n, s):
    return n + n // s[0] + 1


def x_smem(n, split, R):
    """Shared memory of k_xpass<RD, R> (mirrors XCfg in passes.cuh)."""
    a, b, c = split
    rev = (c, b, a) if c > 1 else (b, a, 1)
    tpl = max(tpl_of(n, split), tpl_of(n, rev))
    threads = R * tpl
    row = max(n + 1, padn(n, split), padn(n, rev)) | 1
    nkb = (n + 1 + KB - 1) // KB
    area = (max(R * nkb * KB, R * row) + 1) // 2 * 2
    return 64 + 8 * area + 3 * 4 * R * ((2 * n + 3) // 4 * 4) + 8 * threads


def x_R(n, split):
    """Rows per x tile (complex half length n).  Two rows share each thread;
    small rows take more thread rows so that a CTA has a full warp; the tile
    should let three CTAs share an SM."""
    a, b, c = split
    rev = (c, b, a) if c > 1 else (b, a, 1)
    tpl = max(tpl_of(n, split), tpl_of(n, rev))
    R = 2
    while R * tpl < 64:
        R *= 2
    while R > 1 and (3 * x_smem(n, split, R) > 225 * 1024 or R * tpl > 1024):
        R //= 2
    return R, tpl


def y_fits(n, split):
    """k_ypass<RD> (4 lines, double buffered) fits in shared memory."""
    return 2 * padn(n, split) * KB * 8 + 64 <= SMEM_MAX and KB * tpl_of(n, split) <= 1024


def supported(maxn, start=2):
    out = []
    for n in range(start, maxn + 1):
        if smooth(n) and best_split(n):
            out.append(n)
    return out


def rad_str(s):
    return f"Rad<{s[0]}, {s[1]}, {s[2]}>"


def ranked_splits(n):
    """Every split of n into at most three radices <= 16, best first by the
    heuristic of best_split (so ranked_splits(n)[0] == best_split(n))."""
    if n == 1:
        return [(1, 1, 1)]
    cands = set()
    if n in RADS:
        cands.add((n, 1, 1))
    for a in RADS:
        if n % a:
            continue
        b = n // a
        if b in RADS:
            cands.add((a, b, 1))
        for c in RADS:
            if b % c == 0 and (b // c) in RADS:
                cands.add((a, c, b // c))
    best = best_split(n)
    rest = sorted(cands - {best}, key=lambda s: (tpl_of(n, s), 3 if s[2] > 1 else 2,
                                                 max(r for r in s if r > 1) - min(r for r in s if r > 1), -s[0], s))
    return [best] + rest


def alternates(n, ok, count):
    """Up to `count` splits after the best one that pass ok(split), each with a
    first radix not used by an earlier candidate (the first radix sets the
    global read pattern and the thread count of the first stage)."""
    out = []
    ranked = ranked_splits(n)
    used = {ranked[0][0]}
    for s in ranked[1:]:
        if len(out) == count:
            break
        if s[0] in used or not ok(s):
            continue
        used.add(s[0])
        out.append(s)
    return out


# Autotuning candidates per length (the engine times them at first use and
# keeps the fastest; candidate 0 is the heuristic's choice):
#   lines (z pass, and the y pass where its tile does not fit): the best
#     split at its column tile T, the best alternate split, and the best
#     split with half the column tile
#   y (persistent 4-line tiles): the best split and up to two alternates
#   x: the best split; for half lengths >= X_ALT_MIN one alternate split with
#     the same rows per tile, compiled for the iteration's two families
#     (ratio and update) only -- the set-up families use candidate 0
X_ALT_MIN = 96


def lines_cands(n):
    s0 = best_split(n)
    T0, _ = lines_T(n, s0)
    out = [(s0, T0)]
    if n > 1:
        for s in alternates(n, lambda s: True, 1):
            out.append((s, lines_T(n, s)[0]))
        if T0 >= 4:
            out.append((s0, T0 // 2))
    return out


def y_cands(n):
    return [best_split(n)] + alternates(n, lambda s: y_fits(n, s), 2)


def x_cands(n):
    s0 = best_split(n)
    R0, _ = x_R(n, s0)
    out = [(s0, R0)]
    if n >= X_ALT_MIN:
        def ok(s):
            R, _ = x_R(n, s)
            return R == R0 and x_smem(n, s, R) <= SMEM_MAX
        for s in alternates(n, ok, 1):
            out.append((s, R0))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--max", type=int, default=4096)
    ap.add_argument("--xmax", type=int, default=2048, help="largest complex half length of the x pass")
    ap.add_argument("--parts", type=int, default=8)
    ap.add_argument("--only", type=str, default="", help="comma list of lengths (development builds)")
    args = ap.parse_args()

    lines_ns = supported(args.max, start=1)
    x_ns = [n for n in supported(args.xmax) if x_smem(n, best_split(n), x_R(n, best_split(n))[0]) <= SMEM_MAX]
    if args.only:
        keep = {int(v) for v in args.only.split(",")}
        lines_ns = [n for n in lines_ns if n in keep or n == 1]
        x_ns = [n for n in x_ns if n in keep]
    y_ns = [n for n in lines_ns if n > 1 and y_fits(n, best_split(n))]

    hdr = []
    hdr.append("// generated by gen_plans.py -- do not edit")
    hdr.append("#pragma once")
    hdr.append("#include \"passes.cuh\"")
    hdr.append("namespace dwcu {")
    hdr.append("// one entry per autotuning candidate of a length, candidates of a length in")
    hdr.append("// order (cand 0: the generator's heuristic choice)")
    hdr.append("struct LinesPlan { int n, cand, ra, rb, rc, T, threads; size_t smem; void (*launch)(const LinesArgs &, int, cudaStream_t); };")
    hdr.append("struct XPlan { int n, cand, ra, rb, rc, R, threads; size_t smem; void (*launch)(const XArgs &, cudaStream_t); };")
    hdr.append("struct YPlan { int n, cand, ra, rb, rc, threads; size_t smem; void (*launch)(const YArgs &, cudaStream_t); };")
    for n in lines_ns:
        for c, _ in enumerate(lines_cands(n)):
            hdr.append(f"void launch_lines_{n}_{c}(const LinesArgs &, int, cudaStream_t);")
    for n in x_ns:
        for c, _ in enumerate(x_cands(n)):
            hdr.append(f"void launch_x_{n}_{c}(const XArgs &, cudaStream_t);")
    for n in y_ns:
        for c, _ in enumerate(y_cands(n)):
            hdr.append(f"void launch_y_{n}_{c}(const YArgs &, cudaStream_t);")
    hdr.append("static const LinesPlan kLinesPlans[] = {")
    for n in lines_ns:
        for c, (s, T) in enumerate(lines_cands(n)):
            hdr.append(f"    {{{n}, {c}, {s[0]}, {s[1]}, {s[2]}, {T}, LinesCfg<{rad_str(s)}, {T}>::THREADS, "
                       f"LinesCfg<{rad_str(s)}, {T}>::SMEM_BYTES, launch_lines_{n}_{c}}},")
    hdr.append("};")
    hdr.append("static const XPlan kXPlans[] = {")
    for n in x_ns:
        for c, (s, R) in enumerate(x_cands(n)):
            hdr.append(f"    {{{n}, {c}, {s[0]}, {s[1]}, {s[2]}, {R}, XCfg<{rad_str(s)}, {R}>::THREADS, "
                       f"XCfg<{rad_str(s)}, {R}>::SMEM_BYTES, launch_x_{n}_{c}}},")
    hdr.append("};")
    hdr.append("static const YPlan kYPlans[] = {")
    for n in y_ns:
        for c, s_ in enumerate(y_cands(n)):
            hdr.append(f"    {{{n}, {c}, {s_[0]}, {s_[1]}, {s_[2]}, YCfg<{rad_str(s_)}>::THREADS, "
                       f"YCfg<{rad_str(s_)}>::SMEM_BYTES, launch_y_{n}_{c}}},")
    hdr.append("};")
    hdr.append("}  // namespace dwcu")
    with open(os.path.join(HERE, "plans_gen.h"), "w") as f:
        f.write("\n".join(hdr) + "\n")

    # instantiation files
    for old in os.listdir(HERE):
        if old.startswith("inst_") and old.endswith(".cu"):
            os.remove(os.path.join(HERE, old))
    parts = max(1, args.parts)
    for kind, ns in (("lines", lines_ns), ("x", x_ns), ("y", y_ns)):
        for p in range(parts):
            chunk = ns[p::parts]
            lines = ["// generated by gen_plans.py -- do not edit"]
            if kind == "y":
                # the y pass runs faster with scalar complex adds (dft.cuh)
                lines.append("#define DW_PAIRED_ADDS 0")
            lines += ["#include \"launch.cuh\"", "namespace dwcu {"]
            if kind == "x":
                lines += [f"void launch_x_{n}_0(const XArgs &, cudaStream_t);" for n in chunk]
            for n in chunk:
                if kind == "lines":
                    for c, (s, T) in enumerate(lines_cands(n)):
                        lines.append(f"void launch_lines_{n}_{c}(const LinesArgs &a, int nb, cudaStream_t st) "
                                     f"{{ launch_lines_t<{rad_str(s)}, {T}>(a, nb, st); }}")
                elif kind == "x":
                    for c, (s, R) in enumerate(x_cands(n)):
                        if c == 0:
                            lines.append(f"void launch_x_{n}_0(const XArgs &a, cudaStream_t st) "
                                         f"{{ launch_x_t<{rad_str(s)}, {R}>(a, st); }}")
                        else:
                            lines.append(f"void launch_x_{n}_{c}(const XArgs &a, cudaStream_t st) "
                                         f"{{ if (x_iteration_op(a.op)) launch_x_iter_t<{rad_str(s)}, {R}>(a, st); "
                                         f"else launch_x_{n}_0(a, st); }}")
                else:
                    for c, s in enumerate(y_cands(n)):
                        lines.append(f"void launch_y_{n}_{c}(const YArgs &a, cudaStream_t st) "
                                     f"{{ launch_y_t<{rad_str(s)}>(a, st); }}")
            lines.append("}  // namespace dwcu")
            with open(os.path.join(HERE, f"inst_{kind}_{p}.cu"), "w") as f:
                f.write("\n".join(lines) + "\n")
    nl = sum(len(lines_cands(n)) for n in lines_ns)
    nx = sum(len(x_cands(n)) for n in x_ns)
    ny = sum(len(y_cands(n)) for n in y_ns)
    print(f"lines lengths: {len(lines_ns)} ({nl} plans)  x half-lengths: {len(x_ns)} ({nx} plans)  "
          f"y tiles: {len(y_ns)} ({ny} plans)")


if __name__ == "__main__":
    main()
