"""Generate mr_median_net.cuh: median selectors for windows of n = 3, 5, 9, 11, 15 and 25 values.

Also a rank selector that leaves ranks 7..12 of 20 values on wires 7..12 (for pairs of 5 x 5
windows). Each selector is Batcher's odd-even merge sort (K. E. Batcher, "Sorting networks and their
applications", AFIPS 1968) on the next power of two, with the padding wires known to hold +inf
at generation time (compare-exchanges against them vanish or become moves) and every
compare-exchange that cannot reach the kept outputs removed. What is left is a straight
sequence of fminf / fmaxf on registers; for windows without NaN it returns the exact middle
order statistic. Run: python gen_median_net.py > mr_median_net.cuh
"""
import sys


def oddeven_merge_sort(n):
    ces = []

    def merge(lo, hi, r):
        step = 2 * r
        if step < hi - lo:
            merge(lo, hi, step)
            merge(lo + r, hi, step)
            ces.extend((i, i + r) for i in range(lo + r, hi - r, step))
        else:
            ces.append((lo, lo + r))

    def sort(lo, hi):
        if hi - lo >= 1:
            mid = lo + (hi - lo) // 2
            sort(lo, mid)
            sort(mid + 1, hi)
            merge(lo, hi, 1)

    sort(0, n - 1)
    return ces


def selector(n, outs=None):
    """Pruned network for the middle output of n values, or for the output wires in outs (each
    wire k then holds the k-th smallest value, 0-based)."""
    size = 1
    while size < n:
        size *= 2
    inf = [w >= n for w in range(size)]
    ops = []
    for a, b in oddeven_merge_sort(size):
        if inf[b]:
            continue  # min(x, inf) = x, max = inf: nothing moves
        if inf[a]:
            ops.append(("mov", a, b))  # a takes b's value, b becomes inf
            inf[a], inf[b] = False, True
            continue
        ops.append(("ce", a, b))
    out = n // 2
    live = {out} if outs is None else set(outs)
    kept = []
    for op, a, b in reversed(ops):
        if op == "mov":
            if a in live:
                live.discard(a)
                live.add(b)
                kept.append(("mov", a, b, True, False))
            continue
        la, lb = a in live, b in live
        if la or lb:
            kept.append(("ce", a, b, la, lb))
            live.add(a)
            live.add(b)
    kept.reverse()
    return kept, out


def _body(ops, f):
    for op, a, b, la, lb in ops:
        if op == "mov":
            f.write(f"    v[{a}] = v[{b}];\n")
        elif la and lb:
            f.write(f"    {{ const float t = fminf(v[{a}], v[{b}]); v[{b}] = fmaxf(v[{a}], v[{b}]); v[{a}] = t; }}\n")
        elif la:
            f.write(f"    v[{a}] = fminf(v[{a}], v[{b}]);\n")
        else:
            f.write(f"    v[{b}] = fmaxf(v[{a}], v[{b}]);\n")


def count(ops):
    return sum(o[3] + o[4] for o in ops if o[0] == "ce")


def emit(n, f):
    ops, out = selector(n)
    f.write(f"// middle of {n} values: {count(ops)} min/max operations\n")
    f.write(f"__device__ __forceinline__ float median_net{n}(float (&v)[{n}])\n{{\n")
    _body(ops, f)
    f.write(f"    return v[{out}];\n}}\n\n")


def emit_range(n, lo, hi, f):
    ops, _ = selector(n, range(lo, hi + 1))
    f.write(f"// ranks {lo}..{hi} (0-based) of {n} values into v[{lo}..{hi}]: {count(ops)} min/max operations\n")
    f.write(f"__device__ __forceinline__ void rank_net{n}_{lo}_{hi}(float (&v)[{n}])\n{{\n")
    _body(ops, f)
    f.write("}\n\n")


def main():
    f = sys.stdout
    f.write("// Generated by gen_median_net.py (Batcher odd-even merge sort, pruned to the middle output).\n")
    f.write("#pragma once\n\nnamespace mr {\nnamespace ringalt {\n\n")
    for n in (3, 5, 9, 11, 15, 25):
        emit(n, f)
    # two horizontally adjacent 5x5 windows share 20 values; only their ranks 7..12 can be the
    # middle of either window, which is then the middle of those 6 and the window's own 5
    emit_range(20, 7, 12, f)
    f.write("} // namespace ringalt\n} // namespace mr\n")


if __name__ == "__main__":
    main()
