"""Generate mr_daubechies.h: Daubechies scaling filters dbN, N = 1..30.

N = 1..15 are computed here from their definition (Daubechies, "Ten Lectures on Wavelets",
ch. 6: minimum-phase spectral factorisation):

    |H(w)|^2 = 2 cos^{2N}(w/2) P(sin^2(w/2)),   P(y) = sum_{k<N} C(N-1+k, k) y^k,
    H(z) = sqrt(2) ((1 + z^-1)/2)^N Q(z),  Q(z) = c * prod_k (1 - z_k z^-1),

where for every root y_k of P the factor uses the root z_k of (2 - z - 1/z)/4 = y_k inside
the unit circle. Arithmetic runs at 60 significant digits (mpmath); rounded to float these
equal kipl's WaveletKernel<float> taps bit for bit.

N = 16..30: kipl's own tables of these filters (core/kipl/kipl/include/wavelets/core/
wavelets.hpp, `double daubN[]` in WaveletKernel's constructor) deviate from the exact filters
by more than float rounding, so a computed filter would not reproduce MuhRec's ring cleaning
with those wavelets. The values of those constant tables are the contract for `wname`, so
this generator reads them from the reference source (the path given on the command line) and
stores each as the float the reference's CopyKernel makes of it (the kernels keep only that
float, so nothing else of the table is needed).

Exception: kipl's daub28 table holds 48 values for a 56-tap filter (and not those of db28),
so its kernel copies 8 values from past the end of the array: undefined. The library refuses
daub28; its row here is the computed filter, only so that the table is complete.

usage: python gen_daubechies.py <reference checkout> > mr_daubechies.h
"""
import os
import re
import sys

import mpmath as mp
import numpy as np

mp.mp.dps = 60
NCOMPUTED = 15
NMAX = 30
UNDEFINED = (28,)  # kipl's table is shorter than its filter


def daubechies(n: int):
    if n == 1:
        s = mp.sqrt(2) / 2
        return [s, s]
    p = [mp.binomial(n - 1 + k, k) for k in range(n)]  # coefficients of y^k
    ys = mp.polyroots(list(reversed(p)), maxsteps=400, extraprec=400)
    poly = [mp.mpc(1)]  # coefficients of z^-k
    for y in ys:
        b = 2 - 4 * y  # z + 1/z = b
        disc = mp.sqrt(b * b / 4 - 1)
        z1, z2 = b / 2 + disc, b / 2 - disc
        zk = z1 if abs(z1) < 1 else z2
        poly = [poly[i] - (zk * poly[i - 1] if i > 0 else 0) for i in range(len(poly))] + [-zk * poly[-1]]
    for _ in range(n):  # times (1 + z^-1)
        poly = [poly[i] + (poly[i - 1] if i > 0 else 0) for i in range(len(poly))] + [poly[-1]]
    h = [mp.re(c) for c in poly]
    s = sum(h)
    return [c * mp.sqrt(2) / s for c in h]


def reference_tables(ref_root: str) -> dict:
    """The `double daubN[] = {...}` tables of kipl's WaveletKernel, N > 15, as float."""
    path = os.path.join(ref_root, "core", "kipl", "kipl", "include", "wavelets", "core", "wavelets.hpp")
    src = open(path).read()
    out = {}
    for m in re.finditer(r"double\s+daub(\d+)\s*\[\s*\]\s*=\s*\{([^}]*)\}", src):
        n = int(m.group(1))
        if n > NCOMPUTED and n not in UNDEFINED:
            vals = [float(v) for v in m.group(2).replace("\n", " ").split(",") if v.strip()]
            if len(vals) != 2 * n:
                raise SystemExit(f"daub{n}: {len(vals)} values in the reference table, expected {2 * n}")
            out[n] = [float(np.float32(v)) for v in vals]
    missing = [n for n in range(NCOMPUTED + 1, NMAX + 1) if n not in out and n not in UNDEFINED]
    if missing:
        raise SystemExit(f"reference tables not found for daub{missing}")
    return out


def main():
    if len(sys.argv) != 2 or not os.path.isdir(sys.argv[1]):
        raise SystemExit("usage: python gen_daubechies.py <reference checkout> > mr_daubechies.h")
    ref = reference_tables(sys.argv[1])
    print("// Generated by gen_daubechies.py: Daubechies scaling filters dbN (N = 1..30), h[k],")
    print("// k = 0..2N-1. N <= 15 computed from the minimum-phase spectral factorisation at 60")
    print("// digits; N >= 16 the values of kipl's own tables as float (they differ from the exact")
    print("// filters by more than float rounding, and MuhRec's results follow them). daub28 is")
    print("// computed: kipl's table for it is shorter than the filter, and the library refuses it.")
    print("#pragma once")
    print(f"static const int kDaubMax = {NMAX};")
    print("static const double kDaub[][60] = {")
    for n in range(1, NMAX + 1):
        if n <= NCOMPUTED or n in UNDEFINED:
            h = daubechies(n)
            assert abs(sum(h) - mp.sqrt(2)) < mp.mpf(10) ** -40
            vals = ", ".join(repr(float(c)) for c in h)
        else:
            vals = ", ".join(repr(v) for v in ref[n])
        print(f"    {{{vals}}},")
    print("};")


if __name__ == "__main__":
    main()
