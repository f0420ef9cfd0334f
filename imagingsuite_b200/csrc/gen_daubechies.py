"""Generate mr_daubechies.h: Daubechies scaling filters dbN, N = 1..30.

The coefficients are computed here from their definition (Daubechies, "Ten Lectures on
Wavelets", ch. 6: minimum-phase spectral factorisation), not taken from any table:

    |H(w)|^2 = 2 cos^{2N}(w/2) P(sin^2(w/2)),   P(y) = sum_{k<N} C(N-1+k, k) y^k,
    H(z) = sqrt(2) ((1 + z^-1)/2)^N Q(z),  Q(z) = c * prod_k (1 - z_k z^-1),

where for every root y_k of P the factor uses the root z_k of (2 - z - 1/z)/4 = y_k inside
the unit circle. Arithmetic runs at 60 significant digits (mpmath); the header stores the
values with 17 significant digits (exact for the later rounding to float or double).

usage: python gen_daubechies.py > mr_daubechies.h
"""
import mpmath as mp

mp.mp.dps = 60
NMAX = 30


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


def main():
    print("// Generated by gen_daubechies.py: Daubechies scaling filters dbN (N = 1..30), computed")
    print("// from the minimum-phase spectral factorisation at 60 digits. h[k], k = 0..2N-1.")
    print("#pragma once")
    print(f"static const int kDaubMax = {NMAX};")
    print("static const double kDaub[][60] = {")
    for n in range(1, NMAX + 1):
        h = daubechies(n)
        assert abs(sum(h) - mp.sqrt(2)) < mp.mpf(10) ** -40
        vals = ", ".join(mp.nstr(c, 17, min_fixed=-1, max_fixed=0) if False else repr(float(c)) for c in h)
        print(f"    {{{vals}}},")
    print("};")


if __name__ == "__main__":
    main()
