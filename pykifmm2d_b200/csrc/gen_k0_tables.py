"""Generate k0_tables.h: coefficients for the modified Bessel function K0.

Method (derived here from the mathematics, evaluated with mpmath at 50 digits):
  0 < x <= 2:  K0(x) = P(t) - log(x/2) * I0(t),  t = x^2, with the power series
               I0 = sum_k t^k / (4^k (k!)^2),  P = sum_k (H_k - gamma) t^k / (4^k (k!)^2)
               (H_k the harmonic numbers, H_0 = 0; DLMF 10.31.2 and 10.25.2).
  x > 2:       K0(x) = exp(-x) / sqrt(x) * F(z),  z = 8/x in (0, 4),
               F(z) = sqrt(x) exp(x) K0(x) smooth on [0, 4] (F(0) = sqrt(pi/2)),
               as a Chebyshev series in u = z/2 - 1 on [-1, 1], coefficients from
               the discrete Chebyshev transform at 64 Chebyshev nodes.
Terms are kept while they matter at double (FP64) or single (FP32) precision.

Run:  python pykifmm2d_b200/csrc/gen_k0_tables.py   (rewrites k0_tables.h beside it)
"""
import os

import mpmath as mp

mp.mp.dps = 50
HERE = os.path.dirname(os.path.abspath(__file__))


def series(nterms):
    g = mp.euler
    i0, p = [], []
    h = mp.mpf(0)
    for k in range(nterms):
        if k > 0:
            h += mp.mpf(1) / k
        c = mp.mpf(1) / (mp.mpf(4) ** k * mp.factorial(k) ** 2)
        i0.append(c)
        p.append((h - g) * c)
    return i0, p


def cheb_large(n=64):
    # F(z) = sqrt(x) e^x K0(x), x = 8/z ; u = z/2 - 1
    def F(u):
        z = 2 * (u + 1)
        if z == 0:
            return mp.sqrt(mp.pi / 2)
        x = 8 / z
        return mp.sqrt(x) * mp.exp(x) * mp.besselk(0, x)
    nodes = [mp.cos(mp.pi * (j + mp.mpf(1) / 2) / n) for j in range(n)]
    vals = [F(u) for u in nodes]
    coef = []
    for k in range(n):
        s = sum(vals[j] * mp.cos(mp.pi * k * (j + mp.mpf(1) / 2) / n) for j in range(n))
        coef.append(2 * s / n)
    coef[0] /= 2
    return coef


def trim(c, tol):
    scale = max(abs(v) for v in c)
    last = 0
    for i, v in enumerate(c):
        if abs(v) > tol * scale:
            last = i
    return c[: last + 1]


def fmt(vals, single):
    if single:
        return ",\n    ".join("%.9ef" % float(v) for v in vals)
    return ",\n    ".join("%.17e" % float(v) for v in vals)


def main():
    i0, p = series(40)
    # t <= 4: term k is at most 4^k c_k = 1/(k!)^2 in size; keep while above the precision
    def trim_series(c, tol):
        last = max(i for i, v in enumerate(c) if abs(v) * 4 ** i > tol)
        return c[: last + 1]
    i0_64 = trim_series(i0, 1e-19); p_64 = trim_series(p, 1e-19)
    i0_32 = trim_series(i0, 1e-9); p_32 = trim_series(p, 1e-9)
    ch = cheb_large()
    ch_64 = trim(ch, 1e-18)
    ch_32 = trim(ch, 2e-9)
    out = []
    out.append("/* Generated by gen_k0_tables.py -- do not edit.  Coefficients for K0:")
    out.append(" * x <= 2: K0 = P(x^2) - log(x/2) I0(x^2) with power series in t = x^2;")
    out.append(" * x >  2: K0 = exp(-x)/sqrt(x) * sum_k c_k T_k(u), u = 4/x - 1 (Chebyshev). */")
    out.append("#pragma once")
    for name, vals, single in (("K0_I0_D", i0_64, False), ("K0_P_D", p_64, False), ("K0_CHEB_D", ch_64, False),
                               ("K0_I0_F", i0_32, True), ("K0_P_F", p_32, True), ("K0_CHEB_F", ch_32, True)):
        ty = "float" if single else "double"
        out.append(f"#define {name}_N {len(vals)}")
        out.append(f"static __device__ __constant__ {ty} {name}[{len(vals)}] = {{\n    {fmt(vals, single)}}};")
    open(os.path.join(HERE, "k0_tables.h"), "w").write("\n".join(out) + "\n")
    print("terms: I0 %d/%d  P %d/%d  cheb %d/%d" % (len(i0_64), len(i0_32), len(p_64), len(p_32), len(ch_64), len(ch_32)))


if __name__ == "__main__":
    main()
