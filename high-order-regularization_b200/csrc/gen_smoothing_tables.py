"""Generates hr_smoothing_tables.inc: piecewise polynomials for the smoothing
factors of the on-surface regularized kernels, as functions of s = (r/delta)^2.

With lam = r / delta and E(lam) = (2/sqrt(pi)) lam exp(-lam^2), the on-surface
factors of the 7th-order kernels (2S/utilities.cpp:211-254 and :292-323) are

    s1 = [erf(lam) + (11/5 - 26/15 lam^2 + 4/15 lam^4) E] / r           = G1(s) / delta
    s2 = [erf(lam) + (-1 + (118 lam^2 - 68 lam^4 + 8 lam^6)/15) E] / r^3 = G2(s) / delta^3
    s3 = [erf(lam) + (-1 - 2/3 lam^2 + 52/45 lam^4 - 8/45 lam^6) E] / r^5 = G3(s) / delta^5

where G1 = f1 / lam, G2 = f2 / lam^3, G3 = f3 / lam^5 are even in lam and
therefore analytic in s = lam^2, with the reference's r -> 0 values
(32/5, 256/15, 128/45) / sqrt(pi) as their limits at s = 0.

FP64 tables (the FP64 sums): on s in [0, 64], pieces 0 .. NI centred on the
grid c_i = i * 64 / NI, each a polynomial of degree DEG in t = s - c_i (the
interpolant at DEG + 1 Chebyshev nodes of the piece, solved in 80-digit
arithmetic with mpmath): G1 and G2 64 pieces of degree 13, G3 256 pieces of
degree 9. A kernel finds the piece of s as round-to-nearest(s * NI / 64) with
one fused multiply-add and needs no stored centre. The script checks the
rounded coefficients against the 80-digit function and writes the maximum
relative error into the generated file (~1e-16). FP32 tables (the
reduced-precision path): pieces uniform in s with the piece index floor(s *
NI32 / 64), checked by emulating their FP32 evaluation.

Run from this directory: python gen_smoothing_tables.py
"""
import os

import mpmath as mp

mp.mp.dps = 80
HERE = os.path.dirname(os.path.abspath(__file__))


def E(lam):
    return 2 / mp.sqrt(mp.pi) * lam * mp.exp(-lam * lam)


def G1(s):
    if s == 0:
        return mp.mpf(32) / 5 / mp.sqrt(mp.pi)
    lam = mp.sqrt(s)
    return (mp.erf(lam) + (mp.mpf(11) / 5 - mp.mpf(26) / 15 * s + mp.mpf(4) / 15 * s * s) * E(lam)) / lam


def G2(s):
    if s == 0:
        return mp.mpf(256) / 15 / mp.sqrt(mp.pi)
    lam = mp.sqrt(s)
    return (mp.erf(lam) + (-1 + (118 * s - 68 * s * s + 8 * s ** 3) / 15) * E(lam)) / lam ** 3


def G3(s):
    if s == 0:
        return mp.mpf(128) / 45 / mp.sqrt(mp.pi)
    lam = mp.sqrt(s)
    return (mp.erf(lam) + (-1 - mp.mpf(2) / 3 * s + mp.mpf(52) / 45 * s * s - mp.mpf(8) / 45 * s ** 3) * E(lam)) / lam ** 5


def horner(coef, t):
    p = mp.mpf(0)
    for a in reversed(coef):
        p = p * t + a
    return p


# FP64 tables centred on a uniform grid in s, for an index formed by one
# fused multiply-add: piece i (i = 0 .. NI) is centred at c_i = i * 64 / NI
# and covers s in [c_i - w/2, c_i + w/2] (w = 64 / NI), so the piece of s is
# round-to-nearest(s * NI / 64) and t = s - c_i needs no stored centre. Each
# piece is DEG + 1 monomial coefficients in t, the interpolant at DEG + 1
# Chebyshev nodes of the piece widened by 0.2 % of w at each end (80 digits).
GRID_TABLES = {"G1": (64, 13), "G2": (64, 13), "G3": (256, 9)}


def piece_grid(f, i, ni, deg):
    w = mp.mpf(64) / ni
    c = i * w
    slo = max(mp.mpf(0), c - w / 2 - w * mp.mpf("0.002"))
    shi = c + w / 2 + w * mp.mpf("0.002")
    half, mid = (shi - slo) / 2, (shi + slo) / 2
    n = deg + 1
    ts = [mid + half * mp.cos(mp.pi * (k + mp.mpf(1) / 2) / n) - c for k in range(n)]
    V = mp.matrix(n, n)
    for r, t in enumerate(ts):
        for j in range(n):
            V[r, j] = t ** j
    coef = mp.lu_solve(V, mp.matrix([f(t + c) for t in ts]))
    return [coef[j] for j in range(n)], c


def build_grid(f, ni, deg):
    """Rounded coefficients of pieces 0 .. ni and the worst relative error of
    their exact evaluation over 21 points per piece within [0, 64]."""
    out, worst = [], mp.mpf(0)
    w = mp.mpf(64) / ni
    for i in range(ni + 1):
        coef, c = piece_grid(f, i, ni, deg)
        cd = [float(a) for a in coef]
        for k in range(21):
            sv = mp.mpf(float(c - w / 2 + w * k / 20))
            if sv < 0 or sv > 64:
                continue
            ex = f(sv)
            worst = max(worst, abs(horner([mp.mpf(a) for a in cd], sv - c) - ex) / abs(ex))
        out.append(cd)
    return out, worst


# FP32 tables for the mixed-precision path: NI32 pieces uniform in s (index
# floor(s * NI32 / 64), no square root), degree DEG32, each piece stored as
# 8 floats (centre, coefficients of t^0 .. t^5, 0) = two float4.
NI32 = 128
DEG32 = 5


def piece32(f, i):
    w = mp.mpf(64) / NI32
    slo = max(mp.mpf(0), i * w - mp.mpf("0.01"))
    shi = (i + 1) * w + mp.mpf("0.01")
    c = (i + mp.mpf(1) / 2) * w
    half, mid = (shi - slo) / 2, (shi + slo) / 2
    n = DEG32 + 1
    ts = [mid + half * mp.cos(mp.pi * (k + mp.mpf(1) / 2) / n) - c for k in range(n)]
    V = mp.matrix(n, n)
    for r, t in enumerate(ts):
        for j in range(n):
            V[r, j] = t ** j
    coef = mp.lu_solve(V, mp.matrix([f(t + c) for t in ts]))
    return [coef[j] for j in range(n)], c


def build32(f):
    """Float pieces and the worst relative error of their FP32 Horner evaluation
    (emulated with numpy float32) over 21 points per piece."""
    import numpy as np
    out, worst = [], 0.0
    w = 64.0 / NI32
    for i in range(NI32):
        coef, c = piece32(f, i)
        cf = np.array([float(a) for a in coef], np.float32)
        cc = np.float32(float(c))
        for k in range(21):
            sv = np.float32(i * w + w * k / 20.0)
            t = np.float32(sv - cc)
            v = cf[-1]
            for a in cf[-2::-1]:
                v = np.float32(v * t + a)
            ex = f(mp.mpf(float(sv)))
            worst = max(worst, float(abs(mp.mpf(float(v)) - ex) / abs(ex)))
        out.append([float(cc)] + [float(a) for a in cf] + [0.0] * (6 - DEG32))
    return out, worst


def main():
    lines = ["// Generated by gen_smoothing_tables.py; do not edit.",
             "// Piecewise polynomials G(s), s = (r/delta)^2 in [0, 64], of the on-surface smoothing factors.",
             "// FP64: pieces centred on a uniform grid in s, monomial coefficients in t = s - centre.",
             "// The includer defines HR_SMOOTH_STORAGE (e.g. static __device__ const)."]
    for name, f in (("G1", G1), ("G2", G2), ("G3", G3)):
        ni, deg = GRID_TABLES[name]
        tab, worst = build_grid(f, ni, deg)
        lines.append("// %s on the s grid: pieces 0 .. %d centred at i * %g, degree %d; max relative error %.2e"
                     % (name, ni, 64.0 / ni, deg, float(worst)))
        print(name, "grid max rel err", float(worst))
        lines.append("#define HR_SMOOTHS_%s_PIECES %d" % (name, ni))
        lines.append("#define HR_SMOOTHS_%s_DEG %d" % (name, deg))
        lines.append("HR_SMOOTH_STORAGE double kSmoothS%s[%d * %d] = {" % (name, ni + 1, deg + 1))
        for cd in tab:
            lines.append("    " + ", ".join(repr(v) for v in cd) + ",")
        lines.append("};")
    lines.append("// FP32 tables: %d pieces uniform in s (width %g), degree %d; per piece 8 floats:"
                 % (NI32, 64.0 / NI32, DEG32))
    lines.append("// centre, coefficients of t^0 .. t^%d, 0." % DEG32)
    lines.append("#define HR_SMOOTH32_PIECES %d" % NI32)
    for name, f in (("G1", G1), ("G2", G2), ("G3", G3)):
        tab, worst = build32(f)
        lines.append("// %s (FP32): max relative error of the FP32 evaluation %.2e" % (name, worst))
        print(name, "FP32 max rel err", worst)
        lines.append("HR_SMOOTH_STORAGE float kSmooth32%s[%d * 8] = {" % (name, NI32))
        for row in tab:
            lines.append("    " + ", ".join("%.9ef" % v for v in row) + ",")
        lines.append("};")
    with open(os.path.join(HERE, "hr_smoothing_tables.inc"), "w") as fh:
        fh.write("\n".join(lines) + "\n")


if __name__ == "__main__":
    main()
