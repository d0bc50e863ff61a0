"""Generates dg_dd_tables.h: double-double constants for the device's
correctly rounded FP64 atan2 and sin (dg_ddmath.cuh).

    python dioptrin_b200/csrc/gen_dd_tables.py

Values are computed with Python's decimal module at 70 significant digits
from their Taylor series (pi from Machin's formula), then split into a
nearest-double head and a nearest-double tail.
"""
import os
from decimal import Decimal as D, getcontext

getcontext().prec = 70
STEP = 64  # table spacing 1/64


def atan_series(x: D) -> D:
    # Halve the argument twice with atan(x) = 2 atan(x / (1 + sqrt(1 + x^2))).
    k = 0
    while abs(x) > D(1) / 8:
        x = x / (1 + (1 + x * x).sqrt())
        k += 1
    term, s, n, x2 = x, D(0), 1, x * x
    while True:
        t = term / n
        if abs(t) < D(10) ** -75:
            break
        s += t
        term *= -x2
        n += 2
    return s * (2 ** k)


def pi() -> D:
    return 16 * atan_series(D(1) / 5) - 4 * atan_series(D(1) / 239)


def sin_cos(x: D):
    s, c, term, n = D(0), D(0), D(1), 0
    while True:
        if n % 2 == 0:
            c += term if (n // 2) % 2 == 0 else -term
        else:
            s += term if (n // 2) % 2 == 0 else -term
        n += 1
        term = term * x / n
        if abs(term) < D(10) ** -75:
            break
    return s, c


def split(v: D):
    hi = float(v)
    lo = float(v - D(hi))
    return hi, lo


def hexf(x: float) -> str:
    return x.hex() if x != 0 else "0x0p+0"


def main():
    P = pi()
    lines = ["// Generated by gen_dd_tables.py: double-double (head, tail) constants.",
             "#pragma once", ""]
    for name, v in [("kPi", P), ("kPiHalf", P / 2)]:
        h, l = split(v)
        lines.append(f"static constexpr double {name}Hi = {hexf(h)};")
        lines.append(f"static constexpr double {name}Lo = {hexf(l)};")
    # coefficients 1/(2k+1) of the atan series and 1/k! of sin/cos
    inv_odd = [split(D(1) / (2 * k + 1)) for k in range(12)]
    inv_fact = [split(D(1) / D(__import__("math").factorial(k))) for k in range(20)]
    lines.append("__device__ static const double kInvOdd[12][2] = {" + ", ".join(
        f"{{{hexf(h)}, {hexf(l)}}}" for h, l in inv_odd) + "};")
    lines.append("__device__ static const double kInvFact[20][2] = {" + ", ".join(
        f"{{{hexf(h)}, {hexf(l)}}}" for h, l in inv_fact) + "};")
    atan_tab = [split(atan_series(D(k) / STEP)) for k in range(STEP + 1)]
    lines.append(f"__device__ static const double kAtanTab[{STEP + 1}][2] = {{" + ", ".join(
        f"{{{hexf(h)}, {hexf(l)}}}" for h, l in atan_tab) + "};")
    n_sc = int(float(P / 2) * STEP) + 2
    sc = [sin_cos(D(k) / STEP) for k in range(n_sc)]
    lines.append(f"__device__ static const double kSinTab[{n_sc}][2] = {{" + ", ".join(
        "{%s, %s}" % tuple(hexf(v) for v in split(s)) for s, _ in sc) + "};")
    lines.append(f"__device__ static const double kCosTab[{n_sc}][2] = {{" + ", ".join(
        "{%s, %s}" % tuple(hexf(v) for v in split(c)) for _, c in sc) + "};")
    lines.append(f"static constexpr int kTabStep = {STEP};")
    lines.append(f"static constexpr int kSinTabLen = {n_sc};")
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "dg_dd_tables.h")
    with open(out, "w") as f:
        f.write("\n".join(lines) + "\n")
    print("wrote", out)


if __name__ == "__main__":
    main()
