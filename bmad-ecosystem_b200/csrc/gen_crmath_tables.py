"""Generate bgt_crmath_tables.h: double-double (hi, lo) splits of the series
coefficients and constants used by bgt_crmath.cuh, as exact hex-float
literals.

    python gen_crmath_tables.py > bgt_crmath_tables.h

Coefficients are exact rationals (Taylor series of sin, cos, sinh, cosh, exp,
asin, atan);
pi/2 and pi are taken to 200 bits from a Machin-formula evaluation.
"""
from fractions import Fraction as F
from math import factorial


def pi_fraction(bits=260):
    # Machin: pi = 16 atan(1/5) - 4 atan(1/239), each atan summed to ~bits
    def atan_inv(n):
        s, k, term = F(0), 0, F(1, n)
        eps = F(1, 2 ** bits)
        while term > eps:
            s += term if k % 2 == 0 else -term
            k += 1
            term = F(1, (2 * k + 1) * n ** (2 * k + 1))
        return s
    return 16 * atan_inv(5) - 4 * atan_inv(239)


def to_double(fr: F) -> float:
    # correctly rounded Fraction -> float (Python's float(Fraction) rounds correctly)
    return float(fr)


def split(fr: F, parts=2):
    out = []
    rest = fr
    for _ in range(parts):
        d = to_double(rest)
        out.append(d)
        rest = rest - F(d)
    return out


def hx(d: float) -> str:
    return float.hex(d) if d != 0 else "0.0"


def cody_waite(fr: F, bits=33):
    """Split fr into 3 doubles; the first two carry `bits` significant bits so
    k*p1 and k*p2 are exact for |k| < 2**(53-bits)."""
    out = []
    rest = fr
    for i in range(2):
        d = to_double(rest)
        m, e = float.hex(d), None
        # truncate d to `bits` significant bits
        import math
        ex = math.frexp(d)[1]
        scale = 2.0 ** (bits - ex)
        t = float(int(d * scale)) / scale
        out.append(t)
        rest = rest - F(t)
    out.append(to_double(rest))
    return out


def main():
    pi = pi_fraction()
    lines = ["// Generated by gen_crmath_tables.py -- do not edit.",
             "// Double-double (hi, lo) splits, exact hex-float literals.", "#pragma once", "",
             "namespace bgt {", "namespace cr {", ""]

    def arr(name, vals):
        body = []
        for v in vals:
            h, l = split(v)
            body.append(f"    {{{hx(h)}, {hx(l)}}},")
        # device pass reads __constant__ memory, host passes a static table
        lines.append("#ifdef __CUDACC__")
        lines.append(f"__constant__ double {name}_dev[{len(vals)}][2] = {{")
        lines.extend(body)
        lines.append("};")
        lines.append("#endif")
        lines.append(f"static const double {name}_host[{len(vals)}][2] = {{")
        lines.extend(body)
        lines.append("};")
        lines.append("#ifdef __CUDA_ARCH__")
        lines.append(f"#define {name} {name}_dev")
        lines.append("#else")
        lines.append(f"#define {name} {name}_host")
        lines.append("#endif")

    # sin: (-1)^k / (2k+1)!,  k = 0..16
    arr("SIN_C", [F((-1) ** k, factorial(2 * k + 1)) for k in range(17)])
    # cos: (-1)^k / (2k)!,  k = 0..16
    arr("COS_C", [F((-1) ** k, factorial(2 * k)) for k in range(17)])
    # sinh: 1 / (2k+1)!, cosh: 1 / (2k)!,  k = 0..16
    arr("SINH_C", [F(1, factorial(2 * k + 1)) for k in range(17)])
    arr("COSH_C", [F(1, factorial(2 * k)) for k in range(17)])
    # exp: 1 / k!,  k = 0..40
    arr("EXP_C", [F(1, factorial(k)) for k in range(41)])
    # asin: (2k)! / (4^k (k!)^2 (2k+1)),  k = 0..39
    arr("ASIN_C", [F(factorial(2 * k), 4 ** k * factorial(k) ** 2 * (2 * k + 1)) for k in range(40)])
    # atan: (-1)^k / (2k+1),  k = 0..39
    arr("ATAN_C", [F((-1) ** k, 2 * k + 1) for k in range(40)])
    # scalar constants (no arrays, so usable from both passes)
    h, l = split(pi)
    lines.append(f"#define BGT_CR_PI_HI {hx(h)}")
    lines.append(f"#define BGT_CR_PI_LO {hx(l)}")
    h, l = split(pi / 2)
    lines.append(f"#define BGT_CR_PIO2_HI {hx(h)}")
    lines.append(f"#define BGT_CR_PIO2_LO {hx(l)}")
    h, l = split(2 / pi)
    lines.append(f"#define BGT_CR_TWO_OVER_PI {hx(h)}")
    p = cody_waite(pi / 2)
    lines.append("// pi/2 = CW1 + CW2 + CW3; CW1 and CW2 carry 33 significant bits")
    lines.append(f"#define BGT_CR_PIO2_CW1 {hx(p[0])}")
    lines.append(f"#define BGT_CR_PIO2_CW2 {hx(p[1])}")
    lines.append(f"#define BGT_CR_PIO2_CW3 {hx(p[2])}")
    # residual of the 3-part split, for the error bound
    lines += ["", "}  // namespace cr", "}  // namespace bgt", ""]
    print("\n".join(lines))


if __name__ == "__main__":
    main()
