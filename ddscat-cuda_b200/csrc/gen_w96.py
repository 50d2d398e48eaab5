"""Writes w96.inc: exp(-2 pi i m / 96), m = 0..95, as 21-digit decimal literals.

96 is divisible by every in-register DFT size the line FFTs use (2, 3, 4, 8,
12, 16, 24, 32), so wk<K>(m) = W96^(m * 96 / K).  The values are computed with
Python's decimal module at 40 digits (pi from Machin's formula, cos and sin
from their Taylor series), so every literal is correctly rounded.

    python gen_w96.py > w96.inc
"""
from decimal import Decimal, getcontext

getcontext().prec = 40


def arctan_inv(x):
    """arctan(1/x) for integer x by its Taylor series."""
    x = Decimal(x)
    x2 = x * x
    term = Decimal(1) / x
    total, n, sign = term, 1, 1
    while True:
        term /= x2
        n += 2
        sign = -sign
        t = term / n
        if t < Decimal(10) ** -45:
            return total
        total += sign * t


PI = 4 * (4 * arctan_inv(5) - arctan_inv(239))


def cos_sin(a):
    c, s = Decimal(0), Decimal(0)
    term, k = Decimal(1), 0
    while abs(term) > Decimal(10) ** -45:
        if k % 4 == 0:
            c += term
        elif k % 4 == 1:
            s += term
        elif k % 4 == 2:
            c -= term
        else:
            s -= term
        k += 1
        term = term * a / k
    return c, s


def lit(v):
    if v == 0:
        return "0.0"
    q = f"{v:.21f}".rstrip("0")
    return q + "0" if q.endswith(".") else q


def main():
    re, im = [], []
    for m in range(96):
        c, s = cos_sin(2 * PI * m / 96)
        if m % 24 == 0:
            c, s = [Decimal(1), Decimal(0), Decimal(-1), Decimal(0)][m // 24], [Decimal(0), Decimal(1), Decimal(0), Decimal(-1)][m // 24]
        re.append(c)
        im.append(-s)
    out = ["// exp(-2*pi*i*m/96) = w96re(m) + i*w96im(m); exact decimal literals (21 digits), from gen_w96.py."]
    for name, vals in (("w96re", re), ("w96im", im)):
        out.append(f"DDB_HD constexpr double {name}(int m) {{")
        out.append("  switch (((m % 96) + 96) % 96) {")
        for m, v in enumerate(vals):
            out.append(f"    case {m}: return {lit(v)};")
        out.append("    default: return 0.0;")
        out.append("  }")
        out.append("}")
    print("\n".join(out))


if __name__ == "__main__":
    main()
