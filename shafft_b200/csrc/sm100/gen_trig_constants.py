"""Generate trig_constants.h: cos/sin(2*pi*m/p) for the register butterflies.

Values are evaluated with Python's decimal module at 50 significant digits
(Taylor series after reduction to [0, pi/4]) and printed with 21 significant
digits, so the double literal is the correctly rounded value.  Run:
    python gen_trig_constants.py > trig_constants.h
"""
from decimal import Decimal, getcontext

getcontext().prec = 60
PRIMES = [3, 5, 7, 11, 13]
POW2 = [8, 16, 32]


def pi():
    # Chudnovsky-free: Machin's formula, plenty for 60 digits
    def arctan_inv(x):
        x = Decimal(x)
        total, term, n, sign = Decimal(0), 1 / x, 1, 1
        x2 = x * x
        while True:
            t = term / n
            if t < Decimal(10) ** -58:
                break
            total += sign * t
            term /= x2
            n += 2
            sign = -sign
        return total
    return 4 * (4 * arctan_inv(5) - arctan_inv(239))


PI = pi()


def sin_cos(x):
    s, c = Decimal(0), Decimal(0)
    term = x
    n = 1
    while abs(term) > Decimal(10) ** -58:
        s += term
        term = -term * x * x / ((n + 1) * (n + 2))
        n += 2
    term = Decimal(1)
    n = 0
    while abs(term) > Decimal(10) ** -58:
        c += term
        term = -term * x * x / ((n + 1) * (n + 2))
        n += 2
    return s, c


def cs(m, p):
    s, c = sin_cos(2 * PI * m / p)
    return c, s


print("// Generated by gen_trig_constants.py -- do not edit.")
print("// cos/sin(2*pi*m/p), correctly rounded to double.")
print("#pragma once")
print("namespace shafft_sm100 {")
print("__host__ __device__ constexpr double trig_cos(int p, int m) {")
print("  switch (p * 64 + m) {")
for p in PRIMES + POW2:
    for m in range(p):
        c, s = cs(m, p)
        print(f"    case {p * 64 + m}: return {format(c, '.21e')};")
print("    default: return 0.0;")
print("  }")
print("}")
print("__host__ __device__ constexpr double trig_sin(int p, int m) {")
print("  switch (p * 64 + m) {")
for p in PRIMES + POW2:
    for m in range(p):
        c, s = cs(m, p)
        print(f"    case {p * 64 + m}: return {format(s, '.21e')};")
print("    default: return 0.0;")
print("  }")
print("}")
print("}  // namespace shafft_sm100")
