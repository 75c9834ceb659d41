"""Generate overlap_taylor_table.h: the Taylor coefficients of the Slater overlap integral about one width.

With a = l, b = l (1 + t) and x = r/l the closed form S = F/(8 pi r),
F = 4 a^2 b^2 (e_a - e_b)/D^3 + r (a e_a + b e_b)/D^2, D = b^2 - a^2, is expanded in t with exact rational
arithmetic:  pi l^3 e^x S = sum_n t^n sum_k VALUE[n][k] x^k, and the derivative table follows from
d/dr [e^-x P(x)] = e^-x (P'(x) - P(x))/l.  These are the coefficients the InteraxFF order-2 scheme evaluates
(openmmapi/include/internal/InteraxPairTerms.h:87-113 lists them for orders 0..6).

Run:  python gen_overlap_taylor.py > overlap_taylor_table.h
"""
import sympy as sp

ORDER, TERMS = 6, 9
t, x = sp.symbols("t x")
b = 1 + t
u = x * t / (1 + t)
D = b ** 2 - 1
F_ex = 4 * b ** 2 * (1 - sp.exp(u)) / D ** 3 + x * (1 + b * sp.exp(u)) / D ** 2   # F e^x in units of l
series = sp.series(F_ex / (8 * x), t, 0, ORDER + 1).removeO()
value = []
for n in range(ORDER + 1):
    poly = sp.Poly(sp.expand(sp.simplify(series.coeff(t, n))), x)
    coeffs = [poly.coeff_monomial(x ** k) for k in range(TERMS)]
    value.append(coeffs)
deriv = [[(k + 1) * value[n][k + 1] - value[n][k] if k + 1 < TERMS else -value[n][k] for k in range(TERMS)]
         for n in range(ORDER + 1)]


def fmt(q):
    return "%.17gf" % float(q) if q != 0 else "0.0f"


print("// Generated by gen_overlap_taylor.py from the closed form of the Slater overlap integral (exact rationals).")
print("// pi l^3 e^x S = sum_n t^n sum_k VALUE[n][k] x^k;  DERIV[n][k] = (k+1) VALUE[n][k+1] - VALUE[n][k].")
print("#pragma once")
print("namespace ix {")
for name, table in (("kOverlapTaylorValue", value), ("kOverlapTaylorDeriv", deriv)):
    print(f"__device__ __constant__ const float {name}[{ORDER + 1}][{TERMS}] = {{")
    for n in range(ORDER + 1):
        print("    {" + ", ".join(fmt(q) for q in table[n]) + "},")
    print("};")
print("}  // namespace ix")
