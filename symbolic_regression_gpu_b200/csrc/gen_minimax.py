"""Derives the polynomial coefficients of sr_math.cuh (build-time helper).

Remez exchange algorithm (E. Ya. Remez, 1934) for the weighted minimax
polynomial p of degree n on [a, b]: find c_0..c_n and the levelled error E
with w(x_k) (f(x_k) - p(x_k)) = (-1)^k E on n + 2 reference points, move the
points to the extrema of the error, repeat.  Evaluated in 40-digit arithmetic
(mpmath), so the only rounding left is that of the coefficients to float,
which the exhaustive accuracy test on the device (tests/test_gpu_math.py)
covers.

    python symbolic_regression_gpu_b200/csrc/gen_minimax.py

prints, for
  * sin r = r + r^3 S(z), z = r^2, |r| <= pi/4, S of degree 2, weight: the
    relative error of sin;
  * cos r = 1 + z (-1/2 + z C(z)), C of degree 2, weight: relative error of
    cos;
  * log(1 + f) = f - f^2/2 + f^3 R(f), f in [sqrt(1/2) - 1, sqrt(2) - 1], R of
    degree 7, weight: relative error of log1p;
the coefficients and the levelled relative error.
"""
import mpmath as mp

mp.mp.dps = 40


def remez(f, w, a, b, n, iters=30, grid_points=4000):
    m = n + 2
    xs = [(a + b) / 2 - (b - a) / 2 * mp.cos(mp.pi * k / (m - 1)) for k in range(m)]
    vals = []
    for _ in range(iters):
        A = mp.matrix(m, m)
        rhs = mp.matrix(m, 1)
        for k, x in enumerate(xs):
            for i in range(n + 1):
                A[k, i] = x ** i
            A[k, n + 1] = (-1) ** k / w(x)
            rhs[k] = f(x)
        sol = mp.lu_solve(A, rhs)
        c = [sol[i] for i in range(n + 1)]

        def err(x):
            return w(x) * (f(x) - sum(c[i] * x ** i for i in range(n + 1)))
        grid = [a + (b - a) * mp.mpf(k) / grid_points for k in range(grid_points + 1)]
        vals = [err(x) for x in grid]
        ext = []
        for k in range(len(grid)):
            v = vals[k]
            left = vals[k - 1] if k > 0 else None
            right = vals[k + 1] if k < len(grid) - 1 else None
            if (left is None or abs(v) >= abs(left)) and (right is None or abs(v) >= abs(right)):
                ext.append((grid[k], v))
        alt = []
        for x, v in ext:
            if alt and mp.sign(alt[-1][1]) == mp.sign(v):
                if abs(v) > abs(alt[-1][1]):
                    alt[-1] = (x, v)
            else:
                alt.append((x, v))
        while len(alt) > m:
            if abs(alt[0][1]) < abs(alt[-1][1]):
                alt.pop(0)
            else:
                alt.pop()
        if len(alt) < m:
            break
        xs = [x for x, _ in alt]
    return c, max(abs(v) for v in vals)


def main():
    tiny = mp.mpf(10) ** -30
    zmax = (mp.pi / 4) ** 2

    def s_target(z):
        if z == 0:
            return -mp.mpf(1) / 6
        s = mp.sqrt(z)
        return (mp.sin(s) - s) / (z * s)

    def s_weight(z):
        return (z * mp.sqrt(z)) / mp.sin(mp.sqrt(z)) if z > 0 else tiny

    def c_target(z):
        if z == 0:
            return mp.mpf(1) / 24
        return (mp.cos(mp.sqrt(z)) - 1 + z / 2) / z ** 2

    def c_weight(z):
        return z ** 2 / mp.cos(mp.sqrt(z)) if z > 0 else tiny

    lo, hi = mp.sqrt(mp.mpf(1) / 2) - 1, mp.sqrt(2) - 1

    def l_target(f):
        if f == 0:
            return mp.mpf(1) / 3
        return (mp.log1p(f) - f + f ** 2 / 2) / f ** 3

    def l_weight(f):
        return abs(f ** 3 / mp.log1p(f)) if f != 0 else tiny

    for name, tgt, wt, a, b, n in (("sin S", s_target, s_weight, mp.mpf(0), zmax, 2),
                                   ("cos C", c_target, c_weight, mp.mpf(0), zmax, 2),
                                   ("log R", l_target, l_weight, lo, hi, 7)):
        c, e = remez(tgt, wt, a, b, n)
        print(f"{name}: " + ", ".join(mp.nstr(x, 12) for x in c) + f"   (max rel err {mp.nstr(e, 4)})")


if __name__ == "__main__":
    main()
