"""Regenerates the float minimax coefficients of gft_math.cuh (run: python gft_math_fit.py).

Remez exchange (E. Ya. Remez, 1934) for the polynomial forms the kernels evaluate
after the reduction to |r| <= pi/2 (s = r^2):
  sin r = r + r^3 P(s),   P of degree 3 (sin of degree 9), weight r^3 / sin r: the
                          relative error of sin;
  cos r = 1 + s Q(s),     Q of degree 4 (cos of degree 10), weight s: the absolute
                          error of cos.
Prints the coefficients (lowest order first), the fit's own maximum error, and the
maximum error of the float evaluation (coefficients rounded to float, Horner with
single-rounding fused multiply-adds) against the double-precision function.
"""
import numpy as np

HALF_PI_SQ = (np.pi / 2) ** 2


def remez(f, w, a, b, deg, iters=40, grid=200001):
    n = deg + 2
    k = np.arange(n)
    s = (a + b) / 2 + (b - a) / 2 * np.cos(np.pi * k[::-1] / (n - 1))
    xs = np.linspace(a, b, grid)
    for _ in range(iters):
        A = np.zeros((n, n))
        for i in range(n):
            A[i, :deg + 1] = s[i] ** np.arange(deg + 1)
            A[i, deg + 1] = (-1) ** i / w(s[i])
        sol = np.linalg.solve(A, f(s))
        c = sol[:deg + 1]
        err = w(xs) * (f(xs) - np.polyval(c[::-1], xs))
        ext = [0] + [i for i in range(1, grid - 1) if (err[i] - err[i - 1]) * (err[i + 1] - err[i]) <= 0] + [grid - 1]
        pts = []
        for i in sorted(ext):
            if pts and np.sign(err[i]) == np.sign(err[pts[-1]]):
                if abs(err[i]) > abs(err[pts[-1]]):
                    pts[-1] = i
            else:
                pts.append(i)
        while len(pts) > n:
            pts.pop(0 if abs(err[pts[0]]) < abs(err[pts[-1]]) else -1)
        if len(pts) < n:
            break
        s = xs[pts]
    return c, float(np.max(np.abs(err)))


def sin_p(s):
    r = np.sqrt(s)
    small = s < 1e-6
    return np.where(small, -1 / 6 + s / 120 - s * s / 5040, (np.sin(r) - r) / np.where(small, 1.0, r ** 3))


def sin_w(s):
    r = np.sqrt(np.maximum(s, 1e-30))
    return np.maximum(r ** 3 / np.sin(r), 1e-30)


def cos_q(s):
    small = s < 1e-6
    return np.where(small, -0.5 + s / 24 - s * s / 720, (np.cos(np.sqrt(s)) - 1) / np.where(small, 1.0, s))


def horner_f32(c, r, sin):
    f32 = np.float32
    r = f32(r)
    r2 = f32(r * r)
    p = f32(c[-1])
    for k in c[-2::-1]:
        p = f32(np.float64(p) * np.float64(r2) + np.float64(f32(k)))
    if sin:
        return float(f32(np.float64(f32(p * r2)) * np.float64(r) + np.float64(r)))
    return float(f32(np.float64(p) * np.float64(r2) + 1.0))


if __name__ == "__main__":
    cs, es = remez(sin_p, sin_w, 0.0, HALF_PI_SQ, 3)
    cc, ec = remez(cos_q, lambda s: np.maximum(s, 1e-10), 0.0, HALF_PI_SQ, 4)
    rs = np.linspace(-np.pi / 2, np.pi / 2, 100001)
    es32 = max(abs(horner_f32(cs, r, True) - np.sin(np.float32(r))) / max(abs(np.sin(np.float32(r))), 1e-30)
               for r in rs if r != 0)
    ec32 = max(abs(horner_f32(cc, r, False) - np.cos(np.float32(r))) for r in rs)
    print("sin r = r + r^3 P(r^2): P =", [float(np.float32(v)) for v in cs], "fit rel", es, "float eval rel", es32)
    print("cos r = 1 + r^2 Q(r^2): Q =", [float(np.float32(v)) for v in cc], "fit abs", ec, "float eval abs", ec32)
