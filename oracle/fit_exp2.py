"""Coefficients of the deterministic 2^f used by the rasterisers' blend
(exp2_det in del-splat_b200/csrc/common.cuh and exp2_det_f32 in
oracle/oracle.cpp).

p(f) = 1 + c1 f + c2 f^2 + ... + c5 f^5 approximates 2^f on [-1/2, 1/2];
p(0) = 1 exactly.  c1..c5 minimise the largest relative error
|p(f) / 2^f - 1| over a dense grid, written as a linear program (minimax
fit; scipy's HiGHS solver).  The result is about 6.8e-8 before the
coefficients are rounded to float; the float coefficients evaluated in float
with fused multiply-adds stay within 2.2e-7 over every float of the interval
(one coefficient fewer than the degree-6 Taylor polynomial of e^(f ln 2),
whose float evaluation reaches 2.25e-7).

    python oracle/fit_exp2.py
"""
import numpy as np
from scipy.optimize import linprog


def fit(degree: int = 5, points: int = 4001):
    g = np.linspace(-0.5, 0.5, points)
    w = 2.0 ** -g
    A = np.stack([g ** j * w for j in range(1, degree + 1)], 1)  # relative error is A c + (w - 1)
    base = w - 1.0
    ones = np.ones((len(g), 1))
    A_ub = np.vstack([np.hstack([A, -ones]), np.hstack([-A, -ones])])
    b_ub = np.concatenate([-base, base])
    cost = np.zeros(degree + 1)
    cost[-1] = 1.0
    r = linprog(cost, A_ub=A_ub, b_ub=b_ub, bounds=[(None, None)] * (degree + 1), method="highs")
    return r.x[:-1], r.x[-1]


if __name__ == "__main__":
    c, err = fit()
    print(f"max relative error (grid, unrounded): {err:.3e}")
    for j, v in enumerate(c, 1):
        print(f"c{j} = {float(np.float32(v))!r}f")
