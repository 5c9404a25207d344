"""Derives the coefficients of the engine's single-precision log.

log(m) for m in [sqrt(1/2), sqrt(2)) is written log1p(t) = t + t^2 Q(t) with
t = m - 1 (exact in FP32) and Q a degree-8 polynomial fitted by weighted least
squares on Chebyshev nodes (relative error of the final result as the
weight).  The coefficients, rounded to FP32, are pasted into
new_arch_b200/csrc/scmf_math.cuh and oracle/scmf_oracle.c; run this script to
reproduce them.
"""
import numpy as np

DEG = 8


def fit():
    a, b = np.sqrt(0.5) - 1.0, np.sqrt(2.0) - 1.0
    k = np.arange(4000)
    t = 0.5 * (a + b) + 0.5 * (b - a) * np.cos(np.pi * (k + 0.5) / k.size)
    t = t[np.abs(t) > 1e-6]
    q = (np.log1p(t) - t) / (t * t)
    w = t * t / np.abs(np.log1p(t))        # error of Q scaled to relative error of log1p
    V = np.vander(t, DEG + 1, increasing=True)
    c, *_ = np.linalg.lstsq(V * w[:, None], q * w, rcond=None)
    return np.float32(c)


if __name__ == "__main__":
    c = fit()
    for i, v in enumerate(c):
        print(f"c{i} = {float(v).hex()}  # {float(v):.9g}")
