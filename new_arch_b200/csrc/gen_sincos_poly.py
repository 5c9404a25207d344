"""Derives the coefficients of the engine's Box-Muller sine and cosine.

The angle of a Box-Muller pair is 2*pi*v for a 24-bit v; its quadrant is split
off in integers, leaving g in [-1/2, 1/2] and the quarter-turn angle pi*g/2.
sin(pi g / 2) = g * S(g^2) with S of degree 3 (odd powers g .. g^7) and
cos(pi g / 2) = 1 + g^2 * C(g^2) with C of degree 3 (g^2 .. g^8), fitted by
least squares on Chebyshev nodes of g (absolute error as the weight: the
values are multiplied by the Box-Muller radius).  The coefficients, rounded to
FP32, are pasted into new_arch_b200/csrc/scmf_math.cuh and oracle/scmf_oracle.c;
run this script to reproduce them.
"""
import numpy as np

DEG = 3


def _nodes(n=4000):
    k = np.arange(n)
    g = 0.5 * np.cos(np.pi * (k + 0.5) / n)
    return g[np.abs(g) > 1e-6]


def fit_sin():
    g = _nodes()
    x = g * g
    y = np.sin(0.5 * np.pi * g) / g
    w = np.abs(g)                      # error of S scaled to absolute error of g * S
    V = np.vander(x, DEG + 1, increasing=True)
    c, *_ = np.linalg.lstsq(V * w[:, None], y * w, rcond=None)
    return np.float32(c)


def fit_cos():
    g = _nodes()
    x = g * g
    y = (np.cos(0.5 * np.pi * g) - 1.0) / x
    w = x                              # error of C scaled to absolute error of 1 + g^2 C
    V = np.vander(x, DEG + 1, increasing=True)
    c, *_ = np.linalg.lstsq(V * w[:, None], y * w, rcond=None)
    return np.float32(c)


if __name__ == "__main__":
    for name, c in (("sin S", fit_sin()), ("cos C", fit_cos())):
        print(name)
        for i, v in enumerate(c):
            print(f"  c{i} = {float(v).hex()}  # {float(v):.9g}")
