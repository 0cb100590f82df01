"""The reference's order-of-accuracy test, as a reusable computation.

CongFD1.0/AccuracyTest.cpp:4-83: g(x) = x^k exp(0.75 (x - 1)) with k = 1 on
[-1, 1], n = 2/h cells, cell centres -1 + (i + 1/2) h, ghost values from g,
face values by TCNS5 interpolation of g, MND6 difference; L1, L2 and Linf of
the error against g'(x), and the orders between consecutive h.
"""
import numpy as np

HS = [2.0 / 10.0, 2.0 / 20.0, 2.0 / 30.0, 2.0 / 40.0, 2.0 / 50.0, 2.0 / 60.0]


def g(x, k=1.0):
    return x ** k * np.exp(0.75 * (x - 1))


def dg(x, k=1.0):
    return np.exp(0.75 * (-1 + x)) * k * x ** (k - 1) + 0.75 * np.exp(0.75 * (-1 + x)) * x ** k


def samples(h):
    n = int((1.0 - -1.0) / h)
    x = -1.0 + (np.arange(-4, n + 4) + 0.5) * h
    return n, g(x), -1.0 + (np.arange(n) + 0.5) * h


def errors(deriv, h):
    n, q, xc = samples(h)
    e = np.abs(deriv(q, h) - dg(xc))
    return e.mean(), np.sqrt((e * e).mean()), e.max()


def orders(errs, hs):
    errs = np.array(errs)
    return [np.log(errs[i] / errs[i + 1]) / np.log(hs[i] / hs[i + 1]) for i in range(len(hs) - 1)]
