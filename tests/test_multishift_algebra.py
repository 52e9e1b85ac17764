"""The mixed multishift CG's windowed updates, restated in numpy on the oracle's even-odd
operator (CPU).  Shifted multishift CG (the Jegerlehner recurrences of MMMRMultishiftSolver /
the multishift CG) updates every shift's x_i and p_i once per step.  The GPU solver instead
keeps, per shift, the coefficients of x_i and p_i on the directions P_i at the start of a
window and on the window's residuals R_0..R_{m-1}, and applies them in one pass per 8 steps
(ms_window_step / ms_flush_kernel).  Both orders give the same x_i and p_i."""
import numpy as np
import pytest

from leonardym_b200 import synth
from tests.helpers import CONFIGS, links_for

WIN = 8


def _square_schur(oracle):
    dims, rep, eps, kappa, csw = CONFIGS["su3"]
    E = oracle.Operator(oracle.Geometry(dims), links_for("su3"), "EvenOddImproved", kappa, csw, False)
    odd = synth.lex_coords(dims).sum(axis=1) % 2 == 1

    def S(v):
        w = np.zeros((len(odd),) + v.shape[1:], np.complex128)
        w[odd] = v
        return E.multiply(w)[odd]

    def g5(v):
        w = v.copy()
        w[:, 2:] *= -1
        return w

    return dims, odd, (lambda v: g5(S(g5(S(v)))))  # S^+ S, Hermitian positive definite


class Scalars:
    """The base CG's scalars and the shifted ones (zeta, alpha_i, beta_i), step by step."""

    def __init__(self, sigma, rr):
        self.sigma = np.asarray(sigma, float)
        self.zeta = np.ones_like(self.sigma)
        self.zeta_prev = np.ones_like(self.sigma)
        self.alpha, self.beta, self.rr = 1.0, 0.0, rr

    def alphas(self, pAp):
        a, am1 = self.rr / pAp, self.alpha
        z, zp = self.zeta, self.zeta_prev
        den = zp * am1 * (1.0 + self.sigma * a) + a * self.beta * (zp - z)
        zn = z * zp * am1 / den
        alpha_s = a * zn / z
        self.zeta_prev, self.zeta, self.alpha = z, zn, a
        return a, alpha_s

    def betas(self, rr_new):
        self.beta = rr_new / self.rr
        self.rr = rr_new
        return self.beta * (self.zeta / self.zeta_prev) ** 2


def per_step(A, b, sigma, n):
    sc = Scalars(sigma, np.vdot(b, b).real)
    r, p = b.copy(), b.copy()
    xs = [np.zeros_like(b) for _ in sigma]
    ps = [b.copy() for _ in sigma]
    for _ in range(n):
        Ap = A(p)
        a, alpha_s = sc.alphas(np.vdot(p, Ap).real)
        r = r - a * Ap
        beta_s = sc.betas(np.vdot(r, r).real)
        for i in range(len(sigma)):
            xs[i] = xs[i] + alpha_s[i] * ps[i]
            ps[i] = sc.zeta[i] * r + beta_s[i] * ps[i]
        p = r + sc.beta * p
    return xs, ps


def windowed(A, b, sigma, n):
    sc = Scalars(sigma, np.vdot(b, b).real)
    ns = len(sigma)
    r, p = b.copy(), b.copy()
    xs = [np.zeros_like(b) for _ in sigma]
    P = [b.copy() for _ in sigma]
    R = []
    cx = np.zeros((ns, WIN + 1))
    cp = np.zeros((ns, WIN + 1))
    cp[:, 0] = 1.0

    def flush():
        for i in range(ns):
            xs[i] = xs[i] + cx[i, 0] * P[i] + sum(cx[i, j + 1] * R[j] for j in range(len(R)))
            P[i] = cp[i, 0] * P[i] + sum(cp[i, j + 1] * R[j] for j in range(len(R)))

    for _ in range(n):
        Ap = A(p)
        a, alpha_s = sc.alphas(np.vdot(p, Ap).real)
        r = r - a * Ap
        beta_s = sc.betas(np.vdot(r, r).real)
        m = len(R)
        R.append(r.copy())  # the ring slot of this step's residual
        for i in range(ns):  # ms_window_step
            cx[i, : m + 1] += alpha_s[i] * cp[i, : m + 1]
            cp[i, : m + 1] *= beta_s[i]
            cp[i, m + 1] = sc.zeta[i]
        p = r + sc.beta * p  # the base direction, materialised every step
        if len(R) == WIN:
            flush()
            R.clear()
            cx[:] = 0.0
            cp[:] = 0.0
            cp[:, 0] = 1.0
    if R:
        flush()
    return xs, P


@pytest.mark.parametrize("n", [5, 8, 20])
def test_windowed_updates_equal_per_step_updates(oracle, n):
    dims, odd, A = _square_schur(oracle)
    b = synth.gaussian_spinor(dims, 3, 31)[odd]
    sigma = [0.0, 1e-3, 0.05, 0.5, 2.0]
    x1, p1 = per_step(A, b, sigma, n)
    x2, p2 = windowed(A, b, sigma, n)
    for i in range(len(sigma)):
        assert np.linalg.norm(x1[i] - x2[i]) <= 1e-12 * np.linalg.norm(x1[i]), (n, i)
        assert np.linalg.norm(p1[i] - p2[i]) <= 1e-12 * np.linalg.norm(p1[i]), (n, i)


def test_shifted_solutions_converge(oracle):
    dims, odd, A = _square_schur(oracle)
    b = synth.gaussian_spinor(dims, 3, 32)[odd]
    sigma = [0.0, 0.01, 0.3]
    xs, _ = windowed(A, b, sigma, 120)
    for s, x in zip(sigma, xs):
        assert np.linalg.norm(b - A(x) - s * x) <= 1e-10 * np.linalg.norm(b), s
