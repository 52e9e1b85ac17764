"""The block BiCGStab's reordered iteration, restated in numpy on the oracle's even-odd
Schur operator (CPU): the per-RHS recursion the batched kernels run is the same algorithm
as textbook BiCGStab (inverters/BiConjugateGradient.cpp:321-507), only reordered so that
each stencil launch can carry a fused epilogue:
  alpha = rho / <S^+ rhat, p> is known from the update pass that forms p, before S p;
  s = r - alpha v is formed where v = S p is produced;
  <t, s>, |t|^2, <rhat, s>, <rhat, t> are summed where t = S s is produced, giving
  omega, rho' = <rhat, s> - omega <rhat, t> and beta without another pass."""
import numpy as np
import pytest

from leonardym_b200 import synth
from tests.helpers import CONFIGS, links_for


def _schur(oracle, name):
    dims, rep, eps, kappa, csw = CONFIGS[name]
    E = oracle.Operator(oracle.Geometry(dims), links_for(name), "EvenOddImproved", kappa, csw, False)
    odd = synth.lex_coords(dims).sum(axis=1) % 2 == 1

    def S(v):
        w = np.zeros((len(odd),) + v.shape[1:], np.complex128)
        w[odd] = v
        return E.multiply(w)[odd]

    def g5(v):
        w = v.copy()
        w[:, 2:] *= -1
        return w

    return dims, odd, S, g5


def textbook(S, b, n):
    x = np.zeros_like(b)
    r = b.copy()
    rhat = r.copy()
    p = r.copy()
    rho = np.vdot(rhat, r)
    hist = []
    for _ in range(n):
        v = S(p)
        alpha = rho / np.vdot(rhat, v)
        s = r - alpha * v
        t = S(s)
        omega = np.vdot(t, s) / np.vdot(t, t)
        x = x + alpha * p + omega * s
        r = s - omega * t
        rho_new = np.vdot(rhat, r)
        beta = (rho_new / rho) * (alpha / omega)
        p = r + beta * (p - omega * v)
        rho = rho_new
        hist.append(np.vdot(r, r).real)
    return x, hist


def reordered(S, g5, b, n):
    x = np.zeros_like(b)
    r = b.copy()
    rhat = r.copy()
    p = r.copy()
    rho = np.vdot(rhat, r)
    what = g5(S(g5(rhat)))  # S^+ rhat, formed whenever rhat changes
    alpha = rho / np.vdot(what, p)
    hist = []
    for _ in range(n):
        v = S(p)
        s = r - alpha * v  # epilogue of the launch that forms v
        t = S(s)
        ts, tt = np.vdot(t, s), np.vdot(t, t).real  # epilogue of the launch that forms t
        hs, ht = np.vdot(rhat, s), np.vdot(rhat, t)
        omega = ts / tt
        rho_new = hs - omega * ht
        beta = (rho_new / rho) * (alpha / omega)
        x = x + alpha * p + omega * s  # one update pass: x, r, p and <S^+ rhat, p>
        r = s - omega * t
        p = r + beta * (p - omega * v)
        alpha = rho_new / np.vdot(what, p)
        rho = rho_new
        hist.append(np.vdot(r, r).real)
    return x, hist


@pytest.mark.parametrize("name", ["su3", "su2adj"])
def test_reordered_bicgstab_is_textbook_bicgstab(oracle, name):
    dims, odd, S, g5 = _schur(oracle, name)
    b = synth.gaussian_spinor(dims, 3, 21)[odd]
    # a few iterations: on the SU(2) adjoint case (kappa 0.18, an indefinite Schur operator on
    # which BiCGStab does not converge) the two orders' rounding differences grow ~10x per step
    n = 8
    x1, h1 = textbook(S, b, n)
    x2, h2 = reordered(S, g5, b, n)
    # same iterates up to rounding
    assert np.allclose(h1, h2, rtol=1e-8, atol=0.0)
    assert np.linalg.norm(x1 - x2) <= 1e-9 * np.linalg.norm(x1)


def test_reordered_bicgstab_converges_to_the_schur_solution(oracle):
    dims, odd, S, g5 = _schur(oracle, "su3")
    b = synth.gaussian_spinor(dims, 3, 22)[odd]
    x, hist = reordered(S, g5, b, 60)
    k = next(i for i, h in enumerate(hist) if h < 1e-24 * np.vdot(b, b).real)
    x, _ = reordered(S, g5, b, k + 1)
    assert np.linalg.norm(b - S(x)) <= 1e-10 * np.linalg.norm(b)
