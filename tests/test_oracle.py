"""The oracle against the reference's own known-answer identities
(tests/TestLinearAlgebra.cpp:36-150, tests/TestCommunication.cpp:166-273) and
against the Schur-complement relations of the even-odd operator (CPU)."""
import numpy as np
import pytest

from leonardym_b200 import synth
from tests.helpers import CONFIGS, links_for, rel


@pytest.fixture(scope="module", params=["su3", "su2adj"])
def cfg(request, oracle):
    dims, rep, eps, kappa, csw = CONFIGS[request.param]
    return dict(dims=dims, kappa=kappa, csw=csw, links=links_for(request.param), geom=oracle.Geometry(dims))


def test_neighbour_tables_plus_minus_one(oracle):
    # TestCommunication.cpp:166-203: sup/sdn move by +-1 mod L in one direction
    dims = (4, 6, 2, 8)
    sup, sdn, coord = oracle.geom_tables(dims)
    L = np.array(dims)
    for mu in range(4):
        e = np.zeros(4, int)
        e[mu] = 1
        assert np.array_equal(coord[sup[:, mu]], (coord + e) % L)
        assert np.array_equal(coord[sdn[:, mu]], (coord - e) % L)
    assert np.array_equal(coord, synth.lex_coords(dims))


def test_gamma5_hermiticity(cfg, oracle):
    x = synth.gaussian_spinor(cfg["dims"], 3, 1)
    y = synth.gaussian_spinor(cfg["dims"], 3, 2)
    for kind, csw in (("DiracWilson", 0.0), ("Improved", cfg["csw"])):
        op = oracle.Operator(cfg["geom"], cfg["links"], kind, cfg["kappa"], csw, True)
        h = np.vdot(y, op.multiply(x)) - np.vdot(op.multiply(y), x)
        assert abs(h) < 1e-12 * np.linalg.norm(x) * np.linalg.norm(y)


def test_csw_zero_and_alpha_zero(cfg, oracle):
    x = synth.gaussian_spinor(cfg["dims"], 3, 3)
    w = oracle.Operator(cfg["geom"], cfg["links"], "DiracWilson", cfg["kappa"], 0.0, True)
    c = oracle.Operator(cfg["geom"], cfg["links"], "Improved", cfg["kappa"], 0.0, True)
    assert np.array_equal(w.multiply(x), c.multiply(x))
    assert np.array_equal(w.multiply_add(x, x, 0.0), c.multiply_add(x, x, 0.0))
    c2 = oracle.Operator(cfg["geom"], cfg["links"], "Improved", cfg["kappa"], cfg["csw"], True)
    assert rel(c2.multiply_add(x, x, 0.0), c2.multiply(x)) < 1e-15


def test_gamma5_flag_relation(cfg, oracle):
    x = synth.gaussian_spinor(cfg["dims"], 3, 4)
    q = oracle.Operator(cfg["geom"], cfg["links"], "Improved", cfg["kappa"], cfg["csw"], True).multiply(x)
    d = oracle.Operator(cfg["geom"], cfg["links"], "Improved", cfg["kappa"], cfg["csw"], False).multiply(x)
    q[:, 2:] *= -1
    assert rel(q, d) < 1e-15


def test_even_odd_schur_relations(cfg, oracle):
    # D = [[T_ee, -k H_eo], [-k H_oe, T_oo]]; EO multiply = gamma5 (T_oo - k^2 H_oe T_ee^-1 H_eo) on odd
    dims = cfg["dims"]
    D = oracle.Operator(cfg["geom"], cfg["links"], "Improved", cfg["kappa"], cfg["csw"], False)
    E = oracle.Operator(cfg["geom"], cfg["links"], "EvenOddImproved", cfg["kappa"], cfg["csw"], False)
    odd = synth.lex_coords(dims).sum(axis=1) % 2 == 1
    x = synth.gaussian_spinor(dims, 3, 5)
    xo = x.copy()
    xo[~odd] = 0
    # y_e solves T_ee y_e = k H_eo x_o, i.e. D (y_e + x_o) has zero even part
    Dx = D.multiply(xo)
    ye = E.even_even_inverse(-Dx)
    ye[odd] = 0
    full = ye + xo
    Dfull = D.multiply(full)
    assert np.abs(Dfull[~odd]).max() < 1e-13
    Sx = E.multiply(x)
    assert rel(Sx[odd], Dfull[odd]) < 1e-13
    assert np.array_equal(Sx[~odd], x[~odd])


def test_schur_shadow_identity(cfg, oracle):
    # S^+ = g5 S g5 on the odd sites (S is gamma5-hermitian, as D is): <rhat, S p> equals
    # <g5 S g5 rhat, p>, which is how the block BiCGStab knows alpha = rho / <rhat, S p> from
    # the update pass that forms p, before S p is formed
    dims = cfg["dims"]
    E = oracle.Operator(cfg["geom"], cfg["links"], "EvenOddImproved", cfg["kappa"], cfg["csw"], False)
    odd = synth.lex_coords(dims).sum(axis=1) % 2 == 1
    rhat = synth.gaussian_spinor(dims, 3, 7)
    p = synth.gaussian_spinor(dims, 3, 8)
    rhat[~odd] = 0
    p[~odd] = 0

    def g5(v):
        w = v.copy()
        w[:, 2:] *= -1
        return w

    Sp = E.multiply(p)
    what = g5(E.multiply(g5(rhat)))
    lhs = np.vdot(rhat[odd], Sp[odd])
    rhs = np.vdot(what[odd], p[odd])
    assert abs(lhs - rhs) < 1e-12 * np.linalg.norm(rhat) * np.linalg.norm(Sp)


def test_solvers_converge(cfg, oracle):
    b = synth.gaussian_spinor(cfg["dims"], 3, 6)
    eps = 1e-20 * float(np.vdot(b, b).real)
    Q2 = oracle.Operator(cfg["geom"], cfg["links"], "SquareImproved", cfg["kappa"], cfg["csw"], True)
    rc, x, steps = oracle.cg(Q2, b, eps, 5000)
    assert rc == 1 and np.linalg.norm(b - Q2.multiply(x)) ** 2 < 1.01 * eps
    rc, x2, _ = oracle.bicgstab(Q2, b, eps, 5000)
    assert rc == 1 and rel(x2, x) < 1e-7
    D = oracle.Operator(cfg["geom"], cfg["links"], "Improved", cfg["kappa"], cfg["csw"], False)
    rc, x3, _ = oracle.preconditioned_bicgstab(D, b, eps, 5000)
    assert rc == 1 and np.linalg.norm(b - D.multiply(x3)) / np.linalg.norm(b) < 1e-8
    shifts = [0.3, 0.03]
    rc, sols, _ = oracle.me_multishift(Q2, b, shifts, eps)
    assert rc == 1
    rc, sols2, _ = oracle.mmmr_multishift(Q2, b, shifts, eps)
    assert rc == 1
    for s, a, c in zip(shifts, sols, sols2):
        assert np.linalg.norm(b - Q2.multiply_add(a, a, s)) / np.linalg.norm(b) < 2e-10
        assert np.linalg.norm(b - Q2.multiply_add(c, c, s)) / np.linalg.norm(b) < 2e-10


def test_meson_contractions_restatements(oracle):
    # the vectorised contraction equals the loop-for-loop restatement of MesonCorrelator.cpp:98-157
    rng = np.random.default_rng(3)
    dims = (2, 2, 2, 4)
    V = 32
    props = [rng.standard_normal((V, 4, 3)) + 1j * rng.standard_normal((V, 4, 3)) for _ in range(12)]
    for a, b in zip(oracle.meson_contractions(props, dims), oracle.meson_contractions_loops(props, dims)):
        assert np.max(np.abs(a - b)) <= 1e-13 * np.max(np.abs(b))
    src = oracle.point_sources(dims)
    assert len(src) == 12 and all(s[0, k % 4, k // 4] == 1 and np.count_nonzero(s) == 1 for k, s in enumerate(src))


def test_z2_noise_restatement(oracle):
    n = oracle.z2_noise((4, 4, 4, 8), 11, 2)
    assert n.shape == (4 * 4 * 4 * 8, 4, 3) and set(np.unique(n.real)) == {-1.0, 1.0} and not n.imag.any()
    assert abs(n.real.mean()) < 0.1
    assert not np.array_equal(n, oracle.z2_noise((4, 4, 4, 8), 11, 3))
    assert np.array_equal(n, oracle.z2_noise((4, 4, 4, 8), 11, 2))
