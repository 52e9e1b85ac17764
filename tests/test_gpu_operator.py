"""GPU parity of the operator application against the oracle (through the C ABI).

Bar: FP64 stencil within 1e-13 relative of the oracle, FP32 within 1e-6, FP16
within 1e-2 (storage precision 2^-11 with per-site norms); layout tables bit-exact.
"""
import numpy as np
import pytest

import leonardym_b200 as L
from leonardym_b200 import synth
from tests.helpers import CONFIGS, links_for, rel

pytestmark = pytest.mark.gpu

KINDS = ["DiracWilson", "Improved", "EvenOddImproved", "SquareDiracWilson", "SquareImproved",
         "SquareEvenOddImproved"]
GPU_CLASS = {
    "DiracWilson": L.DiracWilsonOperator, "Improved": L.ImprovedDiracWilsonOperator,
    "EvenOddImproved": L.EvenOddImprovedDiracWilsonOperator, "SquareDiracWilson": L.SquareDiracWilsonOperator,
    "SquareImproved": L.SquareImprovedDiracWilsonOperator,
    "SquareEvenOddImproved": L.SquareEvenOddImprovedDiracWilsonOperator,
}


@pytest.fixture(scope="module", params=["su3", "su2adj"])
def setup(request, oracle):
    name = request.param
    dims, rep, eps, kappa, csw = CONFIGS[name]
    links = links_for(name)
    lat = L.Lattice(dims, rep)
    gid = lat.upload(links)
    geom = oracle.Geometry(dims)
    yield dict(name=name, dims=dims, rep=rep, kappa=kappa, csw=csw, links=links, lat=lat, gid=gid, geom=geom)
    lat.close()


def make(setup, kind, gamma5, oracle):
    gpu = GPU_CLASS[kind](setup["lat"])
    gpu.setKappa(setup["kappa"])
    if kind not in ("DiracWilson", "SquareDiracWilson"):
        gpu.setCSW(setup["csw"])
    gpu.setGamma5(gamma5)
    gpu.setLattice(setup["gid"])
    csw = 0.0 if "Wilson" in kind else setup["csw"]
    orc = oracle.Operator(setup["geom"], setup["links"], kind, setup["kappa"], csw, gamma5)
    return gpu, orc


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("gamma5", [True, False])
def test_multiply_matches_oracle(setup, kind, gamma5, oracle):
    gpu, orc = make(setup, kind, gamma5, oracle)
    x = synth.gaussian_spinor(setup["dims"], 3, 7)
    out = setup["lat"].new_vector()
    gpu.multiply(out, x)
    assert rel(out, orc.multiply(x)) < 1e-13


@pytest.mark.parametrize("kind", ["DiracWilson", "Improved", "SquareDiracWilson", "SquareImproved",
                                  "SquareEvenOddImproved"])
@pytest.mark.parametrize("gamma5", [True, False])
def test_multiply_add_matches_oracle(setup, kind, gamma5, oracle):
    gpu, orc = make(setup, kind, gamma5, oracle)
    x = synth.gaussian_spinor(setup["dims"], 3, 8)
    y = synth.gaussian_spinor(setup["dims"], 3, 9)
    alpha = 0.37 - 0.21j
    out = gpu.multiplyAdd(setup["lat"].new_vector(), x, y, alpha)
    assert rel(out, orc.multiply_add(x, y, alpha)) < 1e-13
    # multiplyAdd(alpha = 0) == multiply (tests/TestLinearAlgebra.cpp:141-144)
    out0 = gpu.multiplyAdd(setup["lat"].new_vector(), x, y, 0.0)
    assert rel(out0, gpu.multiply(x)) < 1e-15


def test_even_odd_multiply_add_unsupported(setup, oracle):
    gpu, _ = make(setup, "EvenOddImproved", True, oracle)
    x = synth.gaussian_spinor(setup["dims"], 3, 10)
    with pytest.raises(L.LymError):
        gpu.multiplyAdd(setup["lat"].new_vector(), x, x, 1.0)


def test_field_strength_matches_oracle(setup, oracle):
    gpu, orc = make(setup, "Improved", True, oracle)
    F = gpu.field_strength()
    Fo = orc.field_strength()
    assert F.shape == Fo.shape
    assert np.abs(F - Fo).max() < 1e-14


def test_gamma5_hermiticity(setup, oracle):
    # TestLinearAlgebra.cpp:36-57: |<y, Q x> - <Q y, x>|^2
    for kind in ("DiracWilson", "Improved"):
        gpu, _ = make(setup, kind, True, oracle)
        x = synth.gaussian_spinor(setup["dims"], 3, 11)
        y = synth.gaussian_spinor(setup["dims"], 3, 12)
        h = np.vdot(y, gpu.multiply(x)) - np.vdot(gpu.multiply(y), x)
        assert abs(h) < 1e-11 * np.linalg.norm(x) * np.linalg.norm(y)


def test_csw_zero_equals_wilson(setup, oracle):
    # TestLinearAlgebra.cpp:122-140
    lat = setup["lat"]
    w = L.DiracWilsonOperator(lat, setup["kappa"])
    w.setLattice(setup["gid"])
    c = L.ImprovedDiracWilsonOperator(lat, setup["kappa"], 0.0)
    c.setLattice(setup["gid"])
    x = synth.gaussian_spinor(setup["dims"], 3, 13)
    assert rel(w.multiply(x), c.multiply(x)) < 1e-15
    assert rel(w.multiplyAdd(x, x, 0.0), c.multiplyAdd(x, x, 0.0)) < 1e-15


@pytest.mark.parametrize("precision,tol", [("single", 1e-6), ("half", 1e-2)])
@pytest.mark.parametrize("kind", ["Improved", "EvenOddImproved", "SquareImproved"])
def test_sloppy_precision_stencil(setup, precision, tol, kind, oracle):
    gpu, orc = make(setup, kind, True, oracle)
    x = synth.gaussian_spinor(setup["dims"], 3, 14)
    assert rel(gpu.multiply_precision(x, precision), orc.multiply(x)) < tol


@pytest.mark.parametrize("kind", ["DiracWilson", "Improved", "EvenOddImproved", "SquareImproved"])
@pytest.mark.parametrize("gamma5", [True, False])
def test_eight_real_links_stencil(setup, kind, gamma5, oracle):
    """The FP32 stencil on SU(3) links stored in 8 reals (lym_set_link_format) against the FP64
    oracle, 1e-6 as the 12-real format; SU(2) adjoint links refuse the format."""
    lat = setup["lat"]
    if setup["rep"] != "su3":
        with pytest.raises(L.LymError):
            lat.set_link_format(8)
        return
    gpu, orc = make(setup, kind, gamma5, oracle)
    x = synth.gaussian_spinor(setup["dims"], 3, 15)
    want = orc.multiply(x)
    try:
        lat.set_link_format(8)
        e8 = rel(gpu.multiply_precision(x, "single"), want)
    finally:
        lat.set_link_format(12)
    e12 = rel(gpu.multiply_precision(x, "single"), want)
    print(f"{kind} gamma5={gamma5}: FP32 stencil error 8 reals {e8:.2e}, 12 reals {e12:.2e}")
    assert e8 < 1e-6 and e12 < 1e-6


def test_eight_real_links_mixed_solve(setup, oracle):
    """The mixed-precision even-odd CG with its FP32 inner iterations on 8-real links still
    reaches the FP64 true residual 1e-10 (re-measured with the oracle)."""
    if setup["rep"] != "su3":
        return
    lat = setup["lat"]
    gpu, orc = make(setup, "Improved", False, oracle)
    b = synth.gaussian_spinor(setup["dims"], 3, 16)
    x = lat.new_vector()
    try:
        lat.set_link_format(8)
        assert L.EvenOddConjugateGradient("single", 1e-10).solve(gpu, b, x)
    finally:
        lat.set_link_format(12)
    assert np.linalg.norm(b - orc.multiply(x)) / np.linalg.norm(b) <= 1e-10


def test_neighbour_tables_bit_exact(setup, oracle):
    sup, sdn = setup["lat"].neighbour_tables()
    osup, osdn, _ = oracle.geom_tables(setup["dims"])
    assert np.array_equal(sup, osup) and np.array_equal(sdn, osdn)


def test_stencil_indices_match_reference_tables(setup, oracle):
    idx = setup["lat"].stencil_indices()
    osup, osdn, coord = oracle.geom_tables(setup["dims"])
    Vh = idx.shape[1]
    for p in range(2):
        lex = idx[p, :, 0]
        assert np.array_equal(lex >> 1, np.arange(Vh))
        assert np.all(coord[lex].sum(axis=1) % 2 == p)
        for mu in range(4):
            assert np.array_equal(idx[p, :, 1 + 2 * mu], osup[lex, mu] >> 1)
            assert np.array_equal(idx[p, :, 2 + 2 * mu], osdn[lex, mu] >> 1)


def test_upload_fundamental_matches_host_conversion(setup, oracle):
    lat = setup["lat"]
    dims = setup["dims"]
    if setup["rep"] == "su3":
        fund = synth.su3_links(dims, 0.3, 99)
        host = synth.antiperiodic_bc(fund, dims)
    else:
        fund = synth.su2_links(dims, 0.3, 99)
        host = synth.antiperiodic_bc(synth.su2_to_adjoint(fund), dims)
    g1 = lat.upload_fundamental(fund, "fermion_antiperiodic")
    g2 = lat.upload(host)
    a = L.ImprovedDiracWilsonOperator(lat, 0.12, 1.1)
    a.setLattice(g1)
    b = L.ImprovedDiracWilsonOperator(lat, 0.12, 1.1)
    b.setLattice(g2)
    x = synth.gaussian_spinor(dims, 3, 15)
    assert rel(a.multiply(x), b.multiply(x)) < 1e-14
