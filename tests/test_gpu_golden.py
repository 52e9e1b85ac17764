"""The GPU library against the golden fixtures produced by the reference's own
code (tests/golden/make_golden.py), through the C ABI."""
import os

import numpy as np
import pytest

import leonardym_b200 as L
from tests.helpers import rel

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
CLS = {"DiracWilson": L.DiracWilsonOperator, "Improved": L.ImprovedDiracWilsonOperator,
       "EvenOddImproved": L.EvenOddImprovedDiracWilsonOperator, "SquareDiracWilson": L.SquareDiracWilsonOperator,
       "SquareImproved": L.SquareImprovedDiracWilsonOperator,
       "SquareEvenOddImproved": L.SquareEvenOddImprovedDiracWilsonOperator}


@pytest.fixture(scope="module", params=["su3", "su2adj"])
def gold(request):
    d = dict(np.load(os.path.join(HERE, "golden", f"reference_{request.param}.npz")))
    d["rep"] = request.param
    dims = tuple(int(v) for v in d["dims"])
    d["lat"] = L.Lattice(dims, request.param)
    d["gid"] = d["lat"].upload(d["links"])
    yield d
    d["lat"].close()


def make(g, kind, gamma5=True):
    op = CLS[kind](g["lat"], float(g["kappa"]))
    if "Wilson" not in kind:
        op.setCSW(float(g["csw"]))
    op.setGamma5(gamma5)
    op.setLattice(g["gid"])
    return op


@pytest.mark.parametrize("kind", list(CLS))
def test_multiply_against_reference(gold, kind):
    for g5 in (1, 0):
        assert rel(make(gold, kind, bool(g5)).multiply(gold["x"]), gold[f"multiply/{kind}/{g5}"]) < 1e-13
    if kind != "EvenOddImproved":
        got = make(gold, kind).multiplyAdd(gold["x"], gold["y"], complex(gold["alpha"]))
        assert rel(got, gold[f"multiply_add/{kind}"]) < 1e-13


def test_field_strength_against_reference(gold):
    assert np.abs(make(gold, "Improved").field_strength() - gold["field_strength"]).max() < 1e-14


def test_fundamental_links_against_reference(gold):
    if gold["rep"] != "su2adj":
        pytest.skip("adjoint map only")
    lat = gold["lat"]
    gid = lat.upload_fundamental(gold["su2_fundamental"], "fermion_antiperiodic")
    a = make(gold, "Improved")
    b = L.ImprovedDiracWilsonOperator(lat, float(gold["kappa"]), float(gold["csw"]))
    b.setLattice(lat.upload(gold["antiperiodic"]))
    a.setLattice(gid)
    assert rel(a.multiply(gold["x"]), b.multiply(gold["x"])) < 1e-14


def test_solvers_against_reference(gold):
    x = gold["x"]
    prec = 1e-20 * float(np.vdot(x, x).real)
    cg = L.ConjugateGradient()
    cg.setPrecision(prec)
    cg.setMaximumSteps(5000)
    sol = gold["lat"].new_vector()
    assert cg.solve(make(gold, "SquareImproved"), x, sol)
    assert abs(cg.getLastSteps() - int(gold["steps/cg"])) <= 2 and rel(sol, gold["solve/cg"]) < 1e-8
    for solver, kind, g5, key in ((L.BiConjugateGradient(), "SquareImproved", True, "bicgstab"),
                                  (L.PreconditionedBiCGStab(), "Improved", False, "preconditioned_bicgstab")):
        solver.setPrecision(prec)
        solver.setMaximumSteps(5000)
        sol = gold["lat"].new_vector()
        assert solver.solve(make(gold, kind, g5), x, sol)
        ref_steps = int(gold[f"steps/{key}"])
        assert abs(solver.getLastSteps() - ref_steps) <= max(3, ref_steps // 4)
        assert rel(sol, gold[f"solve/{key}"]) < 1e-8
    for alg in ("mass_estrapolation", "minimal_residual"):
        ms = L.MultishiftSolver.getInstance(alg)
        ms.setPrecision(prec)
        sols = []
        assert ms.solve(make(gold, "SquareImproved"), x, sols, list(gold["shifts"]))
        for a, b in zip(sols, gold[f"multishift/{alg}"]):
            assert rel(a, b) < 1e-8


def test_rational_evaluate_golden(gold):
    # RationalApproximation::evaluate against the compiled reference's own output
    x = gold["x"]
    prec = 1e-20 * float(np.vdot(x, x).real)
    for kind in ("SquareImproved", "SquareEvenOddImproved"):
        ra = L.RationalApproximation(gold["rational/alphas"], gold["rational/betas"])
        ra.setPrecision(prec)
        ra.setMaximumRecursion(5000)
        out = gold["lat"].new_vector()
        ra.evaluate(make(gold, kind), out, x)
        assert rel(out, gold[f"rational/{kind}"]) < 1e-8


def test_fermion_force_golden(gold):
    # the GPU fermion force against the compiled reference's FermionForce::derivative
    dims = gold["lat"].dims
    for kind, cls in (("DiracWilson", L.DiracWilsonOperator), ("Improved", L.ImprovedDiracWilsonOperator)):
        op = cls(gold["lat"], float(gold["kappa"]))
        if kind == "Improved":
            op.setCSW(float(gold["csw"]))
        op.setLattice(gold["gid"])
        f = np.zeros((int(np.prod(dims)), 4, 3, 3), np.complex128)
        op.getForce().derivative(f, gold["x"], gold["y"], 0.7)
        ref = gold[f"force/{kind}"]
        assert np.max(np.abs(f[:64] - ref)) <= 1e-13 * np.max(np.abs(ref))
