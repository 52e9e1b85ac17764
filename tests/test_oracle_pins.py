"""Pins the oracle to the reference itself: against the golden fixtures that the
reference's own code (compiled from its sources) produced, and, where that
compiled reference is present, against it live on other inputs (CPU)."""
import os

import numpy as np
import pytest

from leonardym_b200 import synth
from tests.helpers import rel

HERE = os.path.dirname(os.path.abspath(__file__))
KINDS = ["DiracWilson", "Improved", "EvenOddImproved", "SquareDiracWilson", "SquareImproved", "SquareEvenOddImproved"]


@pytest.fixture(scope="module", params=["su3", "su2adj"])
def gold(request, oracle):
    d = dict(np.load(os.path.join(HERE, "golden", f"reference_{request.param}.npz")))
    d["rep"] = request.param
    d["geom"] = oracle.Geometry(tuple(int(v) for v in d["dims"]))
    return d


def op(oracle, g, kind, gamma5=True):
    c = 0.0 if "Wilson" in kind else float(g["csw"])
    return oracle.Operator(g["geom"], g["links"], kind, float(g["kappa"]), c, gamma5)


@pytest.mark.parametrize("kind", KINDS)
def test_multiply_pinned(gold, kind, oracle):
    tol = 1e-15 if "EvenOdd" in kind else 0.0  # EO: the 12x12 inverse differs in the last bit
    for g5 in (1, 0):
        assert rel(op(oracle, gold, kind, bool(g5)).multiply(gold["x"]), gold[f"multiply/{kind}/{g5}"]) <= tol
    if kind != "EvenOddImproved":
        got = op(oracle, gold, kind).multiply_add(gold["x"], gold["y"], complex(gold["alpha"]))
        assert rel(got, gold[f"multiply_add/{kind}"]) <= tol


def test_field_strength_pinned(gold, oracle):
    assert np.array_equal(op(oracle, gold, "Improved").field_strength(), gold["field_strength"])


def test_layout_and_boundary_pinned(gold, oracle):
    sup, sdn, _ = oracle.geom_tables(tuple(gold["dims"]))
    assert np.array_equal(sup, gold["sup"]) and np.array_equal(sdn, gold["sdn"])
    dims = tuple(int(v) for v in gold["dims"])
    if gold["rep"] == "su2adj":
        assert np.abs(synth.su2_to_adjoint(gold["su2_fundamental"]) - gold["su2_adjoint"]).max() < 1e-15
        assert np.array_equal(synth.antiperiodic_bc(gold["su2_adjoint"], dims), gold["antiperiodic"])
    else:
        assert np.array_equal(synth.antiperiodic_bc(synth.su3_links(dims, 0.3, 4321), dims), gold["antiperiodic"])


def test_solvers_pinned(gold, oracle):
    x = gold["x"]
    prec = 1e-20 * float(np.vdot(x, x).real)
    rc, sol, steps = oracle.cg(op(oracle, gold, "SquareImproved"), x, prec, 5000)
    assert rc == 1 and steps == int(gold["steps/cg"]) and rel(sol, gold["solve/cg"]) < 1e-12
    # BiCGStab iteration counts move with the summation order of the (OpenMP) reductions
    rc, sol, steps = oracle.bicgstab(op(oracle, gold, "SquareImproved"), x, prec, 5000)
    ref_steps = int(gold["steps/bicgstab"])
    assert rc == 1 and abs(steps - ref_steps) <= max(3, ref_steps // 4) and rel(sol, gold["solve/bicgstab"]) < 1e-8
    rc, sol, _ = oracle.bicgstab(op(oracle, gold, "SquareImproved"), x, prec, 5000, shift=0.05)
    assert rc == 1 and rel(sol, gold["solve/bicgstab_shifted"]) < 1e-8
    rc, sol, steps = oracle.preconditioned_bicgstab(op(oracle, gold, "Improved", False), x, prec, 5000)
    ref_steps = int(gold["steps/preconditioned_bicgstab"])
    assert rc == 1 and abs(steps - ref_steps) <= max(3, ref_steps // 4)
    assert rel(sol, gold["solve/preconditioned_bicgstab"]) < 1e-8


def test_multishift_pinned(gold, oracle):
    x = gold["x"]
    prec = 1e-20 * float(np.vdot(x, x).real)
    shifts = list(gold["shifts"])
    rc, sols, _ = oracle.me_multishift(op(oracle, gold, "SquareImproved"), x, shifts, prec)
    assert rc == 1
    for a, b in zip(sols, gold["multishift/mass_estrapolation"]):
        assert rel(a, b) < 1e-8
    rc, sols, _ = oracle.mmmr_multishift(op(oracle, gold, "SquareImproved"), x, shifts, prec)
    assert rc == 1
    for a, b in zip(sols, gold["multishift/minimal_residual"]):
        assert rel(a, b) < 1e-8


@pytest.mark.parametrize("rep", ["su3", "su2adj"])
def test_live_against_compiled_reference(rep, oracle):
    from oracle import ref as R
    if not R.available(rep):
        pytest.skip("oracle/_ref not built (needs the reference sources)")
    dims = (2, 4, 4, 6)
    kappa, csw = (0.125, 1.3) if rep == "su3" else (0.17, 1.2)
    links = synth.fermion_links(dims, rep, 0.35, 99)
    x = synth.gaussian_spinor(dims, 3, 98)
    ref = R.Reference(dims, links, rep)
    g = oracle.Geometry(dims)
    for kind in KINDS:
        c = 0.0 if "Wilson" in kind else csw
        got = oracle.Operator(g, links, kind, kappa, c, True).multiply(x)
        assert rel(got, ref.multiply(kind, x, kappa, c, True)) <= 1e-15
    # BasicDiracWilsonOperator equals DiracWilsonOperator (TestLinearAlgebra.cpp:145-150)
    assert rel(ref.multiply("BasicDiracWilson", x, kappa), ref.multiply("DiracWilson", x, kappa)) < 1e-15


def test_bicgstab_variants_pinned(gold, oracle):
    """BiCGStab(l) and BiCGStab with a preconditioner operator (BiConjugateGradient.cpp:11-317)
    where the reference converged; the same steps, the same solution."""
    x = gold["x"]
    prec = 1e-20 * float(np.vdot(x, x).real)
    for l in (2, 4):
        if int(gold[f"rc/bicgstab_l{l}"]) != 1:
            continue
        rc, sol, steps = oracle.bicgstab_l(op(oracle, gold, "SquareImproved"), l, x, prec, 5000)
        ref_steps = int(gold[f"steps/bicgstab_l{l}"])
        assert rc == 1 and abs(steps - ref_steps) <= max(3, ref_steps // 4), (l, steps, ref_steps)
        assert rel(sol, gold[f"solve/bicgstab_l{l}"]) < 1e-8
    if int(gold["rc/bicgstab_precond"]) == 1:
        pre = oracle.Operator(gold["geom"], gold["links"], "DiracWilson", 0.05, 0.0, False)
        rc, sol, steps = oracle.bicgstab_precond(op(oracle, gold, "Improved", False), pre, x, prec, 5000)
        assert rc == 1 and steps == int(gold["steps/bicgstab_precond"])
        assert rel(sol, gold["solve/bicgstab_precond"]) < 1e-10


def test_chronological_multishift_pinned(gold, oracle):
    """ChronologicalMultishiftSolver: its first shift (CG from zero) equals the reference's;
    the later shifts, which the reference builds from uninitialised storage (non-finite in
    its run), solve their systems."""
    x = gold["x"]
    prec = 1e-20 * float(np.vdot(x, x).real)
    shifts = list(gold["shifts"])
    A = op(oracle, gold, "SquareImproved")
    rc, sols = oracle.chrono_multishift(A, x, shifts, prec)
    assert rc == 1
    assert rel(sols[0], gold["multishift/chronological/0"]) < 1e-12
    assert not gold["multishift/chronological/finite"][1:].all()
    for s, sh in zip(sols, shifts):
        r = x - A.multiply(s) - sh * s
        assert float(np.vdot(r, r).real) < 4 * prec


def test_rational_evaluate_pinned(gold, oracle):
    # RationalApproximation::evaluate (RationalApproximation.cpp:18-42) on the squared full and
    # even-odd operators, mass-estrapolation multishift
    x = gold["x"]
    prec = 1e-20 * float(np.vdot(x, x).real)
    alphas, betas = list(gold["rational/alphas"]), list(gold["rational/betas"])
    for kind in ("SquareImproved", "SquareEvenOddImproved"):
        rc, out = oracle.rational_evaluate(op(oracle, gold, kind), alphas, betas, x, prec, 5000)
        assert rc == 1
        assert rel(out, gold[f"rational/{kind}"]) < 1e-10
    assert abs(oracle.rational_value(alphas, betas, 0.5 + 0.1j) -
               sum(a / (0.5 + 0.1j + b) for a, b in zip(alphas, betas))) < 1e-15


def test_fermion_force_pinned(gold, oracle):
    # FermionForce::derivative of DiracWilsonFermionForce / ImprovedFermionForce (hmc_forces/)
    from oracle import force as OF
    dims = tuple(int(d) for d in gold["dims"])
    zero = np.zeros((int(np.prod(dims)), 4, 3, 3), np.complex128)
    for kind, clover in (("DiracWilson", False), ("Improved", True)):
        f = OF.fermion_force(dims, gold["links"], gold["x"], gold["y"], float(gold["kappa"]), float(gold["csw"]),
                             clover, 0.7, zero)
        ref = gold[f"force/{kind}"]
        assert np.max(np.abs(f[:64] - ref)) <= 1e-13 * np.max(np.abs(ref))
