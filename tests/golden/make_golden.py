"""Generates tests/golden/reference_<rep>.npz by running LeonardYM's own hot path
compiled from its sources (oracle/_ref, built by oracle/build_ref.sh) on seeded
inputs.  Run from the repository root:  python tests/golden/make_golden.py

The fixtures pin the oracle restatement (tests/test_oracle_pins.py) and the GPU
library (tests/test_gpu_golden.py) on machines where the reference is absent.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from leonardym_b200 import synth  # noqa: E402
from oracle import ref as R  # noqa: E402

DIMS = (4, 4, 2, 4)
CASES = {"su3": (0.13, 1.0, 0.3), "su2adj": (0.18, 1.5, 0.3)}
KINDS = ["DiracWilson", "Improved", "EvenOddImproved", "SquareDiracWilson", "SquareImproved", "SquareEvenOddImproved"]


def make(rep):
    kappa, csw, eps = CASES[rep]
    links = synth.fermion_links(DIMS, rep, eps, 4321)
    x = synth.gaussian_spinor(DIMS, 3, 11)
    y = synth.gaussian_spinor(DIMS, 3, 12)
    ref = R.Reference(DIMS, links, rep)
    out = {"dims": np.array(DIMS), "kappa": kappa, "csw": csw, "links": links, "x": x, "y": y}
    alpha = 0.37 - 0.21j
    out["alpha"] = alpha
    for kind in KINDS:
        c = 0.0 if "Wilson" in kind else csw
        for g5 in (1, 0):
            out[f"multiply/{kind}/{g5}"] = ref.multiply(kind, x, kappa, c, bool(g5))
        if kind != "EvenOddImproved":
            out[f"multiply_add/{kind}"] = ref.multiply_add(kind, x, y, alpha, kappa, c, True)
    out["field_strength"] = ref.field_strength(kappa, csw)
    prec = 1e-20 * float(np.vdot(x, x).real)
    for solver, kind, g5 in (("cg", "SquareImproved", True), ("bicgstab", "SquareImproved", True),
                             ("preconditioned_bicgstab", "Improved", False)):
        rc, sol, steps = ref.solve(kind, solver, x, prec, 5000, kappa, csw, g5)
        assert rc == 1, (rep, solver)
        out[f"solve/{solver}"] = sol
        out[f"steps/{solver}"] = steps
    rc, sol, steps = ref.solve("SquareImproved", "bicgstab_shifted", x, prec, 5000, kappa, csw, True, shift=0.05)
    assert rc == 1
    out["solve/bicgstab_shifted"] = sol
    shifts = np.array([0.5, 0.05, 0.01])
    out["shifts"] = shifts
    for alg in ("mass_estrapolation", "minimal_residual"):
        rc, sols = ref.multishift("SquareImproved", alg, x, shifts, prec, 5000, kappa, csw, True)
        assert rc == 1, alg
        out[f"multishift/{alg}"] = np.stack(sols)
    # RationalApproximation::evaluate (RationalApproximation.cpp:18-42) with the
    # mass-estrapolation multishift, on the squared full and even-odd operators
    out["rational/alphas"] = np.array([0.31, 0.12, 0.047, 0.011])
    out["rational/betas"] = np.array([0.9, 0.17, 0.03, 0.004])
    for kind in ("SquareImproved", "SquareEvenOddImproved"):
        rc, r = ref.rational_evaluate(kind, "mass_estrapolation", out["rational/alphas"], out["rational/betas"], x,
                                      prec, 5000, kappa, csw, True)
        assert rc == 1
        out[f"rational/{kind}"] = r
    # FermionForce::derivative of the Wilson and improved forces (hmc_forces/), weight 0.7 on a
    # zero field; the first 64 sites are kept
    V = int(np.prod(DIMS))
    zero = np.zeros((V, 4, 3, 3), np.complex128)
    for kind in ("DiracWilson", "Improved"):
        out[f"force/{kind}"] = ref.fermion_force(kind, kappa, csw, x, y, 0.7, zero)[:64]
    # BiCGStab(l) and BiCGStab with a preconditioner operator (BiConjugateGradient.cpp:11-317)
    for l in (2, 4):
        rc, sol, steps = ref.solve2("SquareImproved", "bicgstab_l", x, prec, 5000, kappa, csw, True, l=l)
        out[f"rc/bicgstab_l{l}"], out[f"solve/bicgstab_l{l}"], out[f"steps/bicgstab_l{l}"] = rc, sol, steps
    rc, sol, steps = ref.solve2("Improved", "bicgstab_precond", x, prec, 5000, kappa, csw, False,
                                pre_kind="DiracWilson", pre_kappa=0.05, pre_csw=0.0)
    out["rc/bicgstab_precond"], out["solve/bicgstab_precond"], out["steps/bicgstab_precond"] = rc, sol, steps
    # ChronologicalMultishiftSolver: its first shift is plain CG from zero; the later shifts
    # start from a guess built from vectors the reference never initialises, so only the
    # first shift is a fixture (and whether the others came out finite)
    rc, sols = ref.multishift("SquareImproved", "chronological_mass_estrapolation", x, shifts, prec, 5000, kappa,
                              csw, True)
    out["multishift/chronological/0"] = sols[0]
    out["multishift/chronological/finite"] = np.array([bool(np.isfinite(s).all()) for s in sols])
    sup, sdn = R.neighbours(DIMS, rep)
    out["sup"], out["sdn"] = sup, sdn
    if rep == "su2adj":
        fund = synth.su2_links(DIMS, eps, 4321)
        out["su2_fundamental"] = fund
        out["su2_adjoint"] = R.to_adjoint(fund)
        out["antiperiodic"] = R.antiperiodic(DIMS, out["su2_adjoint"], rep)
    else:
        out["antiperiodic"] = R.antiperiodic(DIMS, synth.su3_links(DIMS, eps, 4321), rep)
    return out


if __name__ == "__main__":
    here = os.path.dirname(os.path.abspath(__file__))
    for rep in CASES:
        data = make(rep)
        np.savez_compressed(os.path.join(here, f"reference_{rep}.npz"), **data)
        print(rep, "written", sum(np.asarray(v).nbytes for v in data.values()) // 1024, "KiB raw")
