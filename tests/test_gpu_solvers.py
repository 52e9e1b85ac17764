"""GPU solvers through the C ABI against the oracle's restatement of the
reference solvers.  Every solve's true residual ||b - A x|| / ||b|| is
re-measured with the FP64 oracle operator."""
import numpy as np
import pytest

import leonardym_b200 as L
from leonardym_b200 import synth
from tests.helpers import CONFIGS, links_for, rel

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=["su3", "su2adj"])
def setup(request, oracle):
    name = request.param
    dims, rep, eps, kappa, csw = CONFIGS[name]
    links = links_for(name)
    lat = L.Lattice(dims, rep)
    gid = lat.upload(links)
    geom = oracle.Geometry(dims)
    b = synth.gaussian_spinor(dims, 3, 21)
    yield dict(dims=dims, rep=rep, kappa=kappa, csw=csw, links=links, lat=lat, gid=gid, geom=geom, b=b)
    lat.close()


def gpu_op(setup, cls, gamma5=True):
    op = cls(setup["lat"], setup["kappa"])
    if cls not in (L.DiracWilsonOperator, L.SquareDiracWilsonOperator):
        op.setCSW(setup["csw"])
    op.setGamma5(gamma5)
    op.setLattice(setup["gid"])
    return op


def true_res(oracle_op, b, x, shift=None):
    ax = oracle_op.multiply(x) if shift is None else oracle_op.multiply_add(x, x, shift)
    return float(np.linalg.norm(b - ax) / np.linalg.norm(b))


def test_cg_square_improved(setup, oracle):
    # ConjugateGradient on D^+D (configs: CG on D^dagger D to 1e-10 relative)
    b = setup["b"]
    eps = (1e-10) ** 2 * float(np.vdot(b, b).real)
    op = gpu_op(setup, L.SquareImprovedDiracWilsonOperator)
    cg = L.ConjugateGradient()
    cg.setPrecision(eps)
    cg.setMaximumSteps(5000)
    x = setup["lat"].new_vector()
    assert cg.solve(op, b, x)
    orc = oracle.Operator(setup["geom"], setup["links"], "SquareImproved", setup["kappa"], setup["csw"], True)
    rc, xo, steps = oracle.cg(orc, b, eps, 5000)
    assert rc == 1
    assert abs(cg.getLastSteps() - steps) <= 2
    assert true_res(orc, b, x) < 1.5e-10
    assert rel(x, xo) < 1e-7


def test_bicgstab_square_improved(setup, oracle):
    b = setup["b"]
    eps = (1e-10) ** 2 * float(np.vdot(b, b).real)
    op = gpu_op(setup, L.SquareImprovedDiracWilsonOperator)
    s = L.BiConjugateGradient()
    s.setPrecision(eps)
    s.setMaximumSteps(5000)
    x = setup["lat"].new_vector()
    assert s.solve(op, b, x)
    orc = oracle.Operator(setup["geom"], setup["links"], "SquareImproved", setup["kappa"], setup["csw"], True)
    rc, xo, steps = oracle.bicgstab(orc, b, eps, 5000)
    assert rc == 1
    # BiCGStab's trajectory depends on the summation order of its reductions: on the
    # ill-conditioned systems the iteration counts drift apart while both converge
    assert abs(s.getLastSteps() - steps) <= max(3, steps // 4)
    assert true_res(orc, b, x) < 1.5e-10
    assert rel(x, xo) < 1e-7


def test_bicgstab_shifted(setup, oracle):
    b = setup["b"]
    eps = (1e-10) ** 2 * float(np.vdot(b, b).real)
    op = gpu_op(setup, L.SquareImprovedDiracWilsonOperator)
    s = L.BiConjugateGradient()
    s.setPrecision(eps)
    s.setMaximumSteps(5000)
    x = setup["lat"].new_vector()
    assert s.solve(op, b, x, shift=0.05)
    orc = oracle.Operator(setup["geom"], setup["links"], "SquareImproved", setup["kappa"], setup["csw"], True)
    assert true_res(orc, b, x, 0.05) < 1.5e-10


@pytest.mark.parametrize("gamma5", [False, True])
def test_preconditioned_bicgstab(setup, gamma5, oracle):
    b = setup["b"]
    prec = (1e-10) ** 2 * float(np.vdot(b, b).real)
    op = gpu_op(setup, L.ImprovedDiracWilsonOperator, gamma5)
    s = L.PreconditionedBiCGStab()
    s.setPrecision(prec)
    s.setMaximumSteps(5000)
    x = setup["lat"].new_vector()
    assert s.solve(op, b, x)
    orc = oracle.Operator(setup["geom"], setup["links"], "Improved", setup["kappa"], setup["csw"], gamma5)
    rc, xo, steps = oracle.preconditioned_bicgstab(orc, b, prec, 5000)
    assert rc == 1
    assert abs(s.getLastSteps() - steps) <= max(3, steps // 4)
    # the even-odd path solves D x = b (gamma5 = false operator) whatever the flag
    D = oracle.Operator(setup["geom"], setup["links"], "Improved", setup["kappa"], setup["csw"], False)
    assert true_res(D, b, x) < 1e-8
    assert rel(x, xo) < 1e-7


@pytest.mark.parametrize("mode", ["double", "single", "half"])
def test_even_odd_cg_true_residual(setup, mode, oracle):
    b = setup["b"]
    op = gpu_op(setup, L.ImprovedDiracWilsonOperator, False)
    s = L.EvenOddConjugateGradient(mode, 1e-10)
    x = setup["lat"].new_vector()
    assert s.solve(op, b, x)
    D = oracle.Operator(setup["geom"], setup["links"], "Improved", setup["kappa"], setup["csw"], False)
    r = true_res(D, b, x)
    assert r <= 1e-10
    assert s.stats.true_residual <= 1e-10
    assert abs(s.stats.true_residual - r) < 1e-11


@pytest.mark.parametrize("mode", ["single", "half"])
@pytest.mark.parametrize("cls", ["Improved", "DiracWilson"])
def test_even_odd_bicgstab_mixed_true_residual(setup, mode, cls, oracle):
    b = setup["b"]
    gcls = L.ImprovedDiracWilsonOperator if cls == "Improved" else L.DiracWilsonOperator
    op = gpu_op(setup, gcls, False)
    s = L.EvenOddBiCGStab(mode, 1e-10)
    x = setup["lat"].new_vector()
    assert s.solve(op, b, x), s.stats.as_dict()
    csw = setup["csw"] if cls == "Improved" else 0.0
    D = oracle.Operator(setup["geom"], setup["links"], cls, setup["kappa"], csw, False)
    r = true_res(D, b, x)
    assert r <= 1e-10
    assert abs(s.stats.true_residual - r) < 1e-11
    assert s.stats.reliable_updates >= 1


def test_even_odd_bicgstab_rejects_guess(setup):
    op = gpu_op(setup, L.ImprovedDiracWilsonOperator, False)
    s = L.EvenOddBiCGStab("single", 1e-10)
    x = setup["lat"].new_vector()
    with pytest.raises(L.LymError):
        s.solve(op, setup["b"], x, initial_guess=setup["b"])


def test_even_odd_cg_wilson(setup, oracle):
    b = setup["b"]
    op = gpu_op(setup, L.DiracWilsonOperator, False)
    s = L.EvenOddConjugateGradient("single", 1e-10)
    x = setup["lat"].new_vector()
    assert s.solve(op, b, x)
    D = oracle.Operator(setup["geom"], setup["links"], "DiracWilson", setup["kappa"], 0.0, False)
    assert true_res(D, b, x) <= 1e-10


def test_multishift_mass_estrapolation(setup, oracle):
    b = setup["b"]
    shifts = [0.5, 0.1, 0.01]
    eps = (1e-10) ** 2 * float(np.vdot(b, b).real)
    op = gpu_op(setup, L.SquareImprovedDiracWilsonOperator)
    ms = L.MultishiftSolver.getInstance("mass_estrapolation")
    ms.setPrecision(eps)
    sols = []
    assert ms.solve(op, b, sols, shifts)
    orc = oracle.Operator(setup["geom"], setup["links"], "SquareImproved", setup["kappa"], setup["csw"], True)
    rc, osols, _ = oracle.me_multishift(orc, b, shifts, eps)
    for x, xo, s in zip(sols, osols, shifts):
        assert true_res(orc, b, x, s) < 1.5e-10
        assert rel(x, xo) < 1e-7


def test_multishift_cg(setup, oracle):
    b = setup["b"]
    shifts = list(np.logspace(-4, 0, 12))
    eps = (1e-10) ** 2 * float(np.vdot(b, b).real)
    op = gpu_op(setup, L.SquareImprovedDiracWilsonOperator)
    ms = L.MultishiftSolver.getInstance("multishift_cg")
    ms.setPrecision(eps)
    ms.setMaxSteps(10000)
    sols = []
    assert ms.solve(op, b, sols, shifts)
    orc = oracle.Operator(setup["geom"], setup["links"], "SquareImproved", setup["kappa"], setup["csw"], True)
    for x, s in zip(sols, shifts):
        assert true_res(orc, b, x, s) < 3e-10


def test_multishift_minimal_residual(setup, oracle):
    # MMMRMultishiftSolver: base system = last shift; negative shifts by separate CG
    b = setup["b"]
    shifts = [-0.001, 0.5, 0.1, 0.02]
    eps = (1e-10) ** 2 * float(np.vdot(b, b).real)
    op = gpu_op(setup, L.SquareImprovedDiracWilsonOperator)
    ms = L.MultishiftSolver.getInstance("minimal_residual")
    ms.setPrecision(eps)
    ms.setMaxSteps(10000)
    sols = []
    assert ms.solve(op, b, sols, shifts)
    orc = oracle.Operator(setup["geom"], setup["links"], "SquareImproved", setup["kappa"], setup["csw"], True)
    rc, osols, steps = oracle.mmmr_multishift(orc, b, shifts, eps, 10000)
    assert rc == 1
    for x, xo, s in zip(sols, osols, shifts):
        assert true_res(orc, b, x, s) < 2e-10
        assert rel(x, xo) < 1e-7


@pytest.mark.parametrize("l", [2, 4])
def test_bicgstab_l_matches_oracle(setup, l, oracle):
    # BiConjugateGradient::solve(dirac, source, solution, int l) (BiConjugateGradient.cpp:130-317)
    b = setup["b"]
    eps = (1e-10) ** 2 * float(np.vdot(b, b).real)
    orc = oracle.Operator(setup["geom"], setup["links"], "SquareImproved", setup["kappa"], setup["csw"], True)
    rc, xo, steps = oracle.bicgstab_l(orc, l, b, eps, 3000)
    s = L.BiConjugateGradient()
    s.setPrecision(eps)
    s.setMaximumSteps(3000)
    x = setup["lat"].new_vector()
    ok = s.solve(gpu_op(setup, L.SquareImprovedDiracWilsonOperator), b, x, l=l)
    if rc != 1:  # the algorithm does not converge on this system in the oracle either
        assert not ok or true_res(orc, b, x) < 1.5e-10
        return
    assert ok
    # BiCGStab(l)'s iteration count follows rounding closely on these systems (two
    # FP64 implementations with different summation orders differ by tens of percent), so the
    # checked properties are convergence, the true residual and the solution
    assert s.getLastSteps() <= 2 * steps + 10
    assert true_res(orc, b, x) < 1.5e-10
    assert rel(x, xo) < 1e-7


def test_bicgstab_preconditioned_matches_oracle(setup, oracle):
    # BiConjugateGradient::solve(dirac, source, solution, preconditioner) (BiConjugateGradient.cpp:11-128)
    b = setup["b"]
    eps = (1e-10) ** 2 * float(np.vdot(b, b).real)
    orc = oracle.Operator(setup["geom"], setup["links"], "Improved", setup["kappa"], setup["csw"], False)
    pre_o = oracle.Operator(setup["geom"], setup["links"], "DiracWilson", 0.05, 0.0, False)
    rc, xo, steps = oracle.bicgstab_precond(orc, pre_o, b, eps, 3000)
    pre = L.DiracWilsonOperator(setup["lat"], 0.05)
    pre.setGamma5(False)
    pre.setLattice(setup["gid"])
    s = L.BiConjugateGradient()
    s.setPrecision(eps)
    s.setMaximumSteps(3000)
    x = setup["lat"].new_vector()
    ok = s.solve(gpu_op(setup, L.ImprovedDiracWilsonOperator, False), b, x, preconditioner=pre)
    assert ok == (rc == 1)
    if rc == 1:
        assert abs(s.getLastSteps() - steps) <= max(3, steps // 4)
        assert rel(x, xo) < 1e-7


def test_multishift_chronological(setup, oracle):
    # ChronologicalMultishiftSolver (ChronologicalMultishiftSolver.cpp:11-194): the second solve
    # starts every shift from the first solve's solutions (the chronological guesses)
    b = setup["b"]
    shifts = [0.5, 0.1, 0.01]
    eps = (1e-10) ** 2 * float(np.vdot(b, b).real)
    op = gpu_op(setup, L.SquareImprovedDiracWilsonOperator)
    orc = oracle.Operator(setup["geom"], setup["links"], "SquareImproved", setup["kappa"], setup["csw"], True)
    ms = L.MultishiftSolver.getInstance("chronological_mass_estrapolation")
    ms.setPrecision(eps)
    sols = []
    assert ms.solve(op, b, sols, shifts)
    first_iters = ms.stats.iterations
    rc, osols = oracle.chrono_multishift(orc, b, shifts, eps)
    assert rc == 1
    for x, xo, s in zip(sols, osols, shifts):
        assert true_res(orc, b, x, s) < 1.5e-10
        assert rel(x, xo) < 1e-7
    b2 = b + 1e-3 * synth.gaussian_spinor(setup["dims"], 3, 22)
    sols2 = []
    assert ms.solve(op, b2, sols2, shifts)
    rc, osols2 = oracle.chrono_multishift(orc, b2, shifts, eps, previous=osols)
    for x, xo, s in zip(sols2, osols2, shifts):
        assert true_res(orc, b2, x, s) < 1.5e-10
        assert rel(x, xo) < 1e-7
    assert ms.stats.iterations < first_iters


@pytest.mark.parametrize("mode", ["single", "half"])
def test_multishift_cg_mixed(setup, oracle, mode):
    # RHMC multishift on the squared even-odd operator: FP32 / FP16 inner storage, FP64
    # recurrences; every shift's FP64 true residual <= 1e-10 and the solutions equal the
    # oracle's FP64 mass-estrapolation solutions
    b = setup["b"]
    shifts = list(np.logspace(-4, 0, 12))
    eps = (1e-10) ** 2 * float(np.vdot(b, b).real)
    op = gpu_op(setup, L.SquareEvenOddImprovedDiracWilsonOperator)
    ms = L.MultishiftSolver.getInstance(f"multishift_cg_mixed_{mode}")
    ms.setPrecision(eps)
    ms.setMaxSteps(10000)
    sols = []
    assert ms.solve(op, b, sols, shifts)
    assert ms.stats.true_residual <= 1e-10
    assert ms.stats.reliable_updates >= 1
    orc = oracle.Operator(setup["geom"], setup["links"], "SquareEvenOddImproved", setup["kappa"], setup["csw"],
                          True)
    rc, osols, _ = oracle.me_multishift(orc, b, shifts, eps, 10000)
    assert rc == 1
    for x, xo, s in zip(sols, osols, shifts):
        assert true_res(orc, b, x, s) <= 1.05e-10
        assert rel(x, xo) < 1e-7


def test_multishift_cg_mixed_needs_rhmc_operator(setup):
    op = gpu_op(setup, L.SquareImprovedDiracWilsonOperator)
    ms = L.MultishiftSolver.getInstance("multishift_cg_mixed_single")
    with pytest.raises(L.LymError):
        ms.solve(op, setup["b"], [], [0.1, 0.01])
    op = gpu_op(setup, L.SquareEvenOddImprovedDiracWilsonOperator)
    with pytest.raises(L.LymError):
        ms.solve(op, setup["b"], [], [-1.0, 0.01])


@pytest.mark.parametrize("kind,alg", [("SquareImproved", "mass_estrapolation"),
                                      ("SquareImproved", "minimal_residual"),
                                      ("SquareEvenOddImproved", "mass_estrapolation"),
                                      ("SquareEvenOddImproved", "multishift_cg_mixed_half")])
def test_rational_evaluate(setup, oracle, kind, alg):
    # RationalApproximation::evaluate: sum_i alpha_i (A + beta_i)^{-1} b, against the oracle's
    # restatement (FP64 mass-estrapolation multishift)
    b = setup["b"]
    alphas, betas = [0.31, 0.12, 0.047, 0.011], [0.9, 0.17, 0.03, 0.004]
    eps = (1e-11) ** 2 * float(np.vdot(b, b).real)
    cls = L.SquareImprovedDiracWilsonOperator if kind == "SquareImproved" else L.SquareEvenOddImprovedDiracWilsonOperator
    ra = L.RationalApproximation(alphas, betas, L.MultishiftSolver.getInstance(alg))
    ra.setPrecision(eps)
    ra.setMaximumRecursion(10000)
    out = setup["lat"].new_vector()
    ra.evaluate(gpu_op(setup, cls), out, b)
    orc = oracle.Operator(setup["geom"], setup["links"], kind, setup["kappa"], setup["csw"], True)
    rc, ref = oracle.rational_evaluate(orc, alphas, betas, b, eps, 10000)
    assert rc == 1
    assert rel(out, ref) < 1e-8
    assert abs(ra.evaluate(0.25) - oracle.rational_value(alphas, betas, 0.25)) < 1e-14


def test_rhmc_action_energy_and_force_solves(setup, oracle):
    # NFlavorFermionAction: energy = sum_k Re <phi_k, r_k(A) phi_k>; updateForce's solves
    # x_i = (A + beta_i)^{-1} phi, y_i = D x_i, on the even-odd RHMC operator
    b = setup["b"]
    phi2 = synth.gaussian_spinor(setup["dims"], 3, 23)
    approx = [([0.31, 0.12, 0.047], [0.9, 0.17, 0.03]), ([0.5, 0.2], [0.4, 0.05])]
    eps = (1e-11) ** 2 * float(np.vdot(b, b).real)
    sq = gpu_op(setup, L.SquareEvenOddImprovedDiracWilsonOperator)
    D = gpu_op(setup, L.EvenOddImprovedDiracWilsonOperator)
    ras = []
    for al, be in approx:
        ms = L.MultishiftSolver.getInstance("mass_estrapolation")
        ms.setPrecision(eps)
        ms.setMaxSteps(10000)
        ra = L.RationalApproximation(al, be, ms)
        ra.setPrecision(eps)
        ra.setMaximumRecursion(10000)
        ras.append(ra)
    act = L.NFlavorFermionAction(D, sq, ras)
    act.addPseudoFermion(b)
    act.addPseudoFermion(phi2)
    A = oracle.Operator(setup["geom"], setup["links"], "SquareEvenOddImproved", setup["kappa"], setup["csw"], True)
    Do = oracle.Operator(setup["geom"], setup["links"], "EvenOddImproved", setup["kappa"], setup["csw"], True)
    e_ref = oracle.rhmc_energy(A, approx, [b, phi2], eps, 10000)
    assert abs(act.energy() - e_ref) <= 1e-9 * abs(e_ref)
    Xs, Ys = act.solves()
    for (al, be), phi, X, Y in zip(approx, [b, phi2], Xs, Ys):
        rc, xo, yo = oracle.rhmc_force_solves(A, Do, be, phi, eps, 10000)
        assert rc == 1
        for x, y, xr, yr in zip(X, Y, xo, yo):
            assert rel(x, xr) < 1e-8
            assert rel(y, yr) < 1e-8
