"""RHMC consumers of the multishift solvers, on the GPU through the C ABI:
RationalApproximation (dirac_functions/RationalApproximation.{h,cpp}), the fermion force
(hmc_forces/FermionForce, DiracWilsonFermionForce, ImprovedFermionForce) and the solve, force
and energy parts of NFlavorFermionAction (actions/NFlavorFermionAction.cpp:76-117,193-207)."""
from __future__ import annotations

import ctypes as C
import numbers

import numpy as np

from ._lib import LymError, SolveStats, lib
from .solvers import MultishiftSolver


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


class RationalApproximation:
    """r(x) = sum_i alpha_i / (x + beta_i); precision 1e-12 and 3000 steps by default
    (RationalApproximation.cpp:10-14)."""

    def __init__(self, alphas=None, betas=None, multishiftSolver=None):
        self.alphas = [float(a) for a in (alphas if alphas is not None else [])]
        self.betas = [float(b) for b in (betas if betas is not None else [])]
        self.precision = 1e-12
        self.maximumSteps = 3000
        self.multishiftSolver = multishiftSolver or MultishiftSolver.getInstance("mass_estrapolation")
        self.stats = None

    def evaluate(self, *args):
        """evaluate(x) -> complex r(x) (RationalApproximation.cpp:44-52), or
        evaluate(dirac, output, input): output = sum_i alpha_i (A + beta_i)^{-1} input
        (RationalApproximation.cpp:18-42), A the operator `dirac`."""
        if len(args) == 1 and isinstance(args[0], numbers.Number):
            x = complex(args[0])
            return sum(a / (x + b) for a, b in zip(self.alphas, self.betas))
        dirac, output, source = args
        if len(self.alphas) != len(self.betas) or not self.betas:
            raise LymError(-1, "a rational approximation needs as many alphas as betas")
        lat = dirac.lattice
        src = dirac._vec(source)
        if output.shape != src.shape or output.dtype != np.complex128 or not output.flags.c_contiguous:
            raise LymError(-1, "output must be a contiguous complex128 array shaped like the input")
        a = np.ascontiguousarray(self.alphas, np.float64)
        b = np.ascontiguousarray(self.betas, np.float64)
        st = SolveStats()
        rc = lib().lym_rational_evaluate(lat.handle, dirac.op_id, self.multishiftSolver.algorithm, len(b), _p(a),
                                         _p(b), self.precision, self.maximumSteps, _p(src), _p(output), C.byref(st))
        if rc < 0:
            raise LymError(rc, lib().lym_last_error(lat.handle).decode())
        self.stats = st
        return output

    def setAlphas(self, alphas):
        self.alphas = [float(a) for a in alphas]

    def setBetas(self, betas):
        self.betas = [float(b) for b in betas]

    def getAlphas(self):
        return self.alphas

    def getBetas(self):
        return self.betas

    def setPrecision(self, precision):
        self.precision = float(precision)

    def getPrecision(self):
        return self.precision

    def getMultishiftSolver(self):
        return self.multishiftSolver

    def setMaximumRecursion(self, maximumRecursion):
        self.maximumSteps = int(maximumRecursion)

    def getMaximumRecursion(self):
        return self.maximumSteps


class FermionForce:
    """The fermion force of an operator (DiracOperator::getForce): ImprovedFermionForce at the
    operator's kappa and c_sw for the kinds with a clover term, DiracWilsonFermionForce
    otherwise, on the operator's gauge field."""

    def __init__(self, diracOperator):
        self.diracOperator = diracOperator

    def derivative(self, fermionForce, X, Y, weight):
        """FermionForce::derivative (FermionForce.cpp:11-20): fermionForce[x][mu] -=
        weight * F_mu(x); fermionForce complex128[V, 4, 3, 3] (column-major matrices), in place."""
        op = self.diracOperator
        x, y = op._vec(X), op._vec(Y)
        if fermionForce.dtype != np.complex128 or not fermionForce.flags.c_contiguous:
            raise LymError(-1, "the force field must be a contiguous complex128 array")
        rc = lib().lym_fermion_force(op.lattice.handle, op.op_id, _p(x), _p(y), float(weight),
                                     _p(fermionForce))
        if rc < 0:
            raise LymError(rc, lib().lym_last_error(op.lattice.handle).decode())
        return fermionForce

    def derivative_many(self, fermionForce, Xs, Ys, weights):
        """fermionForce -= sum_i weights[i] F(Xs[i], Ys[i]) in one pass (the link products of
        every clover leaf formed once)."""
        op = self.diracOperator
        xs = [op._vec(x) for x in Xs]
        ys = [op._vec(y) for y in Ys]
        n = len(xs)
        if n == 0:
            return fermionForce
        if fermionForce.dtype != np.complex128 or not fermionForce.flags.c_contiguous:
            raise LymError(-1, "the force field must be a contiguous complex128 array")
        w = np.ascontiguousarray(weights, np.float64)
        xp = (C.c_void_p * n)(*[x.ctypes.data for x in xs])
        yp = (C.c_void_p * n)(*[y.ctypes.data for y in ys])
        rc = lib().lym_fermion_force_multi(op.lattice.handle, op.op_id, n, xp, yp, _p(w), _p(fermionForce))
        if rc < 0:
            raise LymError(rc, lib().lym_last_error(op.lattice.handle).decode())
        return fermionForce


class NFlavorFermionAction:
    """The multishift parts of NFlavorFermionAction: one RationalApproximation per
    pseudofermion, `squareDiracOperator` the operator A of the approximations and
    `diracOperator` the D of updateForce's y_i = D x_i."""

    def __init__(self, diracOperator, squareDiracOperator, rationalApproximations):
        self.diracOperator = diracOperator
        self.squareDiracOperator = squareDiracOperator
        self.rationalApproximations = list(rationalApproximations)
        self.pseudofermions = []

    def addPseudoFermion(self, pseudofermion):
        self.pseudofermions.append(pseudofermion)

    def cleanPseudoFermions(self):
        self.pseudofermions = []

    def energy(self):
        """NFlavorFermionAction::energy (NFlavorFermionAction.cpp:193-207):
        sum_k Re <phi_k, r_k(A) phi_k>."""
        e = 0.0
        for approx, phi in zip(self.rationalApproximations, self.pseudofermions):
            out = self.squareDiracOperator.lattice.new_vector()
            approx.evaluate(self.squareDiracOperator, out, phi)
            e += float(np.vdot(phi, out).real)
        return e

    def solves(self):
        """The solves of NFlavorFermionAction::updateForce (NFlavorFermionAction.cpp:76-96):
        for every pseudofermion, x_i = (A + beta_i)^{-1} phi with the approximation's
        multishift solver and y_i = D x_i.  Returns ([X_k], [Y_k]), lists of lists."""
        Xs, Ys = [], []
        sq, dop = self.squareDiracOperator, self.diracOperator
        lat = sq.lattice
        for approx, phi in zip(self.rationalApproximations, self.pseudofermions):
            src = sq._vec(phi)
            n = len(approx.betas)
            X = [lat.new_vector() for _ in range(n)]
            Y = [lat.new_vector() for _ in range(n)]
            xp = (C.c_void_p * n)(*[x.ctypes.data for x in X])
            yp = (C.c_void_p * n)(*[y.ctypes.data for y in Y])
            b = np.ascontiguousarray(approx.betas, np.float64)
            ms = approx.getMultishiftSolver()
            st = SolveStats()
            rc = lib().lym_rhmc_force_solves(lat.handle, sq.op_id, dop.op_id, ms.algorithm, n, _p(b), ms.epsilon,
                                             ms.maxSteps, _p(src), xp, yp, C.byref(st))
            if rc < 0:
                raise LymError(rc, lib().lym_last_error(lat.handle).decode())
            Xs.append(X)
            Ys.append(Y)
        return Xs, Ys

    def fermionForce(self, boundary_conditions="fermion_antiperiodic"):
        """The fermion force lattice of NFlavorFermionAction::updateForce / derivative
        (NFlavorFermionAction.cpp:53-117): for every approximation and shift,
        force -= alpha_i F(x_i, y_i), then with antiperiodic boundary conditions the sign of
        the t links at t = Lt - 1 (the projection onto the gauge algebra, FermionForce::force,
        is not included)."""
        lat = self.diracOperator.lattice
        force = np.zeros((lat.V, 4, 3, 3), np.complex128)
        ff = FermionForce(self.diracOperator)
        Xs, Ys = self.solves()
        for approx, X, Y in zip(self.rationalApproximations, Xs, Ys):
            ff.derivative_many(force, X, Y, approx.alphas)
        if boundary_conditions == "fermion_antiperiodic":
            Lt = lat.dims[3]
            force.reshape(-1, Lt, 4, 3, 3)[:, Lt - 1, 3] *= -1
        elif boundary_conditions != "fermion_periodic":
            raise LymError(-4, f"boundary conditions {boundary_conditions!r}")
        return force
