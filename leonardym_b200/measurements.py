"""Propagator consumers on the GPU: MesonCorrelator (correlators/MesonCorrelator.cpp) and
ChiralCondensate (fermion_measurements/ChiralCondensate.cpp).  Sources, block solves and
contractions stay in device memory (lym_meson_correlator, lym_chiral_condensate); the
statistics and normalisations of the reference's output are applied here.

Not included: stout smearing of the links, the source time shift and the stochastic
disconnected part of MesonCorrelator (options that default to off), and overlap operators.
The reference draws its noise from a time-seeded generator; here it is a seeded
counter-based one (lym_noise_z2_device), so runs are reproducible."""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from ._lib import LymError, SolveStats, lib
from .solvers import (SOLVER_EO_BICGSTAB_MIXED_HALF, SOLVER_EO_BICGSTAB_MIXED_SINGLE, SOLVER_EO_CG_MIXED_HALF,
                      SOLVER_EO_CG_MIXED_SINGLE)

_SOLVERS = {("bicgstab", "single"): SOLVER_EO_BICGSTAB_MIXED_SINGLE, ("bicgstab", "half"): SOLVER_EO_BICGSTAB_MIXED_HALF,
            ("cg", "single"): SOLVER_EO_CG_MIXED_SINGLE, ("cg", "half"): SOLVER_EO_CG_MIXED_HALF}


def _mean(v):
    """StochasticEstimator::mean (StochasticEstimator.h:48-55)."""
    return sum(v) / len(v)


def _standard_deviation(v):
    """StochasticEstimator::standardDeviation (StochasticEstimator.h:57-65)."""
    m = _mean(v)
    return math.sqrt(sum((x - m) ** 2 for x in v) / (len(v) - 1)) if len(v) > 1 else float("nan")


class _Measurement:
    def __init__(self, diracOperator, tolerance, precision_mode, solver, batch, max_steps):
        if diracOperator.KIND not in (0, 1):
            raise LymError(-4, "propagators are solved for a DiracWilson or Improved operator")
        self.diracOperator = diracOperator
        self.tolerance = float(tolerance)
        self.solver = _SOLVERS[(solver, precision_mode)]
        self.batch = int(batch)
        self.maxSteps = int(max_steps)
        self.stats = None

    def _check(self, rc):
        if rc < 0:
            h = self.diracOperator.lattice.handle
            raise LymError(rc, lib().lym_last_error(h).decode())


class MesonCorrelator(_Measurement):
    """MesonCorrelator::execute: the 12 point-source propagators (gamma5 off, as the
    reference sets it), their connected pion, scalar and PS correlators and the PCAC mass.
    ``tolerance`` is the relative true residual of every solve (the reference's
    ``inverter_precision`` is an absolute squared residual, 1e-11 by default)."""

    def __init__(self, diracOperator, tolerance=1e-10, precision_mode="single", solver="bicgstab", batch=16,
                 max_steps=10000):
        super().__init__(diracOperator, tolerance, precision_mode, solver, batch, max_steps)

    def execute(self):
        op = self.diracOperator
        lat = op.lattice
        Lt = lat.dims[3]
        gamma5 = op.getGamma5()
        op.setGamma5(False)
        try:
            pion, scalar, ps = (np.zeros(Lt) for _ in range(3))
            st = (SolveStats * 12)()
            rc = lib().lym_meson_correlator(lat.handle, op.op_id, self.solver, -self.tolerance, self.maxSteps,
                                            self.batch, pion.ctypes.data, scalar.ctypes.data, ps.ctypes.data, st)
            self._check(rc)
        finally:
            op.setGamma5(gamma5)
        self.stats = list(st)
        # the reference's output (MesonCorrelator.cpp:160-193)
        factor = 4.0 * op.getKappa() ** 2
        pcac = [(ps[(t - 1) % Lt] - ps[(t + 1) % Lt]) / (4.0 * pion[t]) for t in range(Lt)]
        return {"pion_exact": list(factor * pion), "scalar_exact": list(factor * scalar),
                "ps_exact": list(factor * ps), "pcac_mass": pcac, "raw": (pion, scalar, ps),
                "inversion_steps": int(sum(s.iterations for s in st)), "converged": rc == 0}


class ChiralCondensate(_Measurement):
    """ChiralCondensate::execute: per stochastic estimator the condensate <eta, D^-1 eta>/V,
    the pseudo condensate <eta, gamma5 D^-1 eta>/V, the pion norm |D^-1 eta|^2/V and, with
    ``connected``, <eta, D^-2 eta>/V; the mean and standard deviation of each as the
    reference prints them (ChiralCondensate.cpp:120-160)."""

    def __init__(self, diracOperator, number_stochastic_estimators=20, seed=20260, connected=False,
                 tolerance=1e-10, precision_mode="single", solver="bicgstab", batch=16, max_steps=10000):
        super().__init__(diracOperator, tolerance, precision_mode, solver, batch, max_steps)
        self.n = int(number_stochastic_estimators)
        self.seed = int(seed)
        self.connected = bool(connected)

    def execute(self):
        op = self.diracOperator
        lat = op.lattice
        gamma5 = op.getGamma5()
        op.setGamma5(False)
        out = np.zeros((self.n, 8))
        try:
            st = (SolveStats * (2 * self.n))()
            rc = lib().lym_chiral_condensate(lat.handle, op.op_id, self.solver, -self.tolerance, self.maxSteps,
                                             self.batch, self.n, C.c_ulonglong(self.seed), int(self.connected),
                                             out.ctypes.data, st)
            self._check(rc)
        finally:
            op.setGamma5(gamma5)
        self.stats = list(st)[: (2 if self.connected else 1) * self.n]
        names = ["condensate", "pseudocondensate", "pion_norm", "condensate_connected"]
        res = {"estimators": out, "converged": rc == 0}
        for j, name in enumerate(names):
            if name == "condensate_connected" and not self.connected:
                continue
            re, im = list(out[:, 2 * j]), list(out[:, 2 * j + 1])
            res[name] = {"re": _mean(re), "im": _mean(im), "re_error": _standard_deviation(re),
                         "im_error": _standard_deviation(im)}
        return res
