"""Host-side mirror of LeonardYM's Solver and MultishiftSolver interfaces.

* ``Solver.solve(dirac, source, solution, initial_guess=None) -> bool``
  (inverters/Solver.h:13), with ``setPrecision`` / ``setMaximumSteps`` /
  ``getLastSteps`` / ``getLastError`` (Solver.h:35-57).  ``precision`` is the
  reference's absolute threshold on the squared residual norm.
* ``MultishiftSolver.getInstance(name)`` (inverters/MultishiftSolver.cpp:13-27)
  and ``solve(dirac, source, solutions, shifts) -> bool`` (MultishiftSolver.h:28).

Every solve runs on the GPU through lym_solve / lym_multishift.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import LymError, SolveStats, lib

SOLVER_CG, SOLVER_BICGSTAB, SOLVER_EO_BICGSTAB = 0, 1, 2
SOLVER_EO_CG, SOLVER_EO_CG_MIXED_SINGLE, SOLVER_EO_CG_MIXED_HALF = 3, 4, 5
SOLVER_EO_BICGSTAB_MIXED_SINGLE, SOLVER_EO_BICGSTAB_MIXED_HALF = 6, 7
# multishift_cg_mixed_*: the RHMC multishift on SquareEvenOddImprovedDiracWilsonOperator
# (gamma5) with FP32 / FP16 inner storage, FP64 recurrences and per-shift FP64 true residuals
MULTISHIFT = {"mass_estrapolation": 0, "minimal_residual": 1, "multishift_cg": 2,
              "chronological_mass_estrapolation": 3, "multishift_cg_mixed_single": 4,
              "multishift_cg_mixed_half": 5}


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


class Solver:
    ALGORITHM = None

    def __init__(self, name=""):
        self.name = name
        self.precision = 1e-10      # Solver.h:11
        self.maxSteps = 1000
        self.lastError = 0.0
        self.lastSteps = 0
        self.stats = None

    def setPrecision(self, epsilon):
        self.precision = float(epsilon)

    def getPrecision(self):
        return self.precision

    def setMaximumSteps(self, steps):
        self.maxSteps = int(steps)

    def getMaximumSteps(self):
        return self.maxSteps

    def getLastError(self):
        return self.lastError

    def getLastSteps(self):
        return self.lastSteps

    def _run(self, dirac, source, solution, guess, algorithm, precision):
        lat = dirac.lattice
        src = dirac._vec(source)
        if solution.shape != src.shape or solution.dtype != np.complex128 or not solution.flags.c_contiguous:
            raise LymError(-1, "solution must be a contiguous complex128 array shaped like the source")
        g = _p(dirac._vec(guess)) if guess is not None else None
        st = SolveStats()
        rc = lib().lym_solve(lat.handle, dirac.op_id, algorithm, float(precision), int(self.maxSteps), _p(src),
                             _p(solution), g, C.byref(st))
        if rc < 0:
            msg = lib().lym_last_error(lat.handle)
            if rc == -5:  # breakdown: the reference returns false (BiConjugateGradient.cpp:381-384)
                self.stats = st
                self.lastSteps = st.steps
                return False
            raise LymError(rc, msg.decode() if msg else "")
        self.stats = st
        self.lastSteps = st.steps
        self.lastError = st.last_error
        return rc == 0

    def solve(self, dirac, source, solution, initial_guess=None):
        return self._run(dirac, source, solution, initial_guess, self.ALGORITHM, self.precision)


class ConjugateGradient(Solver):
    """inverters/ConjugateGradient.cpp:10-74 (epsilon 1e-11, 3000 steps by default, :6)."""
    ALGORITHM = SOLVER_CG

    def __init__(self):
        super().__init__("ConjugateGradient")
        self.precision = 1e-11
        self.maxSteps = 3000


class BiConjugateGradient(Solver):
    """inverters/BiConjugateGradient.cpp:321-507.  The reference's other overloads are the
    keyword arguments: shift solves (A + shift) x = b (:510-690), l runs BiCGStab(l)
    (:130-317), preconditioner runs BiCGStab with that operator as preconditioner (:11-128)."""
    ALGORITHM = SOLVER_BICGSTAB

    def __init__(self):
        super().__init__("BiConjugateGradient")

    def solve(self, dirac, source, solution, initial_guess=None, shift=None, l=None, preconditioner=None):
        if shift is None and l is None and preconditioner is None:
            return super().solve(dirac, source, solution, initial_guess)
        lat = dirac.lattice
        src = dirac._vec(source)
        g = _p(dirac._vec(initial_guess)) if initial_guess is not None else None
        st = SolveStats()
        if l is not None:
            rc = lib().lym_solve_bicgstab_l(lat.handle, dirac.op_id, int(l), float(self.precision),
                                            int(self.maxSteps), _p(src), _p(solution), g, C.byref(st))
        elif preconditioner is not None:
            rc = lib().lym_solve_preconditioned(lat.handle, dirac.op_id, preconditioner.op_id, float(self.precision),
                                                int(self.maxSteps), _p(src), _p(solution), g, C.byref(st))
        else:
            s = complex(shift)
            rc = lib().lym_solve_shifted(lat.handle, dirac.op_id, s.real, s.imag, float(self.precision),
                                         int(self.maxSteps), _p(src), _p(solution), g, C.byref(st))
        if rc < 0 and rc != -5:
            raise LymError(rc, lib().lym_last_error(lat.handle).decode())
        self.stats = st
        self.lastSteps = st.steps
        self.lastError = st.last_error
        return rc == 0


class PreconditionedBiCGStab(Solver):
    """inverters/PreconditionedBiCGStab.cpp:33-100: even-odd Schur solve of D x = b
    when the operator is an ImprovedDiracWilsonOperator on even extents."""
    ALGORITHM = SOLVER_EO_BICGSTAB

    def __init__(self):
        super().__init__("PreconditionedBiCGStab")


class EvenOddConjugateGradient(Solver):
    """Even-odd Schur CG on (gamma5 S)^2 solving D x = b (no reference counterpart).
    ``precision_mode`` is "double", "single" (FP32 stencil, FP64 reliable updates) or
    "half" (FP16 spinors with per-site norms).  ``tolerance`` is relative:
    ||b - D x|| <= tolerance ||b||, re-measured with the FP64 operator."""

    MODES = {"double": SOLVER_EO_CG, "single": SOLVER_EO_CG_MIXED_SINGLE, "half": SOLVER_EO_CG_MIXED_HALF}

    def __init__(self, precision_mode="double", tolerance=1e-10):
        super().__init__("EvenOddConjugateGradient")
        self.mode = precision_mode
        self.tolerance = float(tolerance)
        self.maxSteps = 20000

    def solve(self, dirac, source, solution, initial_guess=None):
        return self._run(dirac, source, solution, initial_guess, self.MODES[self.mode], -self.tolerance)

    def solve_block(self, dirac, sources, solutions=None, batch=16):
        """Solve D x_j = b_j for many sources through the batched stencil (lym_solve_block).
        Returns (all_converged, solutions); per-source statistics land in self.block_stats."""
        if self.mode == "double":
            raise LymError(-4, "block solves run the mixed-precision inner iterations ('single' or 'half')")
        lat = dirac.lattice
        srcs = [dirac._vec(s) for s in sources]
        if solutions is None:
            solutions = [lat.new_vector() for _ in srcs]
        n = len(srcs)
        sp = (C.c_void_p * n)(*[s.ctypes.data for s in srcs])
        xp = (C.c_void_p * n)(*[x.ctypes.data for x in solutions])
        stats = (SolveStats * n)()
        rc = lib().lym_solve_block(lat.handle, dirac.op_id, self.MODES[self.mode], -self.tolerance,
                                   int(self.maxSteps), n, sp, xp, int(batch), stats)
        if rc < 0:
            raise LymError(rc, lib().lym_last_error(lat.handle).decode())
        self.block_stats = [stats[j] for j in range(n)]
        return rc == 0, solutions


class EvenOddBiCGStab(EvenOddConjugateGradient):
    """Mixed-precision BiCGStab (inverters/BiConjugateGradient.cpp:321-507) on the even-odd
    Schur operator S itself, solving D x = b; "single" (FP32) or "half" (FP16 + norms)
    inner iterations with FP64 reliable updates that restart from the true residual.
    The same interface as EvenOddConjugateGradient, one or many sources; no guess."""

    MODES = {"single": SOLVER_EO_BICGSTAB_MIXED_SINGLE, "half": SOLVER_EO_BICGSTAB_MIXED_HALF}

    def __init__(self, precision_mode="single", tolerance=1e-10):
        super().__init__(precision_mode, tolerance)
        self.name = "EvenOddBiCGStab"


class MultishiftSolver:
    """inverters/MultishiftSolver.h:11-44; epsilon 1e-8, 3000 steps by default
    (MEMultishiftSolver.h:10, MMMRMultishiftSolver.h:8)."""

    def __init__(self, algorithm, epsilon=1e-8, max_steps=3000):
        self.algorithm = algorithm
        self.epsilon = float(epsilon)
        self.maxSteps = int(max_steps)
        self.stats = None

    @staticmethod
    def getInstance(name):
        if name not in MULTISHIFT:
            raise LymError(-1, f"Name {name} of multishift solver is not recognized!")
        return MultishiftSolver(MULTISHIFT[name])

    def setPrecision(self, epsilon):
        self.epsilon = float(epsilon)

    def getPrecision(self):
        return self.epsilon

    def setMaxSteps(self, steps):
        self.maxSteps = int(steps)

    def getMaxSteps(self):
        return self.maxSteps

    def solve(self, dirac, source, solutions, shifts):
        lat = dirac.lattice
        src = dirac._vec(source)
        while len(solutions) < len(shifts):
            solutions.append(lat.new_vector())
        for s in solutions:
            if s.shape != src.shape or s.dtype != np.complex128 or not s.flags.c_contiguous:
                raise LymError(-1, "solutions must be contiguous complex128 arrays shaped like the source")
        if self.algorithm == MULTISHIFT["chronological_mass_estrapolation"]:
            # the chronological guesses are this solver's previous solutions (zeros at first)
            prev = getattr(self, "_chrono", None)
            for k in range(1, len(shifts)):
                solutions[k][...] = prev[k] if prev is not None and k < len(prev) else 0.0
        ptrs = (C.c_void_p * len(shifts))(*[s.ctypes.data for s in solutions[: len(shifts)]])
        sh = np.ascontiguousarray(shifts, dtype=np.float64)
        st = SolveStats()
        rc = lib().lym_multishift(lat.handle, dirac.op_id, self.algorithm, len(shifts), _p(sh), self.epsilon,
                                  self.maxSteps, _p(src), ptrs, C.byref(st))
        if rc < 0:
            raise LymError(rc, lib().lym_last_error(lat.handle).decode())
        if self.algorithm == MULTISHIFT["chronological_mass_estrapolation"]:
            self._chrono = [s.copy() for s in solutions[: len(shifts)]]
        self.stats = st
        return rc == 0
