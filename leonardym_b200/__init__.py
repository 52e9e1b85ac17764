"""B200-native Wilson / Wilson-clover operator and Krylov solvers for LeonardYM.

The compute path is liblym_b200.so (hand-written sm_100a CUDA behind the C ABI
of include/lym_b200.h).  This package is the host-side mirror of the
reference's DiracOperator / Solver / MultishiftSolver interfaces over that ABI.
"""
from ._lib import LymError, SolveStats, build, declared_symbols, lib
from .dirac import (DiracOperator, DiracWilsonOperator, EvenOddImprovedDiracWilsonOperator,
                    ImprovedDiracWilsonOperator, Lattice, SquareDiracWilsonOperator,
                    SquareEvenOddImprovedDiracWilsonOperator, SquareImprovedDiracWilsonOperator)
from .measurements import ChiralCondensate, MesonCorrelator
from .rhmc import FermionForce, NFlavorFermionAction, RationalApproximation
from .solvers import (BiConjugateGradient, ConjugateGradient, EvenOddBiCGStab, EvenOddConjugateGradient,
                      MultishiftSolver, PreconditionedBiCGStab, Solver)

__all__ = [
    "LymError", "SolveStats", "build", "declared_symbols", "lib", "Lattice", "DiracOperator",
    "DiracWilsonOperator", "ImprovedDiracWilsonOperator", "EvenOddImprovedDiracWilsonOperator",
    "SquareDiracWilsonOperator", "SquareImprovedDiracWilsonOperator", "SquareEvenOddImprovedDiracWilsonOperator",
    "Solver", "ConjugateGradient", "BiConjugateGradient", "PreconditionedBiCGStab", "EvenOddConjugateGradient",
    "EvenOddBiCGStab",
    "MultishiftSolver", "RationalApproximation", "NFlavorFermionAction", "MesonCorrelator", "ChiralCondensate", "FermionForce",
]
