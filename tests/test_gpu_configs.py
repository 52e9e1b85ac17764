"""The configs' small cases at their own sizes, through the Python mirror of the reference
interfaces, checked with the oracle's FP64 operators.

* SU(3) Wilson-clover 8^4, kappa 0.13, c_sw 1.0, links exp(0.3 i H): CG on D^dagger D
  (SquareImprovedDiracWilsonOperator) to relative residual 1e-10, against the oracle's
  restatement of ConjugateGradient::solve (same iteration count within 2, same solution).
* SU(2) adjoint Wilson-clover 16^3x32, kappa 0.18, c_sw 1.5, even-odd preconditioned:
  mixed-precision CG (FP32 inner, FP64 reliable updates) against the FP64-only GPU CG:
  both reach ||b - D x|| <= 1e-10 ||b|| measured with the oracle's FP64 operator, and agree to
  1e-8."""
import time

import numpy as np
import pytest

import leonardym_b200 as L
from leonardym_b200 import synth
from tests.helpers import rel

pytestmark = pytest.mark.gpu


def test_su3_8x4_cg_on_ddagd(oracle):
    dims, kappa, csw = (8, 8, 8, 8), 0.13, 1.0
    links = synth.fermion_links(dims, "su3", 0.3, 1235)
    b = synth.gaussian_spinor(dims, 3, 1236)
    eps = (1e-10) ** 2 * float(np.vdot(b, b).real)
    lat = L.Lattice(dims, "su3")
    try:
        op = L.SquareImprovedDiracWilsonOperator(lat, kappa)
        op.setCSW(csw)
        op.setGamma5(True)
        op.setLattice(links)
        cg = L.ConjugateGradient()
        cg.setPrecision(eps)
        cg.setMaximumSteps(5000)
        x = lat.new_vector()
        assert cg.solve(op, b, x)
        orc = oracle.Operator(oracle.Geometry(dims), links, "SquareImproved", kappa, csw, True)
        rc, xo, steps = oracle.cg(orc, b, eps, 5000)
        assert rc == 1
        assert abs(cg.getLastSteps() - steps) <= 2
        assert np.linalg.norm(b - orc.multiply(x)) / np.linalg.norm(b) < 1.5e-10
        assert rel(x, xo) < 1e-7
    finally:
        lat.close()


def test_su2adj_16c32_mixed_cg_vs_fp64(oracle):
    dims, kappa, csw = (16, 16, 16, 32), 0.18, 1.5
    links = synth.fermion_links(dims, "su2adj", 0.3, 1236)
    b = synth.gaussian_spinor(dims, 3, 1237)
    lat = L.Lattice(dims, "su2adj")
    try:
        op = L.ImprovedDiracWilsonOperator(lat, kappa, csw, gamma5=False)
        op.setLattice(links)
        D = oracle.Operator(oracle.Geometry(dims), links, "Improved", kappa, csw, False)
        out = {}
        for mode in ("double", "single"):
            s = L.EvenOddConjugateGradient(mode, 1e-10)
            x = lat.new_vector()
            t0 = time.perf_counter()
            assert s.solve(op, b, x)
            out[mode] = (x, s.stats.iterations, s.stats.seconds, time.perf_counter() - t0)
            assert np.linalg.norm(b - D.multiply(x)) / np.linalg.norm(b) <= 1e-10
        x64, x32 = out["double"][0], out["single"][0]
        # both solve to 1e-10; their difference is bounded by the condition number times that
        # (measured 3.5e-11 on this system)
        assert rel(x32, x64) < 1e-8
        print(f"SU(2) adjoint 16^3x32 EO-CG: solutions differ by {rel(x32, x64):.1e}; "
              f"FP64 {out['double'][1]} iterations {out['double'][2] * 1e3:.1f} ms, "
              f"FP32 inner {out['single'][1]} iterations {out['single'][2] * 1e3:.1f} ms")
    finally:
        lat.close()
