"""The drop-in boundary exercised from the reference side.

oracle/adapter_driver.cpp is linked with LeonardYM's own classes (compiled from its
sources into oracle/_ref by oracle/build_ref.sh) and with liblym_b200.so through the C++
adapter include/lym_leonard_adapter.hpp.  Through the reference's base-class pointers it
checks, against the reference's CPU classes on the same seeded links and source:

* DiracOperator::multiply / multiplyAdd of the six Gpu* operators, both gamma5 flags
  (1e-13 relative);
* the reference's own BiConjugateGradient::solve on GpuSquareEvenOddImproved;
* GpuSolver (CG, BiCGStab) against ConjugateGradient / BiConjugateGradient, the
  solutions (1e-8) and getLastSteps() (equal for CG, within 2 for BiCGStab, whose
  reductions sum in another order);
* GpuPreconditionedBiCGStab (the class MesonCorrelator / ChiralCondensate instantiate)
  on a GPU and on a plain CPU ImprovedDiracWilsonOperator, with and without even-odd
  preconditioning, against PreconditionedBiCGStab;
* GpuMultishiftSolver through MultishiftSolver* against mass_estrapolation and
  minimal_residual;
* DiracOperator::getForce()->derivative against ImprovedFermionForce (1e-12).
"""
import os
import subprocess

import numpy as np
import pytest

from leonardym_b200 import synth

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CASES = {"su3": ((4, 4, 4, 8), 0.13, 1.0), "su2adj": ((4, 4, 4, 8), 0.15, 1.5)}


@pytest.mark.parametrize("rep", ["su3", "su2adj"])
def test_reference_side_adapter(rep, tmp_path):
    exe = os.path.join(ROOT, "oracle", "_ref", f"adapter_driver_{rep}")
    if not os.path.exists(exe):
        pytest.skip("the reference-side driver is built with the reference sources (oracle/build_ref.sh)")
    dims, kappa, csw = CASES[rep]
    links = synth.fermion_links(dims, rep, 0.3, 4321)
    src = synth.gaussian_spinor(dims, 3, 99)
    lp, sp = tmp_path / "links.bin", tmp_path / "source.bin"
    np.ascontiguousarray(links).tofile(lp)
    np.ascontiguousarray(src).tofile(sp)
    r = subprocess.run([exe, *map(str, dims), str(kappa), str(csw), str(lp), str(sp)], capture_output=True, text=True,
                       timeout=600, env={**os.environ, "OMP_NUM_THREADS": "4"})
    lines = [l for l in r.stdout.splitlines() if l.startswith(("ok ", "FAIL ", "   ", "PASSED", "FAILED"))]
    print("\n".join(lines))
    assert r.returncode == 0, "\n".join(l for l in lines if l.startswith("FAIL")) + r.stderr[-2000:]
    assert sum(l.startswith("ok ") for l in lines) >= 40
