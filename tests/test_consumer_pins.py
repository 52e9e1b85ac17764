"""The oracle's propagator consumers pinned to the reference's own MesonCorrelator::execute
(correlators/MesonCorrelator.cpp:22-193) and ChiralCondensate::execute
(fermion_measurements/ChiralCondensate.cpp:84-160), compiled from its sources into
oracle/_ref and run on the same links (the consumer harness captures their printed results
with 17 digits).  The oracle contracts propagators from its own FP64 solves, so the two agree
to what the solver tolerances allow.  The GPU measurements are tested against the oracle in
tests/test_gpu_measurements.py.  The condensate's noise comes from the reference's generator,
seeded, on one thread; the harness returns the vectors it drew."""
import numpy as np
import pytest

from oracle import ref as R
from tests.helpers import CONFIGS, links_for

pytestmark = pytest.mark.skipif(not R.available("su3"), reason="compiled reference not built")


def oracle_solver(oracle, dims, links, kappa, csw):
    geom = oracle.Geometry(dims)
    D5 = oracle.Operator(geom, links, "Improved", kappa, csw, True)
    A = oracle.Operator(geom, links, "SquareImproved", kappa, csw, True)

    def solve(b):  # D x = b through CG on D^+ D x = D^+ b
        g5b = b.copy()
        g5b[:, 2:, :] *= -1
        rhs = D5.multiply(g5b)
        rc, x, _ = oracle.cg(A, rhs, 1e-28 * float(np.vdot(rhs, rhs).real), 20000)
        assert rc == 1
        return x
    return solve


@pytest.mark.parametrize("name", ["su3", "su2adj"])
def test_meson_correlator_matches_reference(name, oracle):
    dims, rep, eps, kappa, csw = CONFIGS[name]
    links = links_for(name)
    want = R.Reference(dims, links, rep).meson_correlator(kappa, csw, 1e-28, 20000)
    solve = oracle_solver(oracle, dims, links, kappa, csw)
    props = [solve(b) for b in oracle.point_sources(dims)]
    got = oracle.meson_output(*oracle.meson_contractions(props, dims), kappa)
    for key in ("pion_exact", "scalar_exact", "ps_exact", "pcac_mass"):
        a, b = np.asarray(got[key]), np.asarray(want[key])
        assert np.max(np.abs(a - b)) <= 1e-9 * np.max(np.abs(b)), (key, a, b)


@pytest.mark.parametrize("name", ["su3", "su2adj"])
def test_chiral_condensate_matches_reference(name, oracle):
    dims, rep, eps, kappa, csw = CONFIGS[name]
    links = links_for(name)
    n = 4
    want, noise = R.Reference(dims, links, rep).chiral_condensate(kappa, csw, 1e-28, 20000, n, True, 12345)
    assert set(np.unique(noise.real)) == {-1.0, 1.0} and not np.any(noise.imag)
    solve = oracle_solver(oracle, dims, links, kappa, csw)
    est = []
    for eta in noise:
        x = solve(eta)
        est.append(oracle.condensate_estimator(eta, x, solve(x)))
    est = np.array(est)  # [n][8]: condensate, pseudo, pion norm, connected (re, im each)
    order = [0, 1, 2, 3, 6, 7, 4, 5]  # the reference prints the connected part before the pion norm
    mean, std = est.mean(axis=0)[order], est.std(axis=0, ddof=1)[order]
    scale = np.max(np.abs(want[:, 0]))
    assert np.max(np.abs(mean - want[:, 0])) <= 1e-9 * scale, (mean, want[:, 0])
    assert np.max(np.abs(std - want[:, 1])) <= 1e-8 * scale, (std, want[:, 1])
