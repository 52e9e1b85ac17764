"""The solve server: requests of mixed volume, representation, kappa and source count
submitted together are continuously batched; every result equals the same request
solved alone (within what the 1e-10 true residual allows) and meets the 1e-10 true
residual re-measured with the FP64 oracle operator."""
import numpy as np
import pytest

import leonardym_b200 as L
from leonardym_b200 import synth
from leonardym_b200.server import SolveServer
from tests.helpers import rel

pytestmark = pytest.mark.gpu

FIELDS = {  # key: dims, rep, eps, seed
    1: ((4, 4, 4, 8), "su3", 0.3, 11),
    2: ((4, 4, 4, 8), "su2adj", 0.3, 12),
    3: ((6, 6, 4, 8), "su3", 0.25, 13),
}


def requests():
    rng = np.random.default_rng(7)
    out = []
    for k in range(10):
        key = [1, 2, 3][k % 3]
        dims, rep = FIELDS[key][0], FIELDS[key][1]
        kappa = rng.uniform(0.12, 0.135) if rep == "su3" else rng.uniform(0.17, 0.185)
        n = int(rng.integers(1, 5))
        srcs = [synth.gaussian_spinor(dims, 3, 1000 * k + j) for j in range(n)]
        out.append((key, kappa, 1.0 + 0.1 * (k % 4), srcs))
    return out


@pytest.fixture(scope="module")
def links():
    return {key: synth.fermion_links(d, rep, eps, seed) for key, (d, rep, eps, seed) in FIELDS.items()}


@pytest.mark.parametrize("precision,batch,solver", [("single", 4, "cg"), ("half", 8, "cg"),
                                                   ("single", 4, "bicgstab"), ("half", 8, "bicgstab")])
def test_server_mix_equals_alone(links, precision, batch, solver, oracle):
    srv = SolveServer(batch=batch, precision=precision, solver=solver)
    try:
        for key, (dims, rep, _, _) in FIELDS.items():
            srv.add_gauge(key, dims, rep, links[key])
        reqs = requests()
        tickets = [srv.submit(key, kappa, csw, srcs) for key, kappa, csw, srcs in reqs]
        results = [srv.wait(t) for t, _ in tickets]
    finally:
        srv.close()
    geoms = {}
    for (key, kappa, csw, srcs), (t, sols), (ok, st) in zip(reqs, tickets, results):
        assert ok and st.status == 0 and st.nsrc == len(srcs)
        assert st.max_true_residual <= 1e-10
        dims, rep = FIELDS[key][0], FIELDS[key][1]
        geoms.setdefault(dims, oracle.Geometry(dims))
        D = oracle.Operator(geoms[dims], links[key], "Improved", kappa, csw, False)
        lat = L.Lattice(dims, rep)
        try:
            op = L.ImprovedDiracWilsonOperator(lat, kappa, csw, gamma5=False)
            op.setLattice(links[key])
            for b, x in zip(srcs, sols):
                assert np.linalg.norm(b - D.multiply(x)) / np.linalg.norm(b) <= 1e-10
                alone = lat.new_vector()
                assert L.EvenOddConjugateGradient(precision, 1e-10).solve(op, b, alone)
                assert rel(x, alone) < 1e-8
        finally:
            lat.close()


def test_server_rejects_unknown_field(links):
    srv = SolveServer(batch=4)
    try:
        with pytest.raises(L.LymError):
            srv.submit(42, 0.13, 1.0, [np.zeros((512, 4, 3), np.complex128)])
    finally:
        srv.close()


def test_server_budget_too_small_fails_request(links):
    dims, rep = FIELDS[1][0], FIELDS[1][1]
    srv = SolveServer(batch=4, hbm_budget=1)  # nothing fits: the request fails, the server survives
    try:
        srv.add_gauge(1, dims, rep, links[1])
        t, _ = srv.submit(1, 0.13, 1.0, [synth.gaussian_spinor(dims, 3, 5)])
        with pytest.raises(L.LymError):
            srv.wait(t)
    finally:
        srv.close()


def test_server_mix_with_a_16c32_field(links, oracle):
    """A 16^3 x 32 field among the small ones: its requests and the small fields' requests
    are batched in the same server (one lane per field, overlapping on the device); every
    result meets the oracle's 1e-10 true residual and equals the same source solved alone."""
    big_key, big = 4, ((16, 16, 16, 32), "su3", 0.25, 14)
    big_links = synth.fermion_links(big[0], big[1], big[2], big[3])
    rng = np.random.default_rng(8)
    reqs = [(1, 0.125, 1.0, [synth.gaussian_spinor(FIELDS[1][0], 3, 2000 + j) for j in range(3)]),
            (big_key, 0.13, 1.7, [synth.gaussian_spinor(big[0], 3, 2100 + j) for j in range(3)]),
            (2, 0.175, 1.5, [synth.gaussian_spinor(FIELDS[2][0], 3, 2200 + j) for j in range(2)]),
            (big_key, float(rng.uniform(0.12, 0.135)), 1.7, [synth.gaussian_spinor(big[0], 3, 2300)]),
            (3, 0.13, 1.2, [synth.gaussian_spinor(FIELDS[3][0], 3, 2400 + j) for j in range(4)])]
    srv = SolveServer(batch=8, precision="single", solver="bicgstab")
    try:
        for key, (dims, rep, _, _) in FIELDS.items():
            srv.add_gauge(key, dims, rep, links[key])
        srv.add_gauge(big_key, big[0], big[1], big_links)
        tickets = [srv.submit(key, kappa, csw, srcs) for key, kappa, csw, srcs in reqs]
        results = [srv.wait(t, timeout=600) for t, _ in tickets]
    finally:
        srv.close()
    all_links = dict(links)
    all_links[big_key] = big_links
    dims_of = {k: v[0] for k, v in FIELDS.items()}
    dims_of[big_key] = big[0]
    rep_of = {k: v[1] for k, v in FIELDS.items()}
    rep_of[big_key] = big[1]
    for (key, kappa, csw, srcs), (t, sols), (ok, st) in zip(reqs, tickets, results):
        assert ok and st.status == 0 and st.max_true_residual <= 1e-10
        D = oracle.Operator(oracle.Geometry(dims_of[key]), all_links[key], "Improved", kappa, csw, False)
        lat = L.Lattice(dims_of[key], rep_of[key])
        try:
            op = L.ImprovedDiracWilsonOperator(lat, kappa, csw, gamma5=False)
            op.setLattice(all_links[key])
            for b, x in zip(srcs, sols):
                assert np.linalg.norm(b - D.multiply(x)) / np.linalg.norm(b) <= 1e-10
                alone = lat.new_vector()
                assert L.EvenOddBiCGStab("single", 1e-10).solve(op, b, alone)
                assert rel(x, alone) < 1e-8
        finally:
            lat.close()
