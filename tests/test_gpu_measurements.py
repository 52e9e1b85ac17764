"""Propagator consumers on the GPU (MesonCorrelator, ChiralCondensate) through the C ABI and
the Python mirror, against the oracle: the device noise bit for bit, the contraction kernel on
arbitrary spinors to rounding, and the full measurements with the oracle's FP64 solves of the
same sources (every GPU solve at a true residual 1e-10)."""
import ctypes as C

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
    op = L.ImprovedDiracWilsonOperator(lat, kappa, csw, gamma5=False)
    op.setLattice(links)
    geom = oracle.Geometry(dims)
    D5 = oracle.Operator(geom, links, "Improved", kappa, csw, True)  # gamma5 D
    A = oracle.Operator(geom, links, "SquareImproved", kappa, csw, True)  # D^+ D

    def solve(b):
        # D x = b through CG on D^+ D x = D^+ b, D^+ b = gamma5 D gamma5 b
        g5b = b.copy()
        g5b[:, 2:, :] *= -1
        rhs = D5.multiply(g5b)
        rc, x, _ = oracle.cg(A, rhs, 1e-26 * float(np.vdot(rhs, rhs).real), 20000)
        assert rc == 1
        return x

    yield dict(dims=dims, kappa=kappa, lat=lat, op=op, solve=solve)
    lat.close()


def test_noise_matches_oracle(setup, oracle):
    import torch
    lat = setup["lat"]
    out = torch.zeros((lat.V, 4, 3), dtype=torch.complex128, device="cuda:0")
    torch.cuda.synchronize()  # the library's stream does not wait for torch's
    for seed, stream in ((7, 0), (7, 5), (123456789, 2)):
        assert L.lib().lym_noise_z2_device(lat.handle, seed, stream, C.c_void_p(out.data_ptr())) == 0
        assert np.array_equal(out.cpu().numpy(), oracle.z2_noise(setup["dims"], seed, stream))


def test_contraction_kernel(setup, oracle):
    # the kernel on arbitrary spinors (host entry point), against the oracle's contraction
    rng = np.random.default_rng(5)
    V = setup["lat"].V
    props = [np.ascontiguousarray(rng.standard_normal((V, 4, 3)) + 1j * rng.standard_normal((V, 4, 3)))
             for _ in range(12)]
    Lt = setup["dims"][3]
    pion, scalar, ps = np.zeros(Lt), np.zeros(Lt), np.zeros(Lt)
    ptrs = (C.c_void_p * 12)(*[p.ctypes.data for p in props])
    assert L.lib().lym_meson_contractions(setup["lat"].handle, ptrs, pion.ctypes.data, scalar.ctypes.data,
                                          ps.ctypes.data) == 0
    ref = oracle.meson_contractions(props, setup["dims"])
    for a, b in zip((pion, scalar, ps), ref):
        assert np.max(np.abs(a - b)) <= 1e-13 * np.max(np.abs(b))


def test_meson_correlator(setup, oracle):
    mc = L.MesonCorrelator(setup["op"], tolerance=1e-10)
    res = mc.execute()
    assert res["converged"]
    props = [setup["solve"](b) for b in oracle.point_sources(setup["dims"])]
    ref = oracle.meson_output(*oracle.meson_contractions(props, setup["dims"]), setup["kappa"])
    for key in ("pion_exact", "scalar_exact", "ps_exact"):
        assert rel(res[key], ref[key]) < 1e-8, key
    assert rel(res["pcac_mass"], ref["pcac_mass"]) < 1e-6


def test_chiral_condensate(setup, oracle):
    n, seed = 3, 99
    cc = L.ChiralCondensate(setup["op"], number_stochastic_estimators=n, seed=seed, connected=True,
                            tolerance=1e-10)
    res = cc.execute()
    assert res["converged"]
    for k in range(n):
        eta = oracle.z2_noise(setup["dims"], seed, k)
        x = setup["solve"](eta)
        y = setup["solve"](x)
        ref = oracle.condensate_estimator(eta, x, y)
        got = res["estimators"][k]
        assert np.max(np.abs(got - ref)) <= 1e-8 * np.max(np.abs(ref))
    est = res["estimators"]
    assert abs(res["condensate"]["re"] - est[:, 0].mean()) < 1e-14 * abs(est[:, 0]).max()
