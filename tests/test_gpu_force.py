"""The fermion force on the GPU (lym_fermion_force) against the oracle's restatement of
FermionForce::derivative with DiracWilsonFermionForce / ImprovedFermionForce, on the whole
field, and NFlavorFermionAction's force from the multishift solutions."""
import ctypes as C

import numpy as np
import pytest

import leonardym_b200 as L
from leonardym_b200 import synth
from oracle import force as OF
from tests.helpers import CONFIGS, links_for

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=["su3", "su2adj"])
def setup(request):
    name = request.param
    dims, rep, eps, kappa, csw = CONFIGS[name]
    links = links_for(name)
    lat = L.Lattice(dims, rep)
    gid = lat.upload(links)
    yield dict(dims=dims, kappa=kappa, csw=csw, links=links, lat=lat, gid=gid)
    lat.close()


@pytest.mark.parametrize("kind", ["DiracWilson", "Improved"])
def test_force_field(setup, kind):
    dims, lat = setup["dims"], setup["lat"]
    op = (L.ImprovedDiracWilsonOperator(lat, setup["kappa"], setup["csw"]) if kind == "Improved"
          else L.DiracWilsonOperator(lat, setup["kappa"]))
    op.setLattice(setup["gid"])
    X, Y = synth.gaussian_spinor(dims, 3, 51), synth.gaussian_spinor(dims, 3, 52)
    rng = np.random.default_rng(9)
    V = int(np.prod(dims))
    f0 = rng.standard_normal((V, 4, 3, 3)) + 1j * rng.standard_normal((V, 4, 3, 3))
    f = f0.copy()
    op.getForce().derivative(f, X, Y, 0.35)
    ref = OF.fermion_force(dims, setup["links"], X, Y, setup["kappa"], setup["csw"], kind == "Improved", 0.35, f0)
    assert np.max(np.abs(f - ref)) <= 1e-13 * np.max(np.abs(ref - f0))
    # device pointers, accumulating twice
    import torch
    dX, dY = (torch.from_numpy(v).to("cuda:0") for v in (X, Y))
    df = torch.from_numpy(f0).to("cuda:0")
    torch.cuda.synchronize()  # the library's stream does not wait for torch's
    for _ in range(2):
        assert L.lib().lym_fermion_force_device(lat.handle, op.op_id, C.c_void_p(dX.data_ptr()),
                                                C.c_void_p(dY.data_ptr()), 0.35, C.c_void_p(df.data_ptr())) == 0
    ref2 = OF.fermion_force(dims, setup["links"], X, Y, setup["kappa"], setup["csw"], kind == "Improved", 0.35, ref)
    assert np.max(np.abs(df.cpu().numpy() - ref2)) <= 1e-13 * np.max(np.abs(ref2 - f0))


def test_action_force(setup, oracle):
    # NFlavorFermionAction::updateForce's fermion force lattice: solves, then -alpha_i F(x_i, y_i)
    dims, lat = setup["dims"], setup["lat"]
    sq = L.SquareImprovedDiracWilsonOperator(lat, setup["kappa"])
    sq.setCSW(setup["csw"])
    sq.setGamma5(True)
    sq.setLattice(setup["gid"])
    D = L.ImprovedDiracWilsonOperator(lat, setup["kappa"], setup["csw"], gamma5=True)
    D.setLattice(setup["gid"])
    phi = synth.gaussian_spinor(dims, 3, 53)
    eps = (1e-12) ** 2 * float(np.vdot(phi, phi).real)
    ms = L.MultishiftSolver.getInstance("mass_estrapolation")
    ms.setPrecision(eps)
    ms.setMaxSteps(10000)
    alphas, betas = [0.2, 0.05], [0.3, 0.02]
    act = L.NFlavorFermionAction(D, sq, [L.RationalApproximation(alphas, betas, ms)])
    act.addPseudoFermion(phi)
    f = act.fermionForce()
    A = oracle.Operator(oracle.Geometry(dims), setup["links"], "SquareImproved", setup["kappa"], setup["csw"], True)
    Do = oracle.Operator(oracle.Geometry(dims), setup["links"], "Improved", setup["kappa"], setup["csw"], True)
    rc, xs, ys = oracle.rhmc_force_solves(A, Do, betas, phi, eps, 10000)
    ref = np.zeros_like(f)
    for a, x, y in zip(alphas, xs, ys):
        ref = OF.fermion_force(dims, setup["links"], x, y, setup["kappa"], setup["csw"], True, a, ref)
    Lt = dims[3]
    ref.reshape(-1, Lt, 4, 3, 3)[:, Lt - 1, 3] *= -1
    assert np.max(np.abs(f - ref)) <= 1e-9 * np.max(np.abs(ref))


def test_force_many_pairs(setup):
    # one pass over n weighted pairs equals n single-pair passes
    dims, lat = setup["dims"], setup["lat"]
    op = L.ImprovedDiracWilsonOperator(lat, setup["kappa"], setup["csw"])
    op.setLattice(setup["gid"])
    ff = op.getForce()
    Xs = [synth.gaussian_spinor(dims, 3, 60 + k) for k in range(3)]
    Ys = [synth.gaussian_spinor(dims, 3, 70 + k) for k in range(3)]
    w = [0.3, -0.1, 0.05]
    V = int(np.prod(dims))
    a = np.zeros((V, 4, 3, 3), np.complex128)
    b = np.zeros_like(a)
    ff.derivative_many(a, Xs, Ys, w)
    for x, y, wi in zip(Xs, Ys, w):
        ff.derivative(b, x, y, wi)
    assert np.max(np.abs(a - b)) <= 1e-13 * np.max(np.abs(b))
