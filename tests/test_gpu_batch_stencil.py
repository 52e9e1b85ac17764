"""The batched (multi-RHS) stencil against the FP64 oracle, one application at a time:
every right-hand side of a batch gets EvenOddImprovedDiracWilsonOperator::multiply
(EvenOddImprovedDiracWilsonOperator.cpp:26-47) of its own operator (kappa and c_sw
differ per slot), for every traversal column and kernel variant the autotuner chooses
between.  Bar: FP32 storage within 1e-6 relative, FP16 storage within 1e-2."""
import pytest

import leonardym_b200 as L
from leonardym_b200 import synth
from leonardym_b200.dirac import batch_tile, multiply_batch, set_batch_tile
from tests.helpers import CONFIGS, links_for, rel

pytestmark = pytest.mark.gpu

TOL = {"single": 1e-6, "half": 1e-2}
CASES = {  # name: dims, rep
    "su3": ((4, 4, 4, 8), "su3"),
    "su2adj": ((4, 4, 4, 8), "su2adj"),
    "su3-6x6": ((6, 6, 4, 8), "su3"),
}


@pytest.fixture(scope="module", params=sorted(CASES))
def setup(request, oracle):
    dims, rep = CASES[request.param]
    if dims == CONFIGS[rep][0]:
        links = links_for(rep)
    else:
        links = synth.fermion_links(dims, rep, 0.25, 31)
    lat = L.Lattice(dims, rep)
    gid = lat.upload(links)
    geom = oracle.Geometry(dims)
    yield dict(dims=dims, rep=rep, links=links, lat=lat, gid=gid, geom=geom)
    lat.close()


def operators(setup, gamma5):
    base = 0.13 if setup["rep"] == "su3" else 0.18
    params = [(base, 1.0), (base - 0.01, 1.7), (base + 0.004, 0.0)]
    gpu = []
    for kappa, csw in params:
        op = L.EvenOddImprovedDiracWilsonOperator(setup["lat"], kappa, csw, gamma5=gamma5)
        op.setLattice(setup["gid"])
        gpu.append(op)
    return params, gpu


def tiles(dims):
    Ly, Lz = dims[1], dims[2]
    # direct-load variants (minb 1, 3, 4), shared-memory staged ones (19, 20), staged with
    # bulk copies (35, 36) and staged with 18-real SU(3) links (83, 84; 19, 20 for the adjoint)
    return [(0, 0, 1), (Ly, Lz, 3), (2, Lz, 4), (2, 2, 19), (1, 1, 20), (0, 0, 19), (2, 2, 35), (Ly, Lz, 36),
            (2, 2, 83), (Ly, Lz, 84)]


@pytest.mark.parametrize("gamma5", [False, True])
@pytest.mark.parametrize("precision", ["single", "half"])
def test_batched_stencil_every_tile(setup, precision, gamma5, oracle):
    params, gpu = operators(setup, gamma5)
    xs = [synth.gaussian_spinor(setup["dims"], 3, 300 + j) for j in range(5)]
    want = []
    for j, x in enumerate(xs):
        kappa, csw = params[j % 3]
        D = oracle.Operator(setup["geom"], setup["links"], "EvenOddImproved", kappa, csw, gamma5)
        want.append(D.multiply(x))
    try:
        for by, bz, minb in tiles(setup["dims"]):
            set_batch_tile(setup["lat"], by, bz, minb)
            got = multiply_batch([gpu[j % 3] for j in range(5)], xs, precision)
            for j in range(5):
                assert rel(got[j], want[j]) < TOL[precision], ((by, bz, minb), j)
    finally:
        set_batch_tile(setup["lat"], -1, 0)


def test_batched_stencil_autotuned(setup, oracle):
    params, gpu = operators(setup, False)
    xs = [synth.gaussian_spinor(setup["dims"], 3, 400 + j) for j in range(3)]
    got = multiply_batch(gpu, xs, "single")
    by, bz, minb = batch_tile(setup["lat"], "single", 4)
    assert minb in (1, 3, 4, 19, 20, 35, 36, 83, 84)
    assert by == 0 or (setup["dims"][1] % by == 0 and setup["dims"][2] % bz == 0)
    for j, x in enumerate(xs):
        D = oracle.Operator(setup["geom"], setup["links"], "EvenOddImproved", params[j][0], params[j][1], False)
        assert rel(got[j], D.multiply(x)) < TOL["single"]


def test_batched_stencil_rejects_bad_tiles(setup):
    with pytest.raises(L.LymError):
        set_batch_tile(setup["lat"], 5, 1, 1)  # by does not divide Ly
    with pytest.raises(L.LymError):
        set_batch_tile(setup["lat"], 2, 2, 2)  # no such kernel variant
