"""Failures made on the host, never on the GPU: a source with NaN or Inf entries, a step
limit of one, an unreachable tolerance, a BiCGStab breakdown (rho = 0), a device
allocation that fails inside a server lane (an injected error code in place of a failing
cudaMalloc), and a bulk-copy wait of the batched stencil reported as given up (the host's
reading of the kernel's status word faked).  Each must end its own solve or request with a status while everything else
completes within tolerance; the reference returns false on the same inputs
(ConjugateGradient.cpp:70-73, BiConjugateGradient.cpp:381-384, 503-506), pinned here
through its compiled code where it runs."""
import ctypes as C
import time

import numpy as np
import pytest

import leonardym_b200 as L
from leonardym_b200 import synth
from leonardym_b200.server import SolveServer
from leonardym_b200.solvers import (SOLVER_BICGSTAB, SOLVER_CG, SOLVER_EO_BICGSTAB, SOLVER_EO_BICGSTAB_MIXED_SINGLE,
                                    SOLVER_EO_CG, SOLVER_EO_CG_MIXED_SINGLE)
from oracle import ref as R
from tests.helpers import CONFIGS, links_for

pytestmark = pytest.mark.gpu

OK, NOT_CONVERGED, ERR_MEMORY, ERR_BREAKDOWN, ERR_TIMEOUT = 0, 1, -3, -5, -7


@pytest.fixture(scope="module")
def su3(oracle):
    dims, rep, eps, kappa, csw = CONFIGS["su3"]
    links = links_for("su3")
    lat = L.Lattice(dims, rep)
    gid = lat.upload(links)
    ops = {}
    for name, cls, g5 in (("square", L.SquareImprovedDiracWilsonOperator, True),
                          ("improved", L.ImprovedDiracWilsonOperator, False)):
        op = cls(lat, kappa, csw, gamma5=g5)
        op.setLattice(gid)
        ops[name] = op
    yield dict(dims=dims, links=links, lat=lat, gid=gid, ops=ops, kappa=kappa, csw=csw,
               D=oracle.Operator(oracle.Geometry(dims), links, "Improved", kappa, csw, False))
    lat.close()


def solve(setup, op, solver, b, precision, max_steps):
    lib = L.lib()
    x = np.full_like(b, 7.0)
    st = L.SolveStats()
    t0 = time.perf_counter()
    rc = lib.lym_solve(setup["lat"].handle, op.op_id, solver, float(precision), int(max_steps),
                       C.c_void_p(b.ctypes.data), C.c_void_p(x.ctypes.data), None, C.byref(st))
    return rc, x, st, time.perf_counter() - t0


CASES = [("square", SOLVER_CG), ("improved", SOLVER_BICGSTAB), ("improved", SOLVER_EO_BICGSTAB),
         ("improved", SOLVER_EO_CG), ("improved", SOLVER_EO_CG_MIXED_SINGLE),
         ("improved", SOLVER_EO_BICGSTAB_MIXED_SINGLE)]


@pytest.mark.parametrize("bad", [np.nan, np.inf])
@pytest.mark.parametrize("opname,solver", CASES)
def test_nonfinite_source_is_not_converged_at_once(su3, opname, solver, bad):
    b = synth.gaussian_spinor(su3["dims"], 3, 5)
    b[17, 2, 1] = bad
    rc, x, st, seconds = solve(su3, su3["ops"][opname], solver, b, -1e-10 if solver >= 3 else 1e-20, 5000)
    assert rc == NOT_CONVERGED, (rc, L.lib().lym_last_error(su3["lat"].handle))
    assert st.converged == 0
    assert b"non-finite" in L.lib().lym_last_error(su3["lat"].handle)
    assert seconds < 2.0  # not 5000 iterations on non-finite residuals
    # the context goes on: the same operator solves a finite source
    good = synth.gaussian_spinor(su3["dims"], 3, 6)
    rc, x, st, _ = solve(su3, su3["ops"][opname], solver, good, -1e-10 if solver >= 3 else 1e-20, 5000)
    assert rc == OK


def test_reference_returns_false_on_a_nonfinite_source(su3):
    if not R.available("su3"):
        pytest.skip("compiled reference not built")
    b = synth.gaussian_spinor(su3["dims"], 3, 5)
    b[17, 2, 1] = np.nan
    ref = R.Reference(su3["dims"], su3["links"], "su3")
    for kind, solver in (("SquareImproved", "cg"), ("Improved", "bicgstab")):
        rc, x, steps = ref.solve(kind, solver, b, 1e-20, 20, su3["kappa"], su3["csw"], kind.startswith("Square"))
        assert rc == 0  # false: not converged


@pytest.mark.parametrize("opname,solver", CASES)
def test_one_step_is_not_converged(su3, opname, solver):
    b = synth.gaussian_spinor(su3["dims"], 3, 8)
    rc, x, st, _ = solve(su3, su3["ops"][opname], solver, b, -1e-10 if solver >= 3 else 1e-20, 1)
    assert rc == NOT_CONVERGED, rc
    assert st.converged == 0 and np.all(np.isfinite(x))


def test_one_step_matches_the_reference(su3):
    if not R.available("su3"):
        pytest.skip("compiled reference not built")
    b = synth.gaussian_spinor(su3["dims"], 3, 8)
    ref = R.Reference(su3["dims"], su3["links"], "su3")
    for opname, kind, solver, name in (("square", "SquareImproved", SOLVER_CG, "cg"),
                                       ("improved", "Improved", SOLVER_BICGSTAB, "bicgstab")):
        rc, x, st, _ = solve(su3, su3["ops"][opname], solver, b, 1e-20, 1)
        rrc, rx, rsteps = ref.solve(kind, name, b, 1e-20, 1, su3["kappa"], su3["csw"], opname == "square")
        assert rc == NOT_CONVERGED and rrc == 0
        assert np.linalg.norm(x - rx) <= 1e-12 * np.linalg.norm(rx)  # the same one step


@pytest.mark.parametrize("opname,solver", CASES)
def test_unreachable_tolerance_runs_to_the_limit(su3, opname, solver):
    b = synth.gaussian_spinor(su3["dims"], 3, 9)
    # an absolute squared residual below what FP64 reaches, or a relative one of 1e-30
    rc, x, st, _ = solve(su3, su3["ops"][opname], solver, b, -1e-30 if solver >= 3 else 1e-300, 400)
    assert rc in (NOT_CONVERGED, ERR_BREAKDOWN), rc
    assert st.converged == 0
    if rc == NOT_CONVERGED:
        assert np.all(np.isfinite(x))
        if opname == "improved":  # the best solution it found still solves D x = b closely
            assert np.linalg.norm(b - su3["D"].multiply(x)) <= 1e-8 * np.linalg.norm(b)


def test_bicgstab_rho_zero_breakdown_as_the_reference(su3, oracle):
    """kappa = 0: D = 1, so with x0 = b the residual r = b - D b is zero and rho = <rhat, r> = 0:
    the reference reports the breakdown and returns false before its convergence test
    (BiConjugateGradient.cpp:381-384); the library returns LYM_ERR_BREAKDOWN, and the
    solution the reference leaves (x = b) is the library's too."""
    lat = su3["lat"]
    op = L.ImprovedDiracWilsonOperator(lat, 0.0, 1.0, gamma5=False)
    op.setLattice(su3["gid"])
    b = synth.gaussian_spinor(su3["dims"], 3, 11)
    rc, x, st, _ = solve(su3, op, SOLVER_BICGSTAB, b, 1e-20, 100)
    assert rc == ERR_BREAKDOWN, rc
    assert st.converged == 0
    if R.available("su3"):
        rrc, rx, rsteps = R.Reference(su3["dims"], su3["links"], "su3").solve("Improved", "bicgstab", b, 1e-20, 100,
                                                                            0.0, 1.0, False)
        assert rrc == 0
        assert np.linalg.norm(x - rx) <= 1e-14 * np.linalg.norm(rx)


@pytest.mark.parametrize("algo", ["cg", "bicgstab"])
def test_block_solve_nonfinite_source_fails_alone(su3, algo):
    s = (L.EvenOddConjugateGradient if algo == "cg" else L.EvenOddBiCGStab)("single", 1e-10)
    srcs = [synth.gaussian_spinor(su3["dims"], 3, 20 + k) for k in range(5)]
    srcs[2][3, 1, 0] = np.nan
    t0 = time.perf_counter()
    ok, sols = s.solve_block(su3["ops"]["improved"], srcs, batch=4)
    assert time.perf_counter() - t0 < 10.0
    assert not ok
    assert s.block_stats[2].converged == 0
    for k in (0, 1, 3, 4):
        r = np.linalg.norm(srcs[k] - su3["D"].multiply(sols[k])) / np.linalg.norm(srcs[k])
        assert s.block_stats[k].converged == 1 and r <= 1e-10, (k, r)


def _residual(D, b, x):
    return np.linalg.norm(b - D.multiply(x)) / np.linalg.norm(b)


def test_server_nonfinite_source_fails_its_request(oracle):
    dims = (8, 8, 8, 8)
    links = synth.fermion_links(dims, "su3", 0.3, 61)
    srv = SolveServer(batch=8, precision="single", solver="bicgstab")
    try:
        srv.add_gauge(0, dims, "su3", links)
        good = [synth.gaussian_spinor(dims, 3, 70 + k) for k in range(3)]
        bad = [synth.gaussian_spinor(dims, 3, 80)]
        bad[0][5, 0, 0] = np.inf
        t1, s1 = srv.submit(0, 0.125, 1.0, good)
        t2, _ = srv.submit(0, 0.125, 1.0, bad + good[:1])
        t3, s3 = srv.submit(0, 0.12, 1.0, good[1:])
        ok2, st2 = srv.wait(t2, timeout=120)
        assert not ok2 and st2.converged == 0
        D = oracle.Operator(oracle.Geometry(dims), links, "Improved", 0.125, 1.0, False)
        D2 = oracle.Operator(oracle.Geometry(dims), links, "Improved", 0.12, 1.0, False)
        for t, sols, srcs, op in ((t1, s1, good, D), (t3, s3, good[1:], D2)):
            ok, st = srv.wait(t, timeout=120)
            assert ok
            assert max(_residual(op, b, x) for b, x in zip(srcs, sols)) <= 1e-10
    finally:
        srv.close()


def test_server_allocation_failure_fails_one_request(oracle):
    """The next device allocation of the lane is made to fail (host-side injection) while a
    request is being solved; the request whose admission meets it (its clover term cannot
    be allocated) ends with LYM_ERR_MEMORY, the one in flight and a later one on the same
    lane complete within tolerance."""
    dims = (16, 16, 16, 32)
    links = synth.fermion_links(dims, "su3", 0.3, 62)
    stride = -(-(int(np.prod(dims)) // 2) // 64) * 64
    clover_term_bytes = 2 * (4 * 18 * 16 + 4 * 9 * 16 + 4 * 9 * 8) * stride  # T and T^-1, FP64 / FP32 / FP16
    srcs = [synth.gaussian_spinor(dims, 3, 90 + k) for k in range(8)]
    srv = SolveServer(batch=8, precision="single", solver="bicgstab")
    try:
        srv.add_gauge(0, dims, "su3", links)
        # warm-up: afterwards the lane's engine, staging buffers and slot vectors exist, so
        # admitting a source on a new operator allocates only that operator's clover term
        t, _ = srv.submit(0, 0.12, 1.0, srcs)
        assert srv.wait(t, timeout=300)[0]
        before = srv.device_bytes()
        tE, solE = srv.submit(0, 0.125, 1.0, srcs)  # in flight while the failure happens
        deadline = time.time() + 30  # until E's clover term is allocated
        while srv.device_bytes() < before + clover_term_bytes and not srv.done(tE) and time.time() < deadline:
            time.sleep(0.0002)
        srv.inject_alloc_failures(0, 1)
        tB, _ = srv.submit(0, 0.13, 1.0, srcs[:2])  # a new operator: its clover allocation fails
        tC, solC = srv.submit(0, 0.125, 1.0, srcs[:2])  # E's operator: nothing to allocate
        with pytest.raises(L.LymError) as err:
            srv.wait(tB, timeout=300)
        assert err.value.code == ERR_MEMORY
        assert b"injected" in (srv._L.lym_server_last_error(srv._ptr) or b"")
        D = oracle.Operator(oracle.Geometry(dims), links, "Improved", 0.125, 1.0, False)
        for t, sols, bs in ((tE, solE, srcs), (tC, solC, srcs[:2])):
            ok, st = srv.wait(t, timeout=300)
            assert ok
            assert max(_residual(D, b, x) for b, x in zip(bs, sols)) <= 1e-10
        # the lane admits new operators again
        tD, solD = srv.submit(0, 0.13, 1.0, srcs[:1])
        assert srv.wait(tD, timeout=300)[0]
        D3 = oracle.Operator(oracle.Geometry(dims), links, "Improved", 0.13, 1.0, False)
        assert _residual(D3, srcs[0], solD[0]) <= 1e-10
    finally:
        srv.close()


def test_bulk_copy_wait_timeout_fails_the_call(su3, oracle):
    """The bulk-copy variant of the batched stencil records a copy wait that gave up in a
    word the host reads after the call; the reading is faked on the host (the kernels run
    as usual): the call returns LYM_ERR_TIMEOUT, and the next call on the same context, with
    the same variant, gives the oracle's result."""
    from leonardym_b200.dirac import multiply_batch, set_batch_tile
    lat = su3["lat"]
    op = L.EvenOddImprovedDiracWilsonOperator(lat, su3["kappa"], su3["csw"], gamma5=False)
    op.setLattice(su3["gid"])
    xs = [synth.gaussian_spinor(su3["dims"], 3, 700 + j) for j in range(4)]
    D = oracle.Operator(oracle.Geometry(su3["dims"]), su3["links"], "EvenOddImproved", su3["kappa"], su3["csw"],
                        False)
    try:
        set_batch_tile(lat, 0, 0, 36)
        assert L.lib().lym_context_inject_copy_wait_timeout(lat.handle) == OK
        with pytest.raises(L.LymError) as err:
            multiply_batch([op] * 4, xs, "single")
        assert err.value.code == ERR_TIMEOUT
        got = multiply_batch([op] * 4, xs, "single")
    finally:
        set_batch_tile(lat, -1, 0)
    for x, y in zip(xs, got):
        assert np.linalg.norm(y - D.multiply(x)) / np.linalg.norm(D.multiply(x)) < 1e-6
