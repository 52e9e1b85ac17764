"""ctypes bindings of the reference's own hot path compiled from its sources
(oracle/build_ref.sh -> oracle/_ref/libleonard_ref_{su3,su2adj}.so).

TEST INFRASTRUCTURE ONLY: used to pin the oracle restatement, to generate the
golden fixtures, and as bench.py's CPU baseline ("kind": "reference").
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS = {}
KIND = {"DiracWilson": 0, "Improved": 1, "EvenOddImproved": 2, "SquareDiracWilson": 3, "SquareImproved": 4,
        "SquareEvenOddImproved": 5, "BasicDiracWilson": 6}
SOLVER = {"cg": 0, "bicgstab": 1, "preconditioned_bicgstab": 2, "bicgstab_shifted": 3}


def path(rep):
    """rep: "su3", "su2adj" (portable builds) or "su3_native" (-march=native)."""
    return os.path.join(_HERE, "_ref", f"libleonard_ref_{rep}.so")


def available(rep="su3"):
    return os.path.exists(path(rep))


_PROBE = """
import sys, numpy as np
sys.path.insert(0, sys.argv[1])
from oracle import ref as R
dims = (4, 4, 4, 4)
rng = np.random.default_rng(5)
links = np.empty((256, 4, 3, 3), np.complex128)
for k in range(256 * 4):
    q, _ = np.linalg.qr(rng.normal(size=(3, 3)) + 1j * rng.normal(size=(3, 3)))
    links.reshape(-1, 3, 3)[k] = q
x = rng.normal(size=(256, 4, 3)) + 1j * rng.normal(size=(256, 4, 3))
ref = R.Reference(dims, links, sys.argv[2])
y = ref.multiply("EvenOddImproved", x, 0.13, 1.0, False)
z = R.Reference(dims, links, "su3").multiply("EvenOddImproved", x, 0.13, 1.0, False)
assert np.linalg.norm(y - z) <= 1e-12 * np.linalg.norm(z)
"""


def runs_here(rep):
    """True when the build `rep` loads and computes correctly on this host, tried in a
    child process (a build for another CPU ends the child, not the caller)."""
    import subprocess
    import sys
    if not available(rep):
        return False
    root = os.path.dirname(_HERE)
    try:
        r = subprocess.run([sys.executable, "-c", _PROBE, root, rep], capture_output=True, timeout=300,
                           env={**os.environ, "OMP_NUM_THREADS": "1"})
    except subprocess.TimeoutExpired:
        return False
    return r.returncode == 0


def lib(rep):
    if rep not in _LIBS:
        L = C.CDLL(path(rep))
        vp, ip, dp, i = C.c_void_p, C.POINTER(C.c_int), C.c_double, C.c_int
        L.ref_multiply.argtypes = [ip, i, dp, dp, i, vp, vp, vp]
        L.ref_multiply_add.argtypes = [ip, i, dp, dp, i, vp, vp, vp, dp, dp, vp]
        L.ref_field_strength.argtypes = [ip, dp, dp, vp, vp]
        L.ref_solve.argtypes = [ip, i, dp, dp, i, vp, i, dp, i, dp, dp, vp, vp, ip]
        L.ref_solve2.argtypes = [ip, i, dp, dp, i, vp, i, dp, i, i, i, dp, dp, vp, vp, ip]
        L.ref_multishift.argtypes = [ip, i, dp, dp, i, vp, i, i, vp, dp, i, vp, C.POINTER(C.c_void_p)]
        L.ref_rational_evaluate.argtypes = [ip, i, dp, dp, i, vp, i, i, vp, vp, dp, i, vp, vp]
        L.ref_fermion_force.argtypes = [ip, i, dp, dp, vp, vp, vp, dp, vp]
        L.ref_neighbours.argtypes = [ip, ip, ip]
        L.ref_antiperiodic.argtypes = [ip, vp]
        if hasattr(L, "ref_to_adjoint"):
            L.ref_to_adjoint.argtypes = [i, vp, vp]
        L.ref_meson_correlator.argtypes = [ip, dp, dp, vp, dp, i, vp]
        L.ref_chiral_condensate.argtypes = [ip, dp, dp, vp, dp, i, i, i, C.c_uint, vp, vp]
        L.ref_gauge_write.argtypes = [ip, i, C.c_char_p, C.c_char_p, i, vp, dp, dp]
        L.ref_gauge_read.argtypes = [ip, i, C.c_char_p, C.c_char_p, i, vp, dp, dp]
        L.ref_bench_prepare.argtypes = [ip, dp, dp, vp]
        L.ref_bench_solve.argtypes = [dp, i, vp, vp, ip]
        L.ref_bench_release.argtypes = []
        _LIBS[rep] = L
    return _LIBS[rep]


def _d(dims):
    return (C.c_int * 4)(*[int(x) for x in dims])


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


FORMATS = {"leonard_format": 0, "muenster_format": 1}


def _dirname(directory):
    d = str(directory)
    return (d if d.endswith(os.sep) else d + os.sep).encode()


def gauge_write(rep, dims, format_name, directory, name, number, links, beta=0.0, kappa=0.0):
    """io/OutputSweep.cpp's writer (one process) on fundamental links complex128[V, 4, N, N]
    (N = 3 for the "su3" build, 2 for "su2adj"); the file number is `number`."""
    links = np.ascontiguousarray(links, np.complex128)
    rc = lib(rep).ref_gauge_write(_d(dims), FORMATS[format_name], _dirname(directory), str(name).encode(),
                                  int(number), _p(links), float(beta), float(kappa))
    assert rc == 0


def gauge_read(rep, dims, format_name, directory, name, number, beta=0.0, kappa=0.0):
    """ReadStartGaugeConfiguration::readConfiguration: (success, fundamental links)."""
    n = 3 if rep.startswith("su3") else 2
    links = np.zeros((int(np.prod(dims)), 4, n, n), np.complex128)
    rc = lib(rep).ref_gauge_read(_d(dims), FORMATS[format_name], _dirname(directory), str(name).encode(),
                                 int(number), _p(links), float(beta), float(kappa))
    return rc == 1, links


class Reference:
    """The reference operators and solvers on one link field."""

    def __init__(self, dims, links, rep=None):
        self.dims = tuple(int(x) for x in dims)
        self.links = np.ascontiguousarray(links)
        self.rep = rep or ("su3" if np.iscomplexobj(self.links) else "su2adj")
        self.L = lib(self.rep)
        self.V = int(np.prod(self.dims))

    def _vec(self):
        return np.zeros((self.V, 4, 3), np.complex128)

    def multiply(self, kind, x, kappa, csw=0.0, gamma5=True):
        x = np.ascontiguousarray(x, np.complex128)
        out = self._vec()
        rc = self.L.ref_multiply(_d(self.dims), KIND[kind], kappa, csw, int(gamma5), _p(self.links), _p(x), _p(out))
        assert rc == 0
        return out

    def multiply_add(self, kind, x, y, alpha, kappa, csw=0.0, gamma5=True):
        x = np.ascontiguousarray(x, np.complex128)
        y = np.ascontiguousarray(y, np.complex128)
        out = self._vec()
        a = complex(alpha)
        rc = self.L.ref_multiply_add(_d(self.dims), KIND[kind], kappa, csw, int(gamma5), _p(self.links), _p(x), _p(y),
                                     a.real, a.imag, _p(out))
        assert rc == 0
        return out

    def field_strength(self, kappa, csw):
        dt = np.complex128 if self.rep == "su3" else np.float64
        F = np.zeros((self.V, 6, 3, 3), dt)
        self.L.ref_field_strength(_d(self.dims), kappa, csw, _p(self.links), _p(F))
        return F

    def solve(self, kind, solver, b, precision, max_steps, kappa, csw=0.0, gamma5=True, shift=0.0):
        b = np.ascontiguousarray(b, np.complex128)
        x = self._vec()
        steps = C.c_int(0)
        s = complex(shift)
        rc = self.L.ref_solve(_d(self.dims), KIND[kind], kappa, csw, int(gamma5), _p(self.links), SOLVER[solver],
                              float(precision), int(max_steps), s.real, s.imag, _p(b), _p(x), C.byref(steps))
        return rc, x, steps.value

    # the reference's propagator consumers on these links (Improved operator, default options)
    def meson_correlator(self, kappa, csw, precision, max_steps):
        """MesonCorrelator::execute: pion_exact, scalar_exact, ps_exact, pcac_mass per t."""
        Lt = self.dims[3]
        out = np.zeros(4 * Lt)
        rc = self.L.ref_meson_correlator(_d(self.dims), float(kappa), float(csw), _p(self.links), float(precision),
                                         int(max_steps), _p(out))
        assert rc == 0
        o = out.reshape(4, Lt)
        return {"pion_exact": o[0], "scalar_exact": o[1], "ps_exact": o[2], "pcac_mass": o[3]}

    def chiral_condensate(self, kappa, csw, precision, max_steps, n, connected, seed):
        """ChiralCondensate::execute with n estimators from a seeded generator (one thread):
        (mean, standard deviation) of condensate, pseudo-condensate, connected part and pion
        norm (re, im each), and the real Z2 noise vectors the reference drew."""
        out = np.zeros(16)
        noise = np.zeros((n, self.V, 4, 3))
        rc = self.L.ref_chiral_condensate(_d(self.dims), float(kappa), float(csw), _p(self.links), float(precision),
                                          int(max_steps), int(n), int(bool(connected)), int(seed), _p(out),
                                          _p(noise))
        assert rc == 0
        return out.reshape(8, 2), noise.astype(np.complex128)

    # the benchmark's CPU baseline: PreconditionedBiCGStab::solve on one held Improved operator
    def bench_prepare(self, kappa, csw):
        rc = self.L.ref_bench_prepare(_d(self.dims), float(kappa), float(csw), _p(self.links))
        assert rc == 0

    def bench_solve(self, b, precision, max_steps, keep_solution=True):
        b = np.ascontiguousarray(b, np.complex128)
        x = self._vec() if keep_solution else None
        steps = C.c_int(0)
        rc = self.L.ref_bench_solve(float(precision), int(max_steps), _p(b), _p(x) if x is not None else None,
                                    C.byref(steps))
        return rc, x, steps.value

    def bench_release(self):
        self.L.ref_bench_release()

    def solve2(self, kind, solver, b, precision, max_steps, kappa, csw=0.0, gamma5=True, l=2, pre_kind="DiracWilson",
               pre_kappa=0.1, pre_csw=0.0):
        """BiCGStab(l) (solver "bicgstab_l") or BiCGStab with a preconditioner operator
        (solver "bicgstab_precond") of the compiled reference."""
        b = np.ascontiguousarray(b, np.complex128)
        x = self._vec()
        steps = C.c_int(0)
        rc = self.L.ref_solve2(_d(self.dims), KIND[kind], kappa, csw, int(gamma5), _p(self.links),
                               {"bicgstab_l": 0, "bicgstab_precond": 1}[solver], float(precision), int(max_steps),
                               int(l), KIND[pre_kind], float(pre_kappa), float(pre_csw), _p(b), _p(x), C.byref(steps))
        return rc, x, steps.value

    def multishift(self, kind, algorithm, b, shifts, epsilon, max_steps, kappa, csw=0.0, gamma5=True):
        b = np.ascontiguousarray(b, np.complex128)
        sols = [self._vec() for _ in shifts]
        ptrs = (C.c_void_p * len(sols))(*[s.ctypes.data for s in sols])
        sh = np.ascontiguousarray(shifts, np.float64)
        alg = {"mass_estrapolation": 0, "minimal_residual": 1, "chronological_mass_estrapolation": 2}[algorithm]
        rc = self.L.ref_multishift(_d(self.dims), KIND[kind], kappa, csw, int(gamma5), _p(self.links), alg,
                                   len(shifts), _p(sh), float(epsilon), int(max_steps), _p(b), ptrs)
        return rc, sols


def _rational(self, kind, algorithm, alphas, betas, b, precision, max_steps, kappa, csw=0.0, gamma5=True):
    b = np.ascontiguousarray(b, np.complex128)
    out = self._vec()
    a = np.ascontiguousarray(alphas, np.float64)
    be = np.ascontiguousarray(betas, np.float64)
    alg = {"mass_estrapolation": 0, "minimal_residual": 1}[algorithm]
    rc = self.L.ref_rational_evaluate(_d(self.dims), KIND[kind], kappa, csw, int(gamma5), _p(self.links), alg,
                                      len(a), _p(a), _p(be), float(precision), int(max_steps), _p(b), _p(out))
    return rc, out


Reference.rational_evaluate = _rational


def _fermion_force(self, kind, kappa, csw, X, Y, weight, force):
    """FermionForce::derivative of DiracWilsonFermionForce ("DiracWilson") or
    ImprovedFermionForce ("Improved"); returns force - weight * derivative."""
    X = np.ascontiguousarray(X, np.complex128)
    Y = np.ascontiguousarray(Y, np.complex128)
    out = np.ascontiguousarray(force, np.complex128).copy()
    self.L.ref_fermion_force(_d(self.dims), {"DiracWilson": 0, "Improved": 1}[kind], kappa, csw, _p(self.links),
                             _p(X), _p(Y), float(weight), _p(out))
    return out


Reference.fermion_force = _fermion_force


def neighbours(dims, rep="su3"):
    V = int(np.prod(dims))
    sup = np.zeros((V, 4), np.int32)
    sdn = np.zeros((V, 4), np.int32)
    lib(rep).ref_neighbours(_d(dims), sup.ctypes.data_as(C.POINTER(C.c_int)), sdn.ctypes.data_as(C.POINTER(C.c_int)))
    return sup, sdn


def antiperiodic(dims, links, rep):
    out = np.ascontiguousarray(links).copy()
    lib(rep).ref_antiperiodic(_d(dims), _p(out))
    return out


def to_adjoint(fund):
    fund = np.ascontiguousarray(fund, np.complex128)
    n = fund.size // 4
    adj = np.zeros(fund.shape[:-2] + (3, 3), np.float64)
    lib("su2adj").ref_to_adjoint(n, _p(fund), _p(adj))
    return adj
