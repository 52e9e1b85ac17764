"""ctypes bindings of the CPU oracle (liblym_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg as the checker.  The product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

KIND = {"DiracWilson": 0, "Improved": 1, "EvenOddImproved": 2,
        "SquareDiracWilson": 3, "SquareImproved": 4, "SquareEvenOddImproved": 5}


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liblym_oracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        vp, ip, dp = C.c_void_p, C.POINTER(C.c_int), C.c_double
        L.orc_geom_tables.argtypes = [ip, vp, vp, vp]
        L.orc_op_init.argtypes = [vp, vp, C.c_int, C.c_int, C.c_int, vp, dp, dp, C.c_int]
        L.orc_multiply.argtypes = [vp, vp, vp]
        L.orc_multiply_add.argtypes = [vp, vp, vp, vp, dp, dp]
        L.orc_cg.argtypes = [vp, vp, vp, vp, dp, C.c_int, ip]
        L.orc_bicgstab.argtypes = [vp, vp, vp, vp, dp, C.c_int, ip, C.POINTER(C.c_double)]
        L.orc_bicgstab_shifted.argtypes = [vp, vp, vp, dp, dp, vp, dp, C.c_int, ip, C.POINTER(C.c_double)]
        L.orc_preconditioned_bicgstab.argtypes = [vp, vp, vp, vp, dp, C.c_int, ip]
        L.orc_me_multishift.argtypes = [vp, vp, C.POINTER(C.c_void_p), C.POINTER(C.c_double), C.c_int, dp, C.c_int]
        L.orc_mmmr_multishift.argtypes = [vp, vp, C.POINTER(C.c_void_p), C.POINTER(C.c_double), C.c_int, dp, C.c_int, ip]
        L.orc_bicgstab_l.argtypes = [vp, C.c_int, vp, vp, vp, dp, C.c_int, ip, C.POINTER(C.c_double)]
        L.orc_bicgstab_precond.argtypes = [vp, vp, vp, vp, vp, dp, C.c_int, ip, C.POINTER(C.c_double)]
        L.orc_chrono_multishift.argtypes = [vp, vp, C.POINTER(C.c_void_p), C.POINTER(C.c_double), C.c_int, dp,
                                            C.c_int]
        L.orc_op_field_strength.argtypes = [vp]
        L.orc_op_field_strength.restype = vp
        L.orc_eo_multiply_even_odd.argtypes = [vp, vp, vp, C.c_int]
        L.orc_eo_multiply_even_even_inverse.argtypes = [vp, vp]
        L.orc_eo_multiply_odd_odd_minus_identity.argtypes = [vp, vp, vp, C.c_int]
        L.orc_geom_init.argtypes = [vp, ip]
        L.orc_geom_free.argtypes = [vp]
        L.orc_op_free.argtypes = [vp]
        L.orc_antiperiodic_bc.argtypes = [ip, vp, C.c_int, C.c_int]
        L.orc_su2_to_adjoint.argtypes = [C.c_int, vp, vp]
        _LIB = L
    return _LIB


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def _ints(v):
    return (C.c_int * len(v))(*[int(x) for x in v])


class _Geom(C.Structure):
    _fields_ = [("dims", C.c_int * 4), ("V", C.c_int), ("sup", C.c_void_p),
                ("sdn", C.c_void_p), ("coord", C.c_void_p)]


class _Op(C.Structure):
    _fields_ = [("g", C.c_void_p), ("nc", C.c_int), ("real_links", C.c_int), ("kind", C.c_int),
                ("links", C.c_void_p), ("F", C.c_void_p), ("Tinv", C.c_void_p),
                ("kappa", C.c_double), ("csw", C.c_double), ("gamma5", C.c_int)]


def geom_tables(dims):
    V = int(np.prod(dims))
    sup = np.empty((V, 4), np.int32)
    sdn = np.empty((V, 4), np.int32)
    coord = np.empty((V, 4), np.int32)
    lib().orc_geom_tables(_ints(dims), _ptr(sup), _ptr(sdn), _ptr(coord))
    return sup, sdn, coord


class Geometry:
    def __init__(self, dims):
        self.dims = tuple(int(d) for d in dims)
        self._g = _Geom()
        rc = lib().orc_geom_init(C.byref(self._g), _ints(self.dims))
        if rc != 0:
            raise RuntimeError(f"orc_geom_init failed: {rc}")
        self.V = self._g.V

    def __del__(self):
        try:
            lib().orc_geom_free(C.byref(self._g))
        except Exception:
            pass


class Operator:
    """Oracle operator of one kind over a fixed fermion-link field."""

    def __init__(self, geom, links, kind, kappa, csw=0.0, gamma5=True):
        self.geom = geom
        self.links = np.ascontiguousarray(links)
        self.real = not np.iscomplexobj(self.links)
        self.nc = int(self.links.shape[-1])
        self._op = _Op()
        k = KIND[kind] if isinstance(kind, str) else int(kind)
        rc = lib().orc_op_init(C.byref(self._op), C.byref(geom._g), self.nc, int(self.real), k,
                               _ptr(self.links), float(kappa), float(csw), int(bool(gamma5)))
        if rc != 0:
            raise RuntimeError(f"orc_op_init failed: {rc}")

    def __del__(self):
        try:
            lib().orc_op_free(C.byref(self._op))
        except Exception:
            pass

    def _vec(self):
        return np.zeros((self.geom.V, 4, self.nc), np.complex128)

    def multiply(self, vin):
        vin = np.ascontiguousarray(vin, dtype=np.complex128)
        out = self._vec()
        rc = lib().orc_multiply(C.byref(self._op), _ptr(out), _ptr(vin))
        if rc != 0:
            raise RuntimeError(f"orc_multiply failed: {rc}")
        return out

    def multiply_add(self, v1, v2, alpha):
        v1 = np.ascontiguousarray(v1, dtype=np.complex128)
        v2 = np.ascontiguousarray(v2, dtype=np.complex128)
        out = self._vec()
        a = complex(alpha)
        rc = lib().orc_multiply_add(C.byref(self._op), _ptr(out), _ptr(v1), _ptr(v2), a.real, a.imag)
        if rc != 0:
            raise RuntimeError(f"orc_multiply_add failed: {rc}")
        return out

    def field_strength(self):
        p = lib().orc_op_field_strength(C.byref(self._op))
        n = self.geom.V * 6 * self.nc * self.nc
        if self.real:
            arr = np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_double)), shape=(n,))
            return arr.copy().reshape(self.geom.V, 6, self.nc, self.nc)
        arr = np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_double)), shape=(2 * n,))
        return arr.copy().view(np.complex128).reshape(self.geom.V, 6, self.nc, self.nc)

    def even_odd(self, vin, part, out=None):
        vin = np.ascontiguousarray(vin, dtype=np.complex128)
        out = self._vec() if out is None else out
        lib().orc_eo_multiply_even_odd(C.byref(self._op), _ptr(out), _ptr(vin), int(part))
        return out

    def even_even_inverse(self, v):
        v = np.ascontiguousarray(v, dtype=np.complex128).copy()
        lib().orc_eo_multiply_even_even_inverse(C.byref(self._op), _ptr(v))
        return v

    def odd_odd_minus_identity(self, out, vin, part):
        out = np.ascontiguousarray(out, dtype=np.complex128).copy()
        vin = np.ascontiguousarray(vin, dtype=np.complex128)
        lib().orc_eo_multiply_odd_odd_minus_identity(C.byref(self._op), _ptr(out), _ptr(vin), int(part))
        return out


def cg(op, src, eps, max_steps=3000, guess=None):
    src = np.ascontiguousarray(src, dtype=np.complex128)
    sol = op._vec()
    steps = C.c_int(0)
    g = _ptr(np.ascontiguousarray(guess, dtype=np.complex128)) if guess is not None else None
    rc = lib().orc_cg(C.byref(op._op), _ptr(src), _ptr(sol), g, float(eps), int(max_steps), C.byref(steps))
    return rc, sol, steps.value


def bicgstab(op, src, precision, max_steps=1000, guess=None, shift=None):
    src = np.ascontiguousarray(src, dtype=np.complex128)
    sol = op._vec()
    steps = C.c_int(0)
    last = C.c_double(0)
    g = _ptr(np.ascontiguousarray(guess, dtype=np.complex128)) if guess is not None else None
    if shift is None:
        rc = lib().orc_bicgstab(C.byref(op._op), _ptr(src), _ptr(sol), g, float(precision), int(max_steps),
                                C.byref(steps), C.byref(last))
    else:
        s = complex(shift)
        rc = lib().orc_bicgstab_shifted(C.byref(op._op), _ptr(src), _ptr(sol), s.real, s.imag, g, float(precision),
                                        int(max_steps), C.byref(steps), C.byref(last))
    return rc, sol, steps.value


def preconditioned_bicgstab(op, src, precision, max_steps=1000, guess=None):
    src = np.ascontiguousarray(src, dtype=np.complex128)
    sol = op._vec()
    steps = C.c_int(0)
    g = _ptr(np.ascontiguousarray(guess, dtype=np.complex128)) if guess is not None else None
    rc = lib().orc_preconditioned_bicgstab(C.byref(op._op), _ptr(src), _ptr(sol), g, float(precision),
                                           int(max_steps), C.byref(steps))
    return rc, sol, steps.value


def _multishift(fn, op, src, shifts, eps, max_steps, with_steps):
    src = np.ascontiguousarray(src, dtype=np.complex128)
    sols = [op._vec() for _ in shifts]
    ptrs = (C.c_void_p * len(sols))(*[s.ctypes.data for s in sols])
    sh = (C.c_double * len(shifts))(*[float(s) for s in shifts])
    if with_steps:
        steps = C.c_int(0)
        rc = fn(C.byref(op._op), _ptr(src), ptrs, sh, len(shifts), float(eps), int(max_steps), C.byref(steps))
        return rc, sols, steps.value
    rc = fn(C.byref(op._op), _ptr(src), ptrs, sh, len(shifts), float(eps), int(max_steps))
    return rc, sols, None


def bicgstab_l(op, l, src, precision, max_steps=1000, guess=None):
    """BiCGStab(l) (inverters/BiConjugateGradient.cpp:130-317)."""
    src = np.ascontiguousarray(src, dtype=np.complex128)
    sol = op._vec()
    steps, last = C.c_int(0), C.c_double(0)
    g = _ptr(np.ascontiguousarray(guess, dtype=np.complex128)) if guess is not None else None
    rc = lib().orc_bicgstab_l(C.byref(op._op), int(l), _ptr(src), _ptr(sol), g, float(precision), int(max_steps),
                              C.byref(steps), C.byref(last))
    return rc, sol, steps.value


def bicgstab_precond(op, pre, src, precision, max_steps=1000, guess=None):
    """BiCGStab with a preconditioner operator (inverters/BiConjugateGradient.cpp:11-128)."""
    src = np.ascontiguousarray(src, dtype=np.complex128)
    sol = op._vec()
    steps, last = C.c_int(0), C.c_double(0)
    g = _ptr(np.ascontiguousarray(guess, dtype=np.complex128)) if guess is not None else None
    rc = lib().orc_bicgstab_precond(C.byref(op._op), C.byref(pre._op), _ptr(src), _ptr(sol), g, float(precision),
                                    int(max_steps), C.byref(steps), C.byref(last))
    return rc, sol, steps.value


def chrono_multishift(op, src, shifts, eps, max_steps=3000, previous=None):
    """ChronologicalMultishiftSolver (inverters/ChronologicalMultishiftSolver.cpp:11-194);
    previous[k]: the chronological guess of shift k (zeros when None)."""
    src = np.ascontiguousarray(src, dtype=np.complex128)
    sols = [np.ascontiguousarray(previous[k], dtype=np.complex128).copy() if previous is not None else op._vec()
            for k in range(len(shifts))]
    ptrs = (C.c_void_p * len(sols))(*[s.ctypes.data for s in sols])
    sh = (C.c_double * len(shifts))(*[float(s) for s in shifts])
    rc = lib().orc_chrono_multishift(C.byref(op._op), _ptr(src), ptrs, sh, len(shifts), float(eps), int(max_steps))
    return rc, sols


def me_multishift(op, src, shifts, eps, max_steps=3000):
    return _multishift(lib().orc_me_multishift, op, src, shifts, eps, max_steps, False)


def mmmr_multishift(op, src, shifts, eps, max_steps=3000):
    return _multishift(lib().orc_mmmr_multishift, op, src, shifts, eps, max_steps, True)


def rational_evaluate(op, alphas, betas, src, precision=1e-12, max_steps=3000, algorithm="mass_estrapolation"):
    """RationalApproximation::evaluate (dirac_functions/RationalApproximation.cpp:18-42): the
    multishift solutions x_i = (A + beta_i)^{-1} src, then output = sum_i alpha_i x_i
    (zeroed, then accumulated in the order of the approximation's terms)."""
    fn = {"mass_estrapolation": me_multishift, "minimal_residual": mmmr_multishift}[algorithm]
    rc, xs, _ = fn(op, src, list(betas), precision, max_steps)
    out = np.zeros_like(xs[0])
    for a, x in zip(alphas, xs):
        out += float(a) * x
    return rc, out


def rational_value(alphas, betas, x):
    """RationalApproximation::evaluate(const complex&) (RationalApproximation.cpp:44-52):
    sum_i alpha_i / (x + beta_i)."""
    r = 0j
    for a, b in zip(alphas, betas):
        r += a / (x + b)
    return r


def rhmc_energy(op, approximations, pseudofermions, precision=1e-12, max_steps=3000):
    """NFlavorFermionAction::energy (actions/NFlavorFermionAction.cpp:193-207): the sum over
    the (alphas, betas) approximations of Re <phi_k, r_k(A) phi_k> on the squared operator."""
    e = 0.0
    for (alphas, betas), phi in zip(approximations, pseudofermions):
        _, out = rational_evaluate(op, alphas, betas, phi, precision, max_steps)
        e += float(np.vdot(phi, out).real)
    return e


def rhmc_force_solves(square_op, dirac_op, betas, phi, precision=1e-12, max_steps=3000):
    """The solves of NFlavorFermionAction::updateForce (NFlavorFermionAction.cpp:76-96) for
    one pseudofermion: x_i = (A + beta_i)^{-1} phi (mass-estrapolation multishift on the
    squared operator), y_i = D x_i."""
    rc, xs, _ = me_multishift(square_op, phi, list(betas), precision, max_steps)
    return rc, xs, [dirac_op.multiply(x) for x in xs]


# gamma_t and gamma5 of the chiral basis (the reference's Gamma tables gammamu[3] and
# _gamma5, utils/Gamma.cpp:9-11)
GAMMA_T = np.array([[0, 0, 1, 0], [0, 0, 0, 1], [1, 0, 0, 0], [0, 1, 0, 0]], dtype=np.complex128)
GAMMA5 = np.diag([1.0, 1.0, -1.0, -1.0]).astype(np.complex128)
GAMMA5_GAMMA_T = GAMMA5 @ GAMMA_T


def point_sources(dims, nc=3):
    """StochasticEstimator::generateSource (StochasticEstimator.cpp:100-112) for every spin
    alpha and colour c, in MesonCorrelator's order c * 4 + alpha."""
    V = int(np.prod(dims))
    out = []
    for c in range(nc):
        for alpha in range(4):
            v = np.zeros((V, 4, nc), dtype=np.complex128)
            v[0, alpha, c] = 1.0
            out.append(v)
    return out


def meson_contractions(props, dims):
    """The connected correlators of MesonCorrelator::execute (MesonCorrelator.cpp:98-157) of
    the 12 point-source propagators props[c * 4 + alpha] (V, 4, 3): per time slice the pion,
    scalar and PS summator results (before the 4 kappa^2 of the output)."""
    V, Lt = int(np.prod(dims)), int(dims[3])
    P = np.stack(props).reshape(3, 4, V, 4, 3)  # [c][alpha][site][mu][d]
    t = np.arange(V) % Lt
    G, g = GAMMA5_GAMMA_T, GAMMA_T
    pion = np.einsum("casmd,casmd->s", P.conj(), P).real
    scalar = np.einsum("mn,ab,casmd,cbsnd->s", G, G, P.conj(), P).real
    ps = (-np.einsum("ab,casmd,cbsmd->s", g, P.conj(), P) + np.einsum("ab,cmsad,cmsbd->s", g, P.conj(), P)).real
    return tuple(np.bincount(t, weights=w, minlength=Lt) for w in (pion, scalar, ps))


def meson_contractions_loops(props, dims):
    """meson_contractions loop for loop as MesonCorrelator.cpp:98-157 (small lattices only)."""
    V, Lt = int(np.prod(dims)), int(dims[3])
    pion, scalar, ps = np.zeros(Lt), np.zeros(Lt), np.zeros(Lt)
    for alpha in range(4):
        for c in range(3):
            for site in range(V):
                for mu in range(4):
                    for d in range(3):
                        v = props[c * 4 + alpha][site, mu, d]
                        pion[site % Lt] += (v.conjugate() * v).real
    for alpha in range(4):
        for beta in range(4):
            for c in range(3):
                for site in range(V):
                    for mu in range(4):
                        for nu in range(4):
                            for d in range(3):
                                z = (GAMMA5_GAMMA_T[mu, nu] * GAMMA5_GAMMA_T[alpha, beta] *
                                     props[c * 4 + alpha][site, mu, d].conjugate() * props[c * 4 + beta][site, nu, d])
                                scalar[site % Lt] += z.real
    for alpha in range(4):
        for beta in range(4):
            for c in range(3):
                for site in range(V):
                    for mu in range(4):
                        for d in range(3):
                            z = -GAMMA_T[alpha, beta] * (props[c * 4 + alpha][site, mu, d].conjugate() *
                                                          props[c * 4 + beta][site, mu, d])
                            z += GAMMA_T[alpha, beta] * (props[c * 4 + mu][site, alpha, d].conjugate() *
                                                         props[c * 4 + mu][site, beta, d])
                            ps[site % Lt] += z.real
    return pion, scalar, ps


def meson_output(pion, scalar, ps, kappa):
    """The normalised correlators and PCAC mass MesonCorrelator writes (MesonCorrelator.cpp:160-193)."""
    Lt = len(pion)
    f = 4.0 * kappa * kappa
    pcac = [(ps[(t - 1) % Lt] - ps[(t + 1) % Lt]) / (4.0 * pion[t]) for t in range(Lt)]
    return {"pion_exact": list(f * np.asarray(pion)), "scalar_exact": list(f * np.asarray(scalar)),
            "ps_exact": list(f * np.asarray(ps)), "pcac_mass": pcac}


def _splitmix64(z):
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def z2_noise(dims, seed, stream, nc=3):
    """The library's real Z2 noise (lym_noise_z2_device): component j of vector `stream` is
    +1 where the top bit of splitmix64(seed + 0x9E3779B97F4A7C15 (stream 12 V + j + 1)) is
    set, else -1 (StochasticEstimator.h:16-31 draws +-1 from a time-seeded generator)."""
    V = int(np.prod(dims))
    n = V * 4 * nc
    with np.errstate(over="ignore"):
        j = np.arange(n, dtype=np.uint64)
        z = np.uint64(seed) + np.uint64(0x9E3779B97F4A7C15) * (np.uint64(stream) * np.uint64(n) + j + np.uint64(1))
        z = _splitmix64(z)
    return np.where((z >> np.uint64(63)) == 1, 1.0, -1.0).astype(np.complex128).reshape(V, 4, nc)


def condensate_estimator(eta, x, y=None):
    """One estimator of ChiralCondensate::execute (ChiralCondensate.cpp:92-118): <eta,x>/V,
    <eta,gamma5 x>/V, <x,x>/V and <eta,y>/V (x = D^-1 eta, y = D^-1 x)."""
    V = eta.shape[0]
    g5x = x.copy()
    g5x[:, 2:, :] *= -1
    out = [np.vdot(eta, x) / V, np.vdot(eta, g5x) / V, np.vdot(x, x) / V, (np.vdot(eta, y) / V) if y is not None else 0j]
    return np.array([[z.real, z.imag] for z in out]).reshape(8)


def squared_norm(v):
    return float(np.vdot(v, v).real)


def dot(a, b):
    return complex(np.vdot(a, b))
