"""Host-side mirror of LeonardYM's DiracOperator interface on the B200 library.

Class and method names, argument meaning and error behaviour follow the
reference (dirac_operators/DiracOperator.h:11-140, DiracOperator.cpp:20-165):

* ``multiply(output, input)`` writes the operator applied to ``input`` into
  ``output`` (DiracOperator.h:90);
* ``multiplyAdd(output, v1, v2, alpha)`` writes ``Op v1 + alpha v2`` (:99);
* ``setKappa`` / ``setCSW`` / ``setGamma5`` / ``setLattice`` (:107-127).

Vectors are numpy ``complex128[V, 4, 3]`` arrays in the reference's raw layout
(site-major, then spin, then colour); links are ``complex128[V, 4, 3, 3]``
(SU(3)) or ``float64[V, 4, 3, 3]`` (SU(2) adjoint), Eigen column-major, i.e.
``links[s, mu, j, i] = U_mu(s)(i, j)``.  Where the reference calls exit()
(DiracOperator.cpp:84-86, EvenOddImprovedDiracWilsonOperator.cpp:49-52) this
layer raises LymError.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import LymError, lib

REPS = {"su3": 0, "su2adj": 1}
BOUNDARY = {"fermion_periodic": 0, "fermion_antiperiodic": 1}
PRECISIONS = {"double": 0, "single": 1, "half": 2}


def _check(ctx_ptr, rc, ok=(0,)):
    if rc not in ok:
        msg = lib().lym_last_error(ctx_ptr)
        raise LymError(rc, msg.decode() if msg else "")
    return rc


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


class Lattice:
    """One lattice geometry and fermion representation on one GPU.

    Replaces the reference's process-global LocalLayout (MPILattice/LocalLayout.h:34-110):
    several geometries may coexist, one context each."""

    def __init__(self, dims, rep="su3", device=0):
        self.dims = tuple(int(d) for d in dims)
        self.rep = rep
        self.nc = 3
        self._ptr = C.c_void_p()
        d = (C.c_int * 4)(*self.dims)
        rc = lib().lym_context_create(d, REPS[rep], int(device), C.byref(self._ptr))
        if rc != 0:
            raise LymError(rc, f"lym_context_create({self.dims}, {rep}) failed")
        self.V = int(np.prod(self.dims))
        self._next_gauge = 1

    @property
    def handle(self):
        return self._ptr

    def close(self):
        if self._ptr:
            lib().lym_context_destroy(self._ptr)
            self._ptr = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def new_vector(self):
        return np.zeros((self.V, 4, self.nc), dtype=np.complex128)

    def link_dtype(self):
        return np.complex128 if self.rep == "su3" else np.float64

    def set_link_format(self, reals):
        """FP32 SU(3) link format of the single-RHS stencils (the mixed solvers' inner
        iterations): 12 reals (default) or 8 reals, for every gauge field of this lattice."""
        _check(self._ptr, lib().lym_set_link_format(self._ptr, int(reals)))

    def upload(self, fermion_links, gauge_id=None):
        """Make a fermion link field resident; returns its id."""
        links = np.ascontiguousarray(fermion_links, dtype=self.link_dtype())
        if links.shape != (self.V, 4, 3, 3):
            raise LymError(-1, f"links must have shape {(self.V, 4, 3, 3)}")
        gid = self._next_gauge if gauge_id is None else int(gauge_id)
        self._next_gauge = max(self._next_gauge, gid + 1)
        _check(self._ptr, lib().lym_gauge_upload(self._ptr, gid, _p(links)))
        return gid

    def upload_fundamental(self, gauge_links, boundary="fermion_antiperiodic", gauge_id=None):
        """Environment::synchronize (Environment.cpp:21-79) on the GPU: fermion links from
        fundamental links (SU(3) itself, or the adjoint of SU(2)) with the boundary condition."""
        links = np.ascontiguousarray(gauge_links, dtype=np.complex128)
        n = 3 if self.rep == "su3" else 2
        if links.shape != (self.V, 4, n, n):
            raise LymError(-1, f"gauge links must have shape {(self.V, 4, n, n)}")
        gid = self._next_gauge if gauge_id is None else int(gauge_id)
        self._next_gauge = max(self._next_gauge, gid + 1)
        _check(self._ptr, lib().lym_gauge_upload_fundamental(self._ptr, gid, _p(links), BOUNDARY[boundary]))
        return gid

    def evict(self, gauge_id):
        _check(self._ptr, lib().lym_gauge_evict(self._ptr, int(gauge_id)))

    def device_bytes(self):
        return int(lib().lym_context_device_bytes(self._ptr))

    def neighbour_tables(self):
        sup = np.empty((self.V, 4), np.int32)
        sdn = np.empty((self.V, 4), np.int32)
        _check(self._ptr, lib().lym_neighbour_tables(self._ptr, sup.ctypes.data_as(C.POINTER(C.c_int)),
                                                      sdn.ctypes.data_as(C.POINTER(C.c_int))))
        return sup, sdn

    def stencil_indices(self):
        out = np.empty((2, self.V // 2, 9), np.int32)
        _check(self._ptr, lib().lym_stencil_indices(self._ptr, out.ctypes.data_as(C.POINTER(C.c_int))))
        return out


class DiracOperator:
    """Base of the operator mirrors; subclasses fix the operator kind."""

    KIND = None
    NAME = ""

    def __init__(self, lattice, kappa=0.0, csw=0.0, gamma5=True):
        self.lattice = lattice
        self._kappa = float(kappa)
        self._csw = float(csw)
        self._gamma5 = bool(gamma5)
        self._op = None
        self._gauge = None
        self.name = self.NAME

    # -- factory (DiracOperator::getInstance, DiracOperator.cpp:20-165) --
    @staticmethod
    def getInstance(name, power, parameters, lattice, basename=""):
        table = {
            (1, "DiracWilson"): DiracWilsonOperator,
            (1, "Improved"): ImprovedDiracWilsonOperator,
            (1, "EvenOddImproved"): EvenOddImprovedDiracWilsonOperator,
            (2, "DiracWilson"): SquareDiracWilsonOperator,
            (2, "Improved"): SquareImprovedDiracWilsonOperator,
            (2, "EvenOddImproved"): SquareEvenOddImprovedDiracWilsonOperator,
        }
        cls = table.get((int(power), name))
        if cls is None:
            raise LymError(-4, f"Dirac Wilson Operator {name} (power {power}) not supported!")
        op = cls(lattice)
        op.setKappa(float(parameters[basename + "kappa"]))
        if "csw" in cls.__name__.lower() or cls.KIND in (1, 2, 4, 5):
            op.setCSW(float(parameters.get(basename + "csw", 1.0)))
        op.name = name
        return op

    # -- parameters --
    def setKappa(self, kappa):
        self._kappa = float(kappa)
        if self._op is not None:
            _check(self.lattice.handle, lib().lym_operator_set_kappa(self.lattice.handle, self._op, self._kappa))

    def getKappa(self):
        return self._kappa

    def getForce(self):
        """DiracOperator::getForce: the fermion force of this operator (on the GPU)."""
        from .rhmc import FermionForce
        return FermionForce(self)

    def setCSW(self, csw):
        self._csw = float(csw)
        if self._op is not None:
            _check(self.lattice.handle, lib().lym_operator_set_csw(self.lattice.handle, self._op, self._csw))

    def getCSW(self):
        return self._csw

    def setGamma5(self, gamma5):
        self._gamma5 = bool(gamma5)
        if self._op is not None:
            _check(self.lattice.handle, lib().lym_operator_set_gamma5(self.lattice.handle, self._op, int(self._gamma5)))

    def getGamma5(self):
        return self._gamma5

    def getName(self):
        return self.name

    def setLattice(self, fermion_links):
        """Upload (array) or attach (resident gauge id) the fermion link field."""
        if isinstance(fermion_links, (int, np.integer)):
            gid = int(fermion_links)
        else:
            gid = self.lattice.upload(fermion_links)
        self._gauge = gid
        h = self.lattice.handle
        if self._op is None:
            op = C.c_int(0)
            _check(h, lib().lym_operator_create(h, gid, self.KIND, self._kappa, self._csw, int(self._gamma5),
                                                 C.byref(op)))
            self._op = op.value
        else:
            _check(h, lib().lym_operator_set_gauge(h, self._op, gid))

    @property
    def op_id(self):
        if self._op is None:
            raise LymError(-1, "setLattice has not been called")
        return self._op

    # -- application --
    def _vec(self, v):
        a = np.ascontiguousarray(v, dtype=np.complex128)
        if a.shape != (self.lattice.V, 4, self.lattice.nc):
            raise LymError(-1, f"vector must have shape {(self.lattice.V, 4, self.lattice.nc)}")
        return a

    def multiply(self, output, input=None):
        """multiply(output, input) as the reference; multiply(input) returns a new vector."""
        if input is None:
            input, output = output, self.lattice.new_vector()
        x = self._vec(input)
        h = self.lattice.handle
        _check(h, lib().lym_multiply(h, self.op_id, _p(output), _p(x)))
        return output

    def multiplyAdd(self, output, vector1, vector2=None, alpha=None):
        """multiplyAdd(output, v1, v2, alpha) = Op v1 + alpha v2; also multiplyAdd(v1, v2, alpha)."""
        if alpha is None:
            vector1, vector2, alpha, output = output, vector1, vector2, self.lattice.new_vector()
        a = complex(alpha)
        v1, v2 = self._vec(vector1), self._vec(vector2)
        h = self.lattice.handle
        _check(h, lib().lym_multiply_add(h, self.op_id, _p(output), _p(v1), _p(v2), a.real, a.imag))
        return output

    def multiply_precision(self, input, precision="double"):
        """The operator applied with single- or half-precision storage (the sloppy stencils)."""
        x = self._vec(input)
        out = self.lattice.new_vector()
        h = self.lattice.handle
        _check(h, lib().lym_multiply_precision(h, self.op_id, PRECISIONS[precision], _p(out), _p(x)))
        return out

    def field_strength(self):
        """F_{mu nu} as ImprovedDiracWilsonOperator::updateFieldStrength computes it."""
        h = self.lattice.handle
        if self.lattice.rep == "su3":
            F = np.empty((self.lattice.V, 6, 3, 3), np.complex128)
        else:
            F = np.empty((self.lattice.V * 6 * 9 * 2,), np.float64)
        _check(h, lib().lym_field_strength(h, self.op_id, _p(F)))
        if self.lattice.rep != "su3":
            F = F[: self.lattice.V * 6 * 9].reshape(self.lattice.V, 6, 3, 3).copy()
        return F

    def destroy(self):
        if self._op is not None and self.lattice.handle:
            lib().lym_operator_destroy(self.lattice.handle, self._op)
            self._op = None


class DiracWilsonOperator(DiracOperator):
    """dirac_operators/DiracWilsonOperator.cpp:16-391"""
    KIND, NAME = 0, "DiracWilson"


class ImprovedDiracWilsonOperator(DiracOperator):
    """dirac_operators/ImprovedDiracWilsonOperator.cpp:22-523"""
    KIND, NAME = 1, "Improved"

    def __init__(self, lattice, kappa=0.0, csw=1.0, gamma5=True):
        super().__init__(lattice, kappa, csw, gamma5)


class EvenOddImprovedDiracWilsonOperator(ImprovedDiracWilsonOperator):
    """dirac_operators/EvenOddImprovedDiracWilsonOperator.cpp:26-317: odd sites get
    gamma5^g (T_oo - D_oe T_ee^-1 D_eo), even sites are copied."""
    KIND, NAME = 2, "EvenOddImproved"

    def multiplyAdd(self, *args, **kwargs):
        raise LymError(-4, "EvenOddImprovedDiracWilsonOperator::multiplyAdd not implemented")


class SquareDiracWilsonOperator(DiracOperator):
    """dirac_operators/SquareDiracWilsonOperator.cpp:12-22"""
    KIND, NAME = 3, "DiracWilson"


class SquareImprovedDiracWilsonOperator(DiracOperator):
    """dirac_operators/SquareImprovedDiracWilsonOperator.cpp:13-23"""
    KIND, NAME = 4, "Improved"

    def __init__(self, lattice, kappa=0.0, csw=1.0, gamma5=True):
        super().__init__(lattice, kappa, csw, gamma5)


class SquareEvenOddImprovedDiracWilsonOperator(DiracOperator):
    """dirac_operators/SquareEvenOddImprovedDiracWilsonOperator.cpp:13-27"""
    KIND, NAME = 5, "EvenOddImproved"

    def __init__(self, lattice, kappa=0.0, csw=1.0, gamma5=True):
        super().__init__(lattice, kappa, csw, gamma5)


def multiply_batch(operators, inputs, precision="single"):
    """EvenOddImprovedDiracWilsonOperator::multiply of operators[j] applied to inputs[j]
    for up to 32 inputs in one batched stencil (FP32 or FP16 storage).  The operators
    share the lattice, the gauge field and the gamma5 flag; kappa and c_sw may differ."""
    if len(operators) != len(inputs) or not inputs:
        raise ValueError("one operator per input")
    lat = operators[0].lattice
    xs = [operators[0]._vec(x) for x in inputs]
    outs = [lat.new_vector() for _ in xs]
    ids = (C.c_int * len(xs))(*[op.op_id for op in operators])
    ip = (C.c_void_p * len(xs))(*[x.ctypes.data for x in xs])
    op_ = (C.c_void_p * len(xs))(*[o.ctypes.data for o in outs])
    _check(lat.handle, lib().lym_multiply_batch(lat.handle, PRECISIONS[precision], len(xs), ids, ip, op_))
    return outs


def set_batch_tile(lattice, by, bz, minb=1):
    """Force the batched stencil's traversal column (by * bz sites of the (y, z) plane;
    by = 0: plain half-site order) and kernel variant (by < 0: autotune)."""
    _check(lattice.handle, lib().lym_set_batch_tile(lattice.handle, by, bz, minb))


def batch_tile(lattice, precision, batch, clover=True):
    """The (by, bz, minb) configuration the batched stencil uses for this key."""
    by, bz, mb = C.c_int(), C.c_int(), C.c_int()
    _check(lattice.handle, lib().lym_get_batch_tile(lattice.handle, PRECISIONS[precision], batch, int(clover),
                                                    C.byref(by), C.byref(bz), C.byref(mb)))
    return by.value, bz.value, mb.value
