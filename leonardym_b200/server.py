"""Solve server: resident gauge fields, continuous batching of solve requests.

Thin binding of the lym_server_* entry points (include/lym_b200.h).  The
scheduling, HBM admission and batching run in the library's worker threads.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import LymError, lib
from .dirac import REPS


class RequestStats(C.Structure):
    _fields_ = [("latency_s", C.c_double), ("queue_s", C.c_double), ("nsrc", C.c_int),
                ("max_iterations", C.c_int), ("max_true_residual", C.c_double), ("converged", C.c_int),
                ("status", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def _bind():
    L = lib()
    vp, i, dp = C.c_void_p, C.c_int, C.c_double
    L.lym_server_create.argtypes = [i, C.c_size_t, i, i, C.POINTER(vp)]
    L.lym_server_destroy.argtypes = [vp]
    L.lym_server_last_error.argtypes = [vp]
    L.lym_server_last_error.restype = C.c_char_p
    L.lym_server_device_bytes.argtypes = [vp]
    L.lym_server_device_bytes.restype = C.c_size_t
    L.lym_server_add_gauge.argtypes = [vp, i, C.POINTER(C.c_int), i, vp]
    L.lym_server_submit.argtypes = [vp, i, dp, dp, i, C.POINTER(vp), C.POINTER(vp), dp, i, C.POINTER(C.c_longlong)]
    L.lym_server_wait.argtypes = [vp, C.c_longlong, dp, C.POINTER(RequestStats)]
    L.lym_server_poll.argtypes = [vp, C.c_longlong, C.POINTER(C.c_int)]
    L.lym_server_inject_alloc_failures.argtypes = [vp, i, i]
    return L


class SolveServer:
    """Serves D x = b requests for Wilson-clover operators on resident gauge fields.

    ``precision`` is the inner storage ("single" or "half"); ``solver`` "cg" (CG on
    (gamma5 S)^2) or "bicgstab" (BiCGStab on S, falling back to CG for a source it breaks
    down on); ``batch`` the number of slots of each field's batched solver; ``hbm_budget``
    caps the server's device bytes."""

    SOLVERS = {("cg", "single"): 4, ("cg", "half"): 5, ("bicgstab", "single"): 6, ("bicgstab", "half"): 7}

    def __init__(self, device=0, hbm_budget=0, batch=16, precision="single", solver="cg"):
        self._L = _bind()
        self._ptr = C.c_void_p()
        code = self.SOLVERS[(solver, precision)]
        rc = self._L.lym_server_create(int(device), int(hbm_budget), int(batch), code, C.byref(self._ptr))
        if rc != 0:
            raise LymError(rc, "lym_server_create failed")
        self._keep = {}
        self._dims = {}

    def close(self):
        if self._ptr:
            self._L.lym_server_destroy(self._ptr)
            self._ptr = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _err(self, rc):
        raise LymError(rc, (self._L.lym_server_last_error(self._ptr) or b"").decode())

    def add_gauge(self, key, dims, rep, fermion_links):
        links = np.ascontiguousarray(fermion_links, dtype=np.complex128 if rep == "su3" else np.float64)
        d = (C.c_int * 4)(*[int(x) for x in dims])
        rc = self._L.lym_server_add_gauge(self._ptr, int(key), d, REPS[rep], links.ctypes.data_as(C.c_void_p))
        if rc != 0:
            self._err(rc)
        self._dims[int(key)] = int(np.prod(dims))

    def submit(self, key, kappa, csw, sources, tol=1e-10, max_steps=20000):
        """Queue a request; returns (ticket, solutions) where solutions fill in when done."""
        srcs = [np.ascontiguousarray(s, dtype=np.complex128) for s in sources]
        sols = [np.zeros_like(s) for s in srcs]
        n = len(srcs)
        sp = (C.c_void_p * n)(*[s.ctypes.data for s in srcs])
        xp = (C.c_void_p * n)(*[x.ctypes.data for x in sols])
        t = C.c_longlong(0)
        rc = self._L.lym_server_submit(self._ptr, int(key), float(kappa), float(csw), n, sp, xp, float(tol),
                                       int(max_steps), C.byref(t))
        if rc != 0:
            self._err(rc)
        self._keep[t.value] = (srcs, sols)  # the library writes into these buffers
        return t.value, sols

    def wait(self, ticket, timeout=600.0):
        st = RequestStats()
        rc = self._L.lym_server_wait(self._ptr, C.c_longlong(ticket), float(timeout), C.byref(st))
        if rc == -7:
            raise TimeoutError(f"request {ticket} not done after {timeout} s")
        self._keep.pop(ticket, None)
        if rc < 0:
            self._err(rc)
        return rc == 0, st

    def done(self, ticket):
        d = C.c_int(0)
        self._L.lym_server_poll(self._ptr, C.c_longlong(ticket), C.byref(d))
        return bool(d.value)

    def inject_alloc_failures(self, key, n):
        """Host-side fault injection for tests: the next n device allocations of the lane
        holding gauge field `key` fail as an out-of-memory cudaMalloc would."""
        rc = self._L.lym_server_inject_alloc_failures(self._ptr, int(key), int(n))
        if rc != 0:
            self._err(rc)

    def device_bytes(self):
        return int(self._L.lym_server_device_bytes(self._ptr))
