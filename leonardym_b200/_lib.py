"""ctypes binding of liblym_b200.so (the C ABI declared in include/lym_b200.h).

The shared library is the product: there is no CPU fallback.  Loading fails
loudly when the library has not been built.
"""
from __future__ import annotations

import ctypes as C
import os
import re
import subprocess

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liblym_b200.so")
HEADER_PATH = os.path.join(os.path.dirname(_HERE), "include", "lym_b200.h")
_LIB = None

OK, NOT_CONVERGED = 0, 1
STATUS_NAMES = {0: "OK", 1: "NOT_CONVERGED", -1: "ERR_ARGUMENT", -2: "ERR_CUDA", -3: "ERR_MEMORY",
                -4: "ERR_UNSUPPORTED", -5: "ERR_BREAKDOWN", -6: "ERR_NOT_FOUND", -7: "ERR_TIMEOUT",
                -8: "ERR_NUMERIC"}


class LymError(RuntimeError):
    def __init__(self, code, message):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {message}")
        self.code = code


class SolveStats(C.Structure):
    _fields_ = [("steps", C.c_int), ("iterations", C.c_int), ("reliable_updates", C.c_int),
                ("converged", C.c_int), ("last_error", C.c_double), ("true_residual", C.c_double),
                ("seconds", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def build(verbose=False):
    """Compile the CUDA library for sm_100a (nvcc cross-compiles without a GPU)."""
    out = subprocess.run(["make", "-j4", "-C", os.path.join(_HERE, "csrc")], capture_output=not verbose, text=True)
    if out.returncode != 0:
        raise RuntimeError("building liblym_b200.so failed:\n" + (out.stdout or "") + (out.stderr or ""))
    return LIB_PATH


def declared_symbols():
    """Names of every function declared in include/lym_b200.h."""
    text = open(HEADER_PATH).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(lym_[a-z0-9_]+)\s*\(", text)))


def lib():
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with leonardym_b200.build() "
                          "(the library has no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    vp, ip, dp, i = C.c_void_p, C.POINTER(C.c_int), C.c_double, C.c_int
    sp = C.POINTER(SolveStats)
    sig = {
        "lym_context_create": (i, [ip, i, i, C.POINTER(vp)]),
        "lym_context_destroy": (None, [vp]),
        "lym_last_error": (C.c_char_p, [vp]),
        "lym_context_volume": (i, [vp]),
        "lym_context_device_bytes": (C.c_size_t, [vp]),
        "lym_context_trim": (i, [vp]),
        "lym_synchronize": (i, [vp]),
        "lym_gauge_upload": (i, [vp, i, vp]),
        "lym_gauge_upload_device": (i, [vp, i, vp]),
        "lym_gauge_upload_fundamental": (i, [vp, i, vp, i]),
        "lym_gauge_evict": (i, [vp, i]),
        "lym_operator_create": (i, [vp, i, i, dp, dp, i, ip]),
        "lym_operator_set_gamma5": (i, [vp, i, i]),
        "lym_operator_set_kappa": (i, [vp, i, dp]),
        "lym_operator_set_csw": (i, [vp, i, dp]),
        "lym_operator_set_gauge": (i, [vp, i, i]),
        "lym_operator_destroy": (i, [vp, i]),
        "lym_multiply": (i, [vp, i, vp, vp]),
        "lym_multiply_add": (i, [vp, i, vp, vp, vp, dp, dp]),
        "lym_multiply_device": (i, [vp, i, vp, vp]),
        "lym_multiply_add_device": (i, [vp, i, vp, vp, vp, dp, dp]),
        "lym_multiply_device_noalloc": (i, [vp, i, vp, vp]),
        "lym_multiply_precision": (i, [vp, i, i, vp, vp]),
        "lym_field_strength": (i, [vp, i, vp]),
        "lym_solve": (i, [vp, i, i, dp, i, vp, vp, vp, sp]),
        "lym_solve_device": (i, [vp, i, i, dp, i, vp, vp, vp, sp]),
        "lym_solve_shifted": (i, [vp, i, dp, dp, dp, i, vp, vp, vp, sp]),
        "lym_solve_bicgstab_l": (i, [vp, i, i, dp, i, vp, vp, vp, sp]),
        "lym_solve_preconditioned": (i, [vp, i, i, dp, i, vp, vp, vp, sp]),
        "lym_solve_block": (i, [vp, i, i, dp, i, i, C.POINTER(vp), C.POINTER(vp), i, sp]),
        "lym_solve_block_device": (i, [vp, i, i, dp, i, i, C.POINTER(vp), C.POINTER(vp), i, sp]),
        "lym_multishift": (i, [vp, i, i, i, vp, dp, i, vp, C.POINTER(vp), sp]),
        "lym_multishift_device": (i, [vp, i, i, i, vp, dp, i, vp, C.POINTER(vp), sp]),
        "lym_rational_evaluate": (i, [vp, i, i, i, vp, vp, dp, i, vp, vp, sp]),
        "lym_meson_contractions": (i, [vp, C.POINTER(vp), vp, vp, vp]),
        "lym_meson_contractions_device": (i, [vp, C.POINTER(vp), vp, vp, vp]),
        "lym_dots_device": (i, [vp, i, C.POINTER(vp), C.POINTER(vp), i, vp]),
        "lym_noise_z2_device": (i, [vp, C.c_ulonglong, C.c_ulonglong, vp]),
        "lym_gauge_file_read": (i, [i, ip, i, C.c_char_p, C.c_char_p, i, vp, vp]),
        "lym_fermion_force": (i, [vp, i, vp, vp, dp, vp]),
        "lym_fermion_force_device": (i, [vp, i, vp, vp, dp, vp]),
        "lym_fermion_force_multi": (i, [vp, i, i, C.POINTER(vp), C.POINTER(vp), vp, vp]),
        "lym_fermion_force_multi_device": (i, [vp, i, i, C.POINTER(vp), C.POINTER(vp), vp, vp]),
        "lym_gauge_file_write": (i, [i, ip, i, vp, C.c_char_p, C.c_char_p, i, dp, dp, dp]),
        "lym_gauge_read": (i, [vp, i, i, C.c_char_p, C.c_char_p, i, i, vp]),
        "lym_meson_correlator": (i, [vp, i, i, dp, i, i, vp, vp, vp, sp]),
        "lym_chiral_condensate": (i, [vp, i, i, dp, i, i, i, C.c_ulonglong, i, vp, sp]),
        "lym_rational_evaluate_device": (i, [vp, i, i, i, vp, vp, dp, i, vp, vp, sp]),
        "lym_rhmc_force_solves": (i, [vp, i, i, i, i, vp, dp, i, vp, C.POINTER(vp), C.POINTER(vp), sp]),
        "lym_rhmc_force_solves_device": (i, [vp, i, i, i, i, vp, dp, i, vp, C.POINTER(vp), C.POINTER(vp), sp]),
        "lym_neighbour_tables": (i, [vp, ip, ip]),
        "lym_stencil_indices": (i, [vp, ip]),
        "lym_context_kernel_launches": (C.c_ulonglong, [vp]),
        "lym_context_engine_stats": (i, [vp, C.POINTER(C.c_double), i]),
        "lym_time_stencil": (i, [vp, i, i, i, i, C.POINTER(C.c_double)]),
        "lym_time_stencil_batch": (i, [vp, i, i, i, i, i, C.POINTER(C.c_double)]),
        "lym_multiply_batch": (i, [vp, i, i, C.POINTER(C.c_int), C.POINTER(vp), C.POINTER(vp)]),
        "lym_set_batch_tile": (i, [vp, i, i, i]),
        "lym_get_batch_tile": (i, [vp, i, i, i, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
        "lym_context_inject_alloc_failures": (i, [vp, i]),
        "lym_context_inject_copy_wait_timeout": (i, [vp]),
        "lym_set_link_format": (i, [vp, i]),
        "lym_host_alloc": (vp, [C.c_size_t]),
        "lym_host_free": (None, [vp]),
    }
    for name, (res, args) in sig.items():
        if not hasattr(L, name):
            continue
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _LIB = L
    return L
