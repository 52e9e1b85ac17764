"""RHMC-style multishift at full size: SU(3) Wilson-clover 48^3x96 (10.6M sites), kappa 0.1365,
c_sw 1.7, 12 shifts log-spaced in [1e-4, 1] on the squared even-odd operator, FP16 inner
storage with per-site norms, FP64 recurrences.  Checked: every shift's FP64 true residual
|b - (A + sigma_i) x_i| / |b| <= 1e-10, re-measured through the library's FP64 multiplyAdd
(SquareEvenOddImprovedDiracWilsonOperator::multiplyAdd semantics), and for the smallest and
the largest shift once more on the host with the FP64 oracle's SquareEvenOddImproved
multiplyAdd (SquareEvenOddImprovedDiracWilsonOperator.cpp:13-27) at the full size (about 70 GB
of host memory and half a minute on 8 threads).  Links and source are generated on the
device (same distribution as the host generator) and copied to the host for the oracle."""
import ctypes as C

import numpy as np
import pytest

import leonardym_b200 as L
from leonardym_b200 import synth

pytestmark = pytest.mark.gpu

DIMS = (48, 48, 48, 96)
KAPPA, CSW, EPS, SEED = 0.1365, 1.7, 0.25, 1239
SHIFTS = list(np.logspace(-4, 0, 12))
TOL = 1e-10


def test_rhmc_multishift_48c96_half(oracle):
    import torch

    lib = L.lib()
    lat = L.Lattice(DIMS, "su3", device=0)
    try:
        h = lat.handle
        links = synth.su3_fermion_links_device(DIMS, EPS, SEED, "cuda:0")
        assert lib.lym_gauge_upload_device(h, 1, C.c_void_p(links.data_ptr())) == 0, lib.lym_last_error(h)
        links_host = links.cpu().numpy()
        del links
        torch.cuda.empty_cache()
        op = C.c_int(0)
        assert lib.lym_operator_create(h, 1, 5, KAPPA, CSW, 1, C.byref(op)) == 0, lib.lym_last_error(h)
        b = synth.gaussian_spinor_device(DIMS, 3, SEED + 1, "cuda:0")
        sols = [torch.zeros_like(b) for _ in SHIFTS]
        torch.cuda.synchronize()  # the library's stream does not wait for torch's
        sh = np.ascontiguousarray(SHIFTS, dtype=np.float64)
        bb = float(torch.vdot(b.flatten(), b.flatten()).real)
        ptrs = (C.c_void_p * len(SHIFTS))(*[s.data_ptr() for s in sols])
        st = L.SolveStats()
        rc = lib.lym_multishift_device(h, op.value, 5, len(SHIFTS), sh.ctypes.data_as(C.c_void_p),
                                       TOL * TOL * bb, 20000, C.c_void_p(b.data_ptr()), ptrs, C.byref(st))
        assert rc == 0, (rc, lib.lym_last_error(h))
        assert st.true_residual <= TOL
        out = torch.empty_like(b)
        worst = 0.0
        for x, s in zip(sols, SHIFTS):
            assert lib.lym_multiply_add_device(h, op.value, C.c_void_p(out.data_ptr()), C.c_void_p(x.data_ptr()),
                                               C.c_void_p(x.data_ptr()), float(s), 0.0) == 0
            r = float(torch.linalg.vector_norm((b - out).flatten())) / np.sqrt(bb)
            worst = max(worst, r)
        print(f"48^3x96 RHMC multishift (FP16 inner): {st.steps} multishift + {st.iterations - st.steps} refinement iterations, "
              f"{st.reliable_updates} reliable updates, {st.seconds:.2f} s, worst true residual {worst:.2e}")
        assert worst <= 1.02 * TOL
        # the oracle's FP64 operator on the host, smallest and largest shift
        D = oracle.Operator(oracle.Geometry(DIMS), links_host, "SquareEvenOddImproved", KAPPA, CSW, True)
        bh = b.cpu().numpy()
        for k in (0, len(SHIFTS) - 1):
            xh = sols[k].cpu().numpy()
            r = np.linalg.norm(bh - D.multiply_add(xh, xh, SHIFTS[k])) / np.linalg.norm(bh)
            print(f"shift {SHIFTS[k]:.1e}: oracle true residual {r:.2e}")
            assert r <= 1.02 * TOL, (k, r)
    finally:
        lat.close()
