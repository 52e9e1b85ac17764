"""The allocation-free even-odd operator entry point (lym_multiply_device_noalloc)
against the ordinary one (lym_multiply_device), through the C ABI.

It serves callers that cannot call cudaMalloc (all device memory owned by one
pre-reserved arena, or a path that must not take cudaMalloc's device-wide
synchronisation): the caller passes device vectors, the intermediate half spinor
lives in a fixed array inside the library.  This file is collected last so that a
run stopping at the first failure has run every other test first.
"""
import ctypes as C

import numpy as np
import pytest

import leonardym_b200 as L
from leonardym_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("rep,kappa,csw", [("su3", 0.13, 1.0), ("su2adj", 0.18, 1.5)])
@pytest.mark.parametrize("gamma5", [True, False])
def test_noalloc_matches_multiply_device(rep, kappa, csw, gamma5):
    import torch

    dims = (8, 8, 8, 8)
    lib = L.lib()
    lat = L.Lattice(dims, rep)
    try:
        op = L.EvenOddImprovedDiracWilsonOperator(lat, kappa, csw, gamma5)
        op.setLattice(synth.fermion_links(dims, rep, 0.3, 77))
        V = lat.V
        for call in range(2):  # two calls in a row: the shared scratch keeps the last call's contents
            x = synth.gaussian_spinor(dims, 3, 100 + call)
            dx = torch.from_numpy(x.view(np.float64).reshape(-1)).cuda()
            ref = torch.zeros_like(dx)
            out = torch.full_like(dx, float("nan"))
            torch.cuda.synchronize()  # the library's stream does not wait for torch's
            rc = lib.lym_multiply_device(lat.handle, op.op_id, C.c_void_p(ref.data_ptr()), C.c_void_p(dx.data_ptr()))
            assert rc == 0, lib.lym_last_error(lat.handle)
            rc = lib.lym_multiply_device_noalloc(lat.handle, op.op_id, C.c_void_p(out.data_ptr()),
                                                 C.c_void_p(dx.data_ptr()))
            assert rc == 0, lib.lym_last_error(lat.handle)
            a = out.cpu().numpy()
            b = ref.cpu().numpy()
            assert a.shape == (V * 24,)
            assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-13
    finally:
        lat.close()


def test_noalloc_rejects_what_it_cannot_do():
    import torch

    lib = L.lib()
    lat = L.Lattice((4, 4, 4, 4), "su3")
    try:
        op = L.EvenOddImprovedDiracWilsonOperator(lat, 0.12, 1.0)
        op.setLattice(synth.fermion_links((4, 4, 4, 4), "su3", 0.3, 78))
        d = torch.zeros(lat.V * 24, dtype=torch.float64, device="cuda")
        e = torch.zeros_like(d)
        # the clover term is not built before the first ordinary use: building it would allocate
        assert lib.lym_multiply_device_noalloc(lat.handle, op.op_id, C.c_void_p(e.data_ptr()),
                                               C.c_void_p(d.data_ptr())) == -1
        w = L.ImprovedDiracWilsonOperator(lat, 0.12, 1.0)
        w.setLattice(op._gauge)
        assert lib.lym_multiply_device_noalloc(lat.handle, w.op_id, C.c_void_p(e.data_ptr()),
                                               C.c_void_p(d.data_ptr())) == -4
        # the output may not alias the input; the reason is kept for lym_last_error
        assert lib.lym_multiply_device_noalloc(lat.handle, op.op_id, C.c_void_p(d.data_ptr()),
                                               C.c_void_p(d.data_ptr())) == -1
        assert b"distinct" in lib.lym_last_error(lat.handle)
    finally:
        lat.close()
    big = L.Lattice((16, 16, 16, 64), "su3")  # 262144 sites: beyond the fixed scratch
    try:
        op = L.EvenOddImprovedDiracWilsonOperator(big, 0.12, 1.0)
        op.setLattice(synth.fermion_links((16, 16, 16, 64), "su3", 0.3, 79))
        d = torch.zeros(big.V * 24, dtype=torch.float64, device="cuda")
        e = torch.zeros_like(d)
        assert lib.lym_multiply_device(big.handle, op.op_id, C.c_void_p(e.data_ptr()), C.c_void_p(d.data_ptr())) == 0
        assert lib.lym_multiply_device_noalloc(big.handle, op.op_id, C.c_void_p(e.data_ptr()),
                                               C.c_void_p(d.data_ptr())) == -1
        assert b"131072" in lib.lym_last_error(big.handle)
    finally:
        big.close()
