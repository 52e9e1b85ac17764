"""Seeded synthetic inputs: group properties and reproducibility (CPU)."""
import numpy as np

from leonardym_b200 import synth


def test_su3_links_special_unitary_and_seeded():
    dims = (2, 2, 2, 4)
    a = synth.su3_links(dims, 0.25, 5)
    b = synth.su3_links(dims, 0.25, 5)
    assert np.array_equal(a, b)
    U = np.swapaxes(a, -1, -2).reshape(-1, 3, 3)
    I = np.einsum("nij,nkj->nik", U, U.conj())
    assert np.abs(I - np.eye(3)).max() < 1e-14
    assert np.abs(np.linalg.det(U) - 1).max() < 1e-14


def test_adjoint_links_orthogonal_and_bc():
    dims = (2, 2, 2, 4)
    f = synth.fermion_links(dims, "su2adj", 0.3, 3)
    R = np.swapaxes(f, -1, -2).reshape(-1, 4, 3, 3)
    dets = np.linalg.det(R)
    t = synth.lex_coords(dims)[:, 3]
    assert np.allclose(dets[t == 3, 3], -1, atol=1e-13)
    assert np.allclose(dets[t != 3, 3], 1, atol=1e-13)
    assert np.allclose(dets[:, :3], 1, atol=1e-13)
    RR = np.einsum("nmij,nmkj->nmik", R, R)
    assert np.abs(RR - np.eye(3)).max() < 1e-13


def test_sources():
    dims = (2, 2, 2, 4)
    p = synth.point_source(dims, 3, 2, 1)
    assert p[0, 2, 1] == 1 and np.count_nonzero(p) == 1
    z = synth.z2_source(dims, 3, 1)
    assert np.allclose(np.abs(z), 1.0)
