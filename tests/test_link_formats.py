"""The 8-real SU(3) link parametrisation the FP32 stencils can read (GaugeF8 in
lym_common.cuh), restated in numpy on the seeded links of the test lattices: the words
(a2, a3), (b1, arg a1, arg c1) of V = s U in SU(3) rebuild V from unitarity, in FP64
to rounding and in FP32 within a bound that grows as |a1| nears 1 (N = 1 - |a1|^2)."""
import numpy as np

from leonardym_b200 import synth


def words(U):
    """The 8 reals and the sign of each link U (column-major [..., j, i] -> row-major V)."""
    M = np.swapaxes(U, -1, -2)  # M[..., i, j] = U(i, j)
    det = np.linalg.det(M)
    s = np.where(det.real < 0, -1.0, 1.0)
    V = M * s[..., None, None]
    a2, a3, b1 = V[..., 0, 1], V[..., 0, 2], V[..., 1, 0]
    return a2, a3, b1, np.angle(V[..., 0, 0]), np.angle(V[..., 2, 0]), s, V


def rebuild(a2, a3, b1, ta, tc, dtype):
    c = np.complex128 if dtype == np.float64 else np.complex64
    a2, a3, b1 = a2.astype(c), a3.astype(c), b1.astype(c)
    ta, tc = ta.astype(dtype), tc.astype(dtype)
    N = (np.abs(a2) ** 2 + np.abs(a3) ** 2).astype(dtype)
    ra = np.sqrt(np.maximum(1 - N, 0)).astype(dtype)
    rc = np.sqrt(np.maximum(N - np.abs(b1) ** 2, 0)).astype(dtype)
    a1 = ra * np.exp(1j * ta).astype(c)
    c1 = rc * np.exp(1j * tc).astype(c)
    t2, t3 = np.conj(a1) * a2, np.conj(a1) * a3
    V = np.empty(a2.shape + (3, 3), c)
    V[..., 0, 0], V[..., 0, 1], V[..., 0, 2] = a1, a2, a3
    V[..., 1, 0], V[..., 2, 0] = b1, c1
    V[..., 1, 1] = -(np.conj(c1 * a3) + t2 * b1) / N
    V[..., 1, 2] = (np.conj(c1 * a2) - t3 * b1) / N
    V[..., 2, 1] = (np.conj(b1 * a3) - t2 * c1) / N
    V[..., 2, 2] = -(np.conj(b1 * a2) + t3 * c1) / N
    return V, N


def test_eight_real_links_rebuild_the_link():
    U = synth.fermion_links((4, 4, 4, 8), "su3", 0.3, 1234)
    a2, a3, b1, ta, tc, s, V = words(U)
    R64, N = rebuild(a2, a3, b1, ta, tc, np.float64)
    assert np.max(np.abs(R64 - V)) < 1e-12
    R32, N = rebuild(a2, a3, b1, ta, tc, np.float32)
    err = np.max(np.abs(R32 - V), axis=(-1, -2))
    # FP32 rounding, amplified by 1 / N where |a1| is close to 1
    assert np.all(err < 2e-6 / np.minimum(N, 1.0) + 1e-6)
    assert np.any(s < 0)  # the antiperiodic links go through the sign table
