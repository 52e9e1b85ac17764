"""Seeded synthetic lattices: gauge links and sources.

All arrays use the reference's raw host layout (the memory of
``Lattice<T, LocalLayout>::getRawData()``, MPILattice/Lattice.h:228-234):

* site index ``t + Lt*(z + Lz*(y + Ly*x))`` (LocalLayout.h:149-163),
* gauge links ``complex128[V, 4, N, N]`` as an Eigen column-major matrix, i.e.
  numpy array ``u[site, mu, j, i] = U_mu(site)(i, j)``,
* spinors ``complex128[V, 4, dVL]`` (``GaugeVector[4]``).

Random numbers come from numpy's counter-based Philox generator, so a
(seed, shape) pair always yields the same field on any machine.
"""
from __future__ import annotations

import numpy as np

__all__ = [
    "volume", "gell_mann", "su3_links", "su2_links", "su2_to_adjoint",
    "antiperiodic_bc", "fermion_links", "gaussian_spinor", "point_source", "z2_source",
    "lex_coords", "su3_fermion_links_device", "gaussian_spinor_device",
]


def volume(dims):
    return int(dims[0]) * int(dims[1]) * int(dims[2]) * int(dims[3])


def lex_coords(dims):
    """Coordinates (x, y, z, t) of every site in the reference's index order."""
    x, y, z, t = np.meshgrid(*[np.arange(d) for d in dims], indexing="ij")
    return np.stack([x.ravel(), y.ravel(), z.ravel(), t.ravel()], axis=1)


def gell_mann():
    l = np.zeros((8, 3, 3), dtype=np.complex128)
    l[0, 0, 1] = l[0, 1, 0] = 1
    l[1, 0, 1] = -1j; l[1, 1, 0] = 1j
    l[2, 0, 0] = 1; l[2, 1, 1] = -1
    l[3, 0, 2] = l[3, 2, 0] = 1
    l[4, 0, 2] = -1j; l[4, 2, 0] = 1j
    l[5, 1, 2] = l[5, 2, 1] = 1
    l[6, 1, 2] = -1j; l[6, 2, 1] = 1j
    l[7] = np.diag([1, 1, -2]) / np.sqrt(3)
    return l


def _pauli():
    s = np.zeros((3, 2, 2), dtype=np.complex128)
    s[0] = [[0, 1], [1, 0]]
    s[1] = [[0, -1j], [1j, 0]]
    s[2] = [[1, 0], [0, -1]]
    return s


def _expi_hermitian(H, eps):
    """exp(i eps H) for a batch of Hermitian matrices via eigendecomposition."""
    w, v = np.linalg.eigh(H)
    ph = np.exp(1j * eps * w)
    return np.einsum("...ij,...j,...kj->...ik", v, ph, v.conj())


def _reunit(U):
    """Gram-Schmidt over rows then det-phase removal, as ReUnit (utils/ReUnit.cpp:15-28)."""
    U = U.copy()
    n = U.shape[-1]
    for i in range(n):
        for j in range(i):
            proj = np.sum(U[..., j, :].conj() * U[..., i, :], axis=-1)
            U[..., i, :] -= proj[..., None] * U[..., j, :]
        nv = np.sqrt(np.sum((U[..., i, :].conj() * U[..., i, :]).real, axis=-1))
        U[..., i, :] /= nv[..., None]
    d = np.linalg.det(U)
    U[..., n - 1, :] *= np.exp(-1j * np.angle(d))[..., None]
    return U


def _rng(seed, stream):
    return np.random.Generator(np.random.Philox(key=[int(seed), int(stream)]))


def _chunked_links(dims, seed, make, nc, chunk=1 << 18):
    V = volume(dims)
    out = np.empty((V, 4, nc, nc), dtype=np.complex128)
    flat = out.reshape(V * 4, nc, nc)
    n = V * 4
    for c0 in range(0, n, chunk):
        c1 = min(n, c0 + chunk)
        rng = _rng(seed, c0 // chunk)
        U = make(rng, c1 - c0)
        flat[c0:c1] = np.swapaxes(U, -1, -2)  # store column-major: [j, i] = U(i, j)
    return out


def su3_links(dims, eps, seed):
    """SU(3) links U = exp(i eps H), H = sum_a h_a lambda_a, h_a ~ N(0,1), reunitarised."""
    lam = gell_mann()

    def make(rng, n):
        h = rng.standard_normal((n, 8))
        H = np.einsum("na,aij->nij", h, lam)
        return _reunit(_expi_hermitian(H, eps))

    return _chunked_links(dims, seed, make, 3)


def su2_links(dims, eps, seed):
    """SU(2) links U = exp(i eps sigma.n), n ~ N(0,1)^3, reunitarised."""
    sig = _pauli()

    def make(rng, n):
        v = rng.standard_normal((n, 3))
        H = np.einsum("na,aij->nij", v, sig)
        return _reunit(_expi_hermitian(H, eps))

    return _chunked_links(dims, seed, make, 2)


def su2_to_adjoint(links2):
    """Adjoint links adj(a,b) = 2 Re tr(T_a U T_b U^+), T = sigma/2
    (utils/ConvertLattice.h:24-34,100-105).  Input complex [.., 2, 2] column-major,
    output float64 [.., 3, 3] column-major (out[..., b, a] = adj(a, b))."""
    U = np.swapaxes(links2, -1, -2)  # row-major U(i,j)
    T = _pauli() / 2
    Ud = np.conj(np.swapaxes(U, -1, -2))
    adj = np.einsum("aij,...jk,bkl,...li->...ab", T, U, T, Ud).real * 2.0
    return np.ascontiguousarray(np.swapaxes(adj, -1, -2))


def antiperiodic_bc(links, dims):
    """switchAntiperiodicBc (LatticeBoundaryConditions.h:8-14): negate U_t at t = Lt-1."""
    out = links.copy()
    Lt = int(dims[3])
    out.reshape(-1, Lt, *links.shape[1:])[:, Lt - 1, 3] *= -1
    return out


def fermion_links(dims, rep, eps, seed, bc="fermion_antiperiodic"):
    """Fermion link field as Environment::synchronize builds it (Environment.cpp:21-79):
    fundamental links (rep 'su3') or the adjoint of SU(2) links (rep 'su2adj'),
    then the boundary condition folded into the links."""
    if rep == "su3":
        L = su3_links(dims, eps, seed)
    elif rep == "su2adj":
        L = su2_to_adjoint(su2_links(dims, eps, seed))
    else:
        raise ValueError(f"unknown representation {rep!r}")
    if bc == "fermion_antiperiodic":
        L = antiperiodic_bc(L, dims)
    elif bc != "fermion_periodic":
        raise ValueError(f"unsupported boundary condition {bc!r}")
    return np.ascontiguousarray(L)


def gaussian_spinor(dims, nc, seed, stream=1 << 20):
    """Complex-normal spinor, E|z|^2 = 1 per component."""
    V = volume(dims)
    rng = _rng(seed, stream)
    a = rng.standard_normal((V, 4, nc, 2)) * np.sqrt(0.5)
    return np.ascontiguousarray(a[..., 0] + 1j * a[..., 1])


def point_source(dims, nc, alpha, c):
    """StochasticEstimator::generateSource (fermion_measurements/StochasticEstimator.cpp:100-112)."""
    v = np.zeros((volume(dims), 4, nc), dtype=np.complex128)
    v[0, alpha, c] = 1.0
    return v


def z2_source(dims, nc, seed, stream=1 << 21):
    """Z2 x Z2 noise with entries (+-1 +-i)/sqrt(2)."""
    V = volume(dims)
    rng = _rng(seed, stream)
    b = rng.integers(0, 2, size=(V, 4, nc, 2)) * 2 - 1
    return np.ascontiguousarray((b[..., 0] + 1j * b[..., 1]) / np.sqrt(2.0))


def _reunit_torch(U):
    """_reunit on a batch of torch matrices (rows Gram-Schmidt, then the det phase)."""
    import torch

    U = U.clone()
    n = U.shape[-1]
    for i in range(n):
        for j in range(i):
            proj = (U[:, j, :].conj() * U[:, i, :]).sum(-1)
            U[:, i, :] -= proj[:, None] * U[:, j, :]
        nv = (U[:, i, :].abs() ** 2).sum(-1).sqrt()
        U[:, i, :] /= nv[:, None]
    a = U
    d = (a[:, 0, 0] * (a[:, 1, 1] * a[:, 2, 2] - a[:, 1, 2] * a[:, 2, 1])
         - a[:, 0, 1] * (a[:, 1, 0] * a[:, 2, 2] - a[:, 1, 2] * a[:, 2, 0])
         + a[:, 0, 2] * (a[:, 1, 0] * a[:, 2, 1] - a[:, 1, 1] * a[:, 2, 0]))
    U[:, n - 1, :] *= torch.exp(-1j * torch.angle(d))[:, None]
    return U


def su3_fermion_links_device(dims, eps, seed, device, chunk=1 << 22):
    """SU(3) fermion links on a CUDA device: U = exp(i eps H), H = sum_a h_a lambda_a with
    h_a ~ N(0,1) from torch's seeded device generator, reunitarised, antiperiodic in time
    (U_t negated at t = Lt-1).  The distribution of su3_links + antiperiodic_bc, for lattices
    whose host generation would take minutes; not the same numbers.  Returns a torch
    complex128 tensor [V, 4, 3, 3] in the column-major link layout."""
    import torch

    V = volume(dims)
    n = 4 * V
    out = torch.empty((V, 4, 3, 3), dtype=torch.complex128, device=device)
    flat = out.view(n, 3, 3)
    lam = torch.from_numpy(gell_mann()).to(device=device, dtype=torch.complex128)
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    for c0 in range(0, n, chunk):
        c1 = min(n, c0 + chunk)
        h = torch.randn((c1 - c0, 8), generator=g, device=device, dtype=torch.float64)
        H = torch.einsum("na,aij->nij", h.to(torch.complex128), lam)
        U = _reunit_torch(torch.linalg.matrix_exp(1j * float(eps) * H))
        flat[c0:c1] = U.transpose(-1, -2)
        del h, H, U
    Lt = int(dims[3])
    out.view(-1, Lt, 4, 3, 3)[:, Lt - 1, 3] *= -1
    torch.cuda.synchronize(device)  # written before the library's stream reads it
    return out


def gaussian_spinor_device(dims, nc, seed, device):
    """Complex-normal spinor (E|z|^2 = 1 per component) from torch's seeded device generator,
    as a torch complex128 tensor [V, 4, nc] (the device is synchronised before it returns: the
    library's stream does not wait for torch's)."""
    import torch

    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    a = torch.randn((volume(dims), 4, nc, 2), generator=g, device=device, dtype=torch.float64) * np.sqrt(0.5)
    out = torch.view_as_complex(a).contiguous()
    torch.cuda.synchronize(device)  # written before the library's stream reads it
    return out
