"""Restatement of LeonardYM's fermion force (TEST INFRASTRUCTURE ONLY: the checker of the
library's lym_fermion_force).  FermionForce::derivative (hmc_forces/FermionForce.cpp:11-20)
with DiracWilsonFermionForce::derivative (hmc_forces/DiracWilsonFermionForce.cpp:10-53) and
ImprovedFermionForce::derivative (hmc_forces/ImprovedFermionForce.cpp:11-268), vectorised over
sites.  Layouts as the reference's raw data: fermion links [V, 4, N, N] column-major
([site, mu, j, i] = U(i, j); real for the adjoint), spinors [V, 4, 3], force [V, 4, 3, 3]
complex column-major."""
from __future__ import annotations

import numpy as np

_S = [np.array([[0, 1], [1, 0]], complex), np.array([[0, -1j], [1j, 0]]), np.array([[1, 0], [0, -1]], complex)]
_Z = np.zeros((2, 2), complex)
GAMMA = [np.block([[_Z, -1j * s], [1j * s, _Z]]) for s in _S] + [np.block([[_Z, np.eye(2)], [np.eye(2), _Z]])]
GAMMA5 = np.diag([1.0, 1.0, -1.0, -1.0]).astype(complex)
G5_ID_MINUS = [GAMMA5 @ (np.eye(4) - g) for g in GAMMA]  # Gamma::g5idmg
G5_ID_PLUS = [GAMMA5 @ (np.eye(4) + g) for g in GAMMA]  # Gamma::g5idpg
G5_SIGMA = [[GAMMA5 @ (0.5j * (GAMMA[m] @ GAMMA[n] - GAMMA[n] @ GAMMA[m])) for n in range(4)] for m in range(4)]


def _geometry(dims):
    V = int(np.prod(dims))
    s = np.arange(V)
    c = np.empty((V, 4), int)
    c[:, 3] = s % dims[3]
    r = s // dims[3]
    c[:, 2] = r % dims[2]
    r //= dims[2]
    c[:, 1] = r % dims[1]
    c[:, 0] = r // dims[1]
    return c


def _shift(dims, c, *moves):
    c = c.copy()
    for mu, d in moves:
        c[:, mu] = (c[:, mu] + d) % dims[mu]
    return c[:, 3] + dims[3] * (c[:, 2] + dims[2] * (c[:, 1] + dims[1] * c[:, 0]))


def _tensor(x, y):
    """FermionForce::tensor per site: result(i, j) = y[i] conj(x[j])."""
    return np.einsum("si,sj->sij", y, x.conj())


def _mv(M, v):
    return np.einsum("sij,sj->si", M, v)


def _dag(M):
    return np.conj(np.swapaxes(M, -1, -2))


def derivative(dims, links, X, Y, kappa, csw, clover):
    """F_mu(x) for all x and mu: [V, 4, 3, 3] row-major."""
    U = np.swapaxes(np.asarray(links), -1, -2).astype(complex)  # [s, mu, i, j]
    c = _geometry(dims)
    s = np.arange(len(c))
    out = np.zeros((len(c), 4, 3, 3), complex)
    for mu in range(4):
        xp = _shift(dims, c, (mu, 1))
        Um = U[:, mu]
        F = np.zeros((len(c), 3, 3), complex)
        for A, B in ((X, Y), (Y, X)):
            for al in range(4):
                t = -kappa * np.einsum("b,sbd->sd", G5_ID_MINUS[mu][al], B[xp])
                F += _tensor(A[s, al], t)
                t = -kappa * np.einsum("b,sbd->sd", G5_ID_PLUS[mu][al], np.einsum("sji,sbj->sbi", Um.conj(), B))
                F -= _tensor(_mv(Um, A[xp, al]), t)
        if clover:
            Fc = np.zeros_like(F)
            ikc = 1j * kappa * csw
            for nu in range(4):
                if nu == mu:
                    continue
                xpn, xmn = _shift(dims, c, (nu, 1)), _shift(dims, c, (nu, -1))
                xpm_mn, xpm_pn = _shift(dims, c, (mu, 1), (nu, -1)), _shift(dims, c, (mu, 1), (nu, 1))
                Unu_x, Unu_xpm, Umu_xpn = U[:, nu], U[xp, nu], U[xpn, mu]
                Unu_xpm_mn, Umu_xmn, Unu_xmn = U[xpm_mn, nu], U[xmn, mu], U[xmn, nu]
                mm = lambda *Ms: Ms[0] if len(Ms) == 1 else np.einsum("sij,sjk->sik", Ms[0], mm(*Ms[1:]))
                terms = [  # (sign, L or None, R or None, projection site) as ImprovedFermionForce.cpp:225-268
                    (+1, mm(Unu_xpm, _dag(Umu_xpn), _dag(Unu_x)), None, s),
                    (-1, _dag(Um), mm(Um, _dag(Unu_xpm_mn), _dag(Umu_xmn), Unu_xmn), s),
                    (+1, mm(Unu_xpm, _dag(Umu_xpn)), Unu_x, xpn),
                    (-1, mm(_dag(Um), _dag(Unu_xmn)), mm(Um, _dag(Unu_xpm_mn), _dag(Umu_xmn)), xmn),
                    (+1, None, mm(Unu_x, Umu_xpn, _dag(Unu_xpm)), xp),
                    (-1, mm(_dag(Um), _dag(Unu_xmn), Umu_xmn, Unu_xpm_mn), Um, xp),
                    (+1, Unu_xpm, mm(Unu_x, Umu_xpn), xpm_pn),
                    (-1, mm(_dag(Um), _dag(Unu_xmn), Umu_xmn), mm(Um, _dag(Unu_xpm_mn)), xpm_mn),
                ]
                for sg, L, R, ps in terms:
                    for A, B in ((X, Y), (Y, X)):
                        for al in range(4):
                            p = ikc * np.einsum("b,sbd->sd", G5_SIGMA[mu][nu][al], B[ps])
                            lp = _mv(L, p) if L is not None else p
                            ra = _mv(R, A[ps, al]) if R is not None else A[ps, al]
                            Fc += sg * _tensor(ra, lp)
            F = Fc / 4.0 + F
        out[:, mu] = F
    return out


def fermion_force(dims, links, X, Y, kappa, csw, clover, weight, force):
    """FermionForce::derivative: force - weight * F (column-major [V, 4, 3, 3])."""
    F = derivative(dims, links, np.asarray(X), np.asarray(Y), kappa, csw, clover)
    return np.asarray(force) - weight * np.swapaxes(F, -1, -2)
