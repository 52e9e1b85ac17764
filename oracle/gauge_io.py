"""Restatement of LeonardYM's gauge-configuration formats (TEST INFRASTRUCTURE ONLY: the
checker of the library's lym_gauge_file_read / lym_gauge_file_write).  Readers follow
starters/ReadStartGaugeConfiguration.cpp:51-480, writers io/OutputSweep.cpp:32-440 for one
process; XDR values as numpy big-endian types.  Links: complex128[V, 4, N, N] with
[site, mu, j, i] = U_mu(site)(i, j), site t + Lt (z + Lz (y + Ly x)).

Pinned to the reference's own reader and writer, compiled with the XDR shim of
oracle/xdr_shim (tests/test_gauge_io.py)."""
from __future__ import annotations

import os

import numpy as np


def _lex(dims):
    x, y, z, t = np.meshgrid(*[np.arange(d) for d in dims], indexing="ij")
    return (t + dims[3] * (z + dims[2] * (y + dims[1] * x))).reshape(-1), np.stack([x, y, z, t], -1).reshape(-1, 4)


def _xfast_sites(dims):
    """Sites in the muenster files' order: t, z, y, x loops with x innermost."""
    t, z, y, x = np.meshgrid(*[np.arange(dims[k]) for k in (3, 2, 1, 0)], indexing="ij")
    return (t + dims[3] * (z + dims[2] * (y + dims[1] * x))).reshape(-1)


def write_leonard(dims, links, directory, name, number, plaquette):
    nc = links.shape[-1]
    sites, coords = _lex(dims)
    U = np.swapaxes(links, -1, -2)[sites]  # [k, mu, i, j] row-major per link
    rec = np.empty(len(sites), dtype=[("c", ">i4", 4), ("u", ">f8", (4, nc, nc, 2))])
    rec["c"] = coords
    rec["u"] = np.stack([U.real, U.imag], -1)
    base = os.path.join(directory, f"{name}_{number}")
    rec.tofile(base + "_0.txt")
    with open(base + ".descriptor.txt", "w") as f:
        f.write(f"{dims[0]} {dims[1]} {dims[2]} {dims[3]}\n1 1 1 1\n1\n{len(sites)}\n{plaquette:.13g}\n")


def read_leonard(dims, nc, directory, name, number):
    base = os.path.join(directory, f"{name}_{number}")
    tok = open(base + ".descriptor.txt").read().split()
    g, nproc, localsize, plaq = [int(v) for v in tok[:4]], int(tok[8]), int(tok[9]), float(tok[10])
    assert g == list(dims)
    links = np.zeros((int(np.prod(dims)), 4, nc, nc), np.complex128)
    dt = np.dtype([("c", ">i4", 4), ("u", ">f8", (4, nc, nc, 2))])
    for p in range(nproc):
        rec = np.fromfile(f"{base}_{p}.txt", dtype=dt, count=localsize)
        x, y, z, t = rec["c"].T
        site = t + dims[3] * (z + dims[2] * (y + dims[1] * x))
        U = rec["u"][..., 0] + 1j * rec["u"][..., 1]  # [k, mu, i, j]
        links[site] = np.swapaxes(U, -1, -2)
    return links, plaq


def write_muenster_su2(dims, links, directory, name, number, plaquette, beta, kappa):
    sites = _xfast_sites(dims)
    U = links[sites]  # [k, mu, j, i]
    a = np.conj(U[:, :, 0, 0])  # U^+(0,0)
    b = np.conj(U[:, :, 0, 1])  # U^+(0,1) = conj U(1,0)
    body = np.stack([a.real, a.imag, b.real, b.imag], -1).astype(">f4")
    tail_f = np.array([plaquette, 0, 0, beta, kappa, 0, 0, 0], ">f4")
    tail_i = np.array([number, 0, 0, 0, 0, 0, *dims, 0], ">i4")
    with open(os.path.join(directory, f"0:{number}:{name}"), "wb") as f:
        f.write(body.tobytes() + tail_f.tobytes() + tail_i.tobytes())


def read_muenster_su2(dims, directory, name, number):
    raw = open(os.path.join(directory, f"0:{number}:{name}"), "rb").read()
    V = int(np.prod(dims))
    body = np.frombuffer(raw, ">f4", count=16 * V).astype(np.float64).reshape(V, 4, 2, 2)
    c = body[..., 0] + 1j * body[..., 1]  # [k, mu, ii]
    links = np.zeros((V, 4, 2, 2), np.complex128)
    sites = _xfast_sites(dims)
    m = np.zeros((V, 4, 2, 2), np.complex128)  # [k, mu, i, j]
    m[:, :, 0, 0] = np.conj(c[:, :, 0])
    m[:, :, 1, 1] = c[:, :, 0]
    m[:, :, 0, 1] = -c[:, :, 1]
    m[:, :, 1, 0] = np.conj(c[:, :, 1])
    links[sites] = np.swapaxes(m, -1, -2)
    plaq = float(np.frombuffer(raw, ">f4", count=1, offset=64 * V)[0])
    return links, plaq


def write_muenster_su3(dims, links, directory, name, number, plaquette, beta):
    sites = _xfast_sites(dims)
    U = np.swapaxes(links[sites], -1, -2)[:, :, :, :2]  # [k, mu, ii, jj < 2]
    body = np.stack([U.real, -U.imag], -1).astype(">f4")
    tail = np.array(dims, ">i4").tobytes() + np.array([np.float32(beta), -1.0 / 12.0, plaquette], ">f8").tobytes()
    with open(os.path.join(directory, f"{name}.config-{number}"), "wb") as f:
        f.write(body.tobytes() + tail)


def read_muenster_su3(dims, directory, name, number):
    raw = open(os.path.join(directory, f"{name}.config-{number}"), "rb").read()
    V = int(np.prod(dims))
    body = np.frombuffer(raw, ">f4", count=48 * V).astype(np.float64).reshape(V, 4, 3, 2, 2)
    m = np.zeros((V, 4, 3, 3), np.complex128)
    m[..., :2] = body[..., 0] + 1j * -body[..., 1]
    col0 = m[..., :, 0] / np.sqrt(np.sum(np.abs(m[..., :, 0]) ** 2, -1))[..., None]
    m[..., :, 0] = col0
    s = np.sum(m[..., :, 1] * np.conj(m[..., :, 0]), -1)
    m[..., :, 1] -= s[..., None] * m[..., :, 0]
    m[..., :, 1] /= np.sqrt(np.sum(np.abs(m[..., :, 1]) ** 2, -1))[..., None]
    c = np.conj(m)
    m[..., 0, 2] = c[..., 1, 0] * c[..., 2, 1] - c[..., 2, 0] * c[..., 1, 1]
    m[..., 1, 2] = c[..., 2, 0] * c[..., 0, 1] - c[..., 0, 0] * c[..., 2, 1]
    m[..., 2, 2] = c[..., 0, 0] * c[..., 1, 1] - c[..., 1, 0] * c[..., 0, 1]
    links = np.zeros_like(m)
    links[_xfast_sites(dims)] = np.swapaxes(m, -1, -2)
    plaq = float(np.frombuffer(raw, ">f8", count=1, offset=192 * V + 16 + 16)[0])
    return links, plaq
