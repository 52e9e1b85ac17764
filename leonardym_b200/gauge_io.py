"""Gauge-configuration files of LeonardYM (io/OutputSweep.cpp, starters/ReadStartGaugeConfiguration.cpp)
through the C ABI: read_configuration / write_configuration on host arrays (no GPU needed),
and Lattice-resident loading via lym_gauge_read."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from ._lib import LymError, lib

FORMATS = {"leonard_format": 0, "muenster_format": 1}


def _dir(directory):
    d = str(directory)
    return (d if d.endswith(os.sep) else d + os.sep).encode()


def read_configuration(format_name, dims, nc, directory, name, number):
    """Fundamental links complex128[V, 4, nc, nc] ([site, mu, j, i] = U(i, j)) and the
    plaquette stored in the file."""
    V = int(np.prod(dims))
    links = np.zeros((V, 4, nc, nc), np.complex128)
    plaq = C.c_double(0.0)
    d = (C.c_int * 4)(*[int(x) for x in dims])
    rc = lib().lym_gauge_file_read(FORMATS[format_name], d, int(nc), _dir(directory), str(name).encode(), int(number),
                                   links.ctypes.data, C.byref(plaq))
    if rc != 0:
        raise LymError(rc, f"reading {format_name} configuration {name} {number} from {directory} failed")
    return links, plaq.value


def write_configuration(format_name, links, dims, directory, name, number, plaquette=0.0, beta=0.0, kappa=0.0):
    links = np.ascontiguousarray(links, np.complex128)
    nc = links.shape[-1]
    d = (C.c_int * 4)(*[int(x) for x in dims])
    rc = lib().lym_gauge_file_write(FORMATS[format_name], d, nc, links.ctypes.data, _dir(directory),
                                    str(name).encode(), int(number), float(plaquette), float(beta), float(kappa))
    if rc != 0:
        raise LymError(rc, f"writing {format_name} configuration {name} {number} to {directory} failed")


from .dirac import BOUNDARY  # noqa: E402


def load_configuration(lattice, format_name, directory, name, number, boundary="fermion_antiperiodic",
                       gauge_id=None):
    """Read a configuration of the lattice's extents and make its fermion links resident
    (ReadStartGaugeConfiguration then Environment::synchronize); returns (gauge id, plaquette)."""
    gid = lattice._next_gauge if gauge_id is None else int(gauge_id)
    lattice._next_gauge = max(lattice._next_gauge, gid + 1)
    plaq = C.c_double(0.0)
    rc = lib().lym_gauge_read(lattice.handle, gid, FORMATS[format_name], _dir(directory), str(name).encode(),
                              int(number), BOUNDARY[boundary], C.byref(plaq))
    if rc != 0:
        raise LymError(rc, lib().lym_last_error(lattice.handle).decode())
    return gid, plaq.value
