"""Shared helpers of the test suite (seeded lattices, error norms)."""
import numpy as np

from leonardym_b200 import synth

CONFIGS = {
    # name: (dims, rep, eps, kappa, csw)
    "su3": ((4, 4, 4, 8), "su3", 0.3, 0.13, 1.0),
    "su2adj": ((4, 4, 4, 8), "su2adj", 0.3, 0.18, 1.5),
}


def links_for(name, seed=1234):
    dims, rep, eps, kappa, csw = CONFIGS[name]
    return synth.fermion_links(dims, rep, eps, seed)


def rel(a, b):
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / (nb if nb > 0 else 1.0))
