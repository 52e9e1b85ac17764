"""Gauge-configuration files (leonard_format, muenster_format) through the library's host
readers and writers (no GPU), against the oracle's restatement of the reference's reader
and writer; and a configuration loaded from a file on the GPU."""
import numpy as np
import pytest

import leonardym_b200 as L
from leonardym_b200 import gauge_io, synth
from oracle import gauge_io as OG

DIMS = (4, 2, 2, 6)


def fund(nc, seed=5):
    return synth.su3_links(DIMS, 0.3, seed) if nc == 3 else synth.su2_links(DIMS, 0.3, seed)


@pytest.mark.parametrize("nc", [2, 3])
def test_leonard_format(tmp_path, nc):
    U = fund(nc)
    gauge_io.write_configuration("leonard_format", U, DIMS, tmp_path, "cfg", 7, plaquette=0.5123456789012)
    V, p = OG.read_leonard(DIMS, nc, str(tmp_path), "cfg", 7)
    assert np.array_equal(V, U) and abs(p - 0.5123456789012) < 1e-13
    OG.write_leonard(DIMS, U, str(tmp_path), "ref", 3, 0.25)
    W, p = gauge_io.read_configuration("leonard_format", DIMS, nc, tmp_path, "ref", 3)
    assert np.array_equal(W, U) and p == 0.25


def test_muenster_su2(tmp_path):
    U = fund(2)
    gauge_io.write_configuration("muenster_format", U, DIMS, tmp_path, "run", 4, plaquette=0.61, beta=2.25,
                                 kappa=0.18)
    A, pa = gauge_io.read_configuration("muenster_format", DIMS, 2, tmp_path, "run", 4)
    B, pb = OG.read_muenster_su2(DIMS, str(tmp_path), "run", 4)
    assert np.array_equal(A, B) and pa == pb == np.float32(0.61)
    assert np.max(np.abs(A - U)) < 1e-6  # float storage
    OG.write_muenster_su2(DIMS, U, str(tmp_path), "ref", 1, 0.6, 2.25, 0.18)
    C_, _ = gauge_io.read_configuration("muenster_format", DIMS, 2, tmp_path, "ref", 1)
    assert np.array_equal(C_, OG.read_muenster_su2(DIMS, str(tmp_path), "ref", 1)[0])


def test_muenster_su3(tmp_path):
    U = fund(3)
    gauge_io.write_configuration("muenster_format", U, DIMS, tmp_path, "run", 2, plaquette=0.58, beta=5.6)
    A, pa = gauge_io.read_configuration("muenster_format", DIMS, 3, tmp_path, "run", 2)
    B, pb = OG.read_muenster_su3(DIMS, str(tmp_path), "run", 2)
    assert np.max(np.abs(A - B)) < 1e-14 and pa == pb == 0.58
    assert np.max(np.abs(A - U)) < 2e-6
    # re-orthonormalised: unitary to rounding, det 1
    m = np.swapaxes(A, -1, -2).reshape(-1, 3, 3)
    assert np.max(np.abs(m @ np.conj(np.swapaxes(m, -1, -2)) - np.eye(3))) < 1e-14
    assert np.max(np.abs(np.linalg.det(m) - 1)) < 1e-14


def test_errors(tmp_path):
    with pytest.raises(L.LymError) as e:
        gauge_io.read_configuration("leonard_format", DIMS, 3, tmp_path, "missing", 1)
    assert e.value.code == -6
    gauge_io.write_configuration("leonard_format", fund(3), DIMS, tmp_path, "cfg", 1)
    with pytest.raises(L.LymError) as e:
        gauge_io.read_configuration("leonard_format", (4, 2, 2, 8), 3, tmp_path, "cfg", 1)
    assert e.value.code == -1


@pytest.mark.gpu
@pytest.mark.parametrize("rep,nc", [("su3", 3), ("su2adj", 2)])
def test_load_configuration_on_gpu(tmp_path, rep, nc):
    U = fund(nc)
    gauge_io.write_configuration("leonard_format", U, DIMS, tmp_path, "cfg", 1)
    lat = L.Lattice(DIMS, rep)
    try:
        gid, _ = gauge_io.load_configuration(lat, "leonard_format", tmp_path, "cfg", 1)
        gid2 = lat.upload_fundamental(U)
        x = synth.gaussian_spinor(DIMS, 3, 1)
        a = L.ImprovedDiracWilsonOperator(lat, 0.13, 1.0, gamma5=False)
        a.setLattice(gid)
        b = L.ImprovedDiracWilsonOperator(lat, 0.13, 1.0, gamma5=False)
        b.setLattice(gid2)
        assert np.array_equal(a.multiply(x), b.multiply(x))
    finally:
        lat.close()


# ---- pinned to the reference's own reader and writer (compiled with an XDR shim) ----------
def _needs_reference():
    from oracle import ref as R
    if not (R.available("su3") and R.available("su2adj")):
        pytest.skip("compiled reference not built")
    return R


@pytest.mark.parametrize("nc,fmt", [(3, "leonard_format"), (2, "leonard_format"), (2, "muenster_format"),
                                    (3, "muenster_format")])
def test_files_of_the_reference_load_here_and_back(tmp_path, nc, fmt):
    """A configuration written by the reference's OutputSweep reads back here (the library's
    host reader and the oracle restatement) as the reference's own reader reads it, and one
    written here reads in the reference's ReadStartGaugeConfiguration."""
    R = _needs_reference()
    rep = "su3" if nc == 3 else "su2adj"
    U = fund(nc)
    beta, kappa = (5.6, 0.13) if nc == 3 else (2.25, 0.18)
    R.gauge_write(rep, DIMS, fmt, tmp_path, "refcfg", 5, U, beta, kappa)
    ok, Ur = R.gauge_read(rep, DIMS, fmt, tmp_path, "refcfg", 5, beta, kappa)
    assert ok
    A, _ = gauge_io.read_configuration(fmt, DIMS, nc, tmp_path, "refcfg", 5)
    if fmt == "leonard_format":
        assert np.array_equal(Ur, U) and np.array_equal(A, U)
        B, _ = OG.read_leonard(DIMS, nc, str(tmp_path), "refcfg", 5)
    elif nc == 2:
        assert np.array_equal(A, Ur) and np.max(np.abs(A - U)) < 1e-6
        B, _ = OG.read_muenster_su2(DIMS, str(tmp_path), "refcfg", 5)
    else:  # SU(3): two columns as floats, the third rebuilt and re-orthonormalised on reading
        assert np.max(np.abs(A - Ur)) < 1e-14 and np.max(np.abs(A - U)) < 2e-6
        B, _ = OG.read_muenster_su3(DIMS, str(tmp_path), "refcfg", 5)
    assert np.max(np.abs(B - A)) < 1e-14
    # and the other way: written by the library, read by the reference
    gauge_io.write_configuration(fmt, U, DIMS, tmp_path, "ourcfg", 6, plaquette=0.5, beta=beta, kappa=kappa)
    ok, Ur2 = R.gauge_read(rep, DIMS, fmt, tmp_path, "ourcfg", 6, beta, kappa)
    assert ok
    A2, _ = gauge_io.read_configuration(fmt, DIMS, nc, tmp_path, "ourcfg", 6)
    assert np.max(np.abs(Ur2 - A2)) < (0 if fmt == "leonard_format" or nc == 2 else 1e-14) + 1e-300


@pytest.mark.gpu
@pytest.mark.parametrize("rep,nc,fmt", [("su3", 3, "leonard_format"), ("su3", 3, "muenster_format"),
                                        ("su2adj", 2, "muenster_format")])
def test_reference_file_on_gpu(tmp_path, rep, nc, fmt):
    """A file the reference's OutputSweep wrote, loaded into a resident gauge id on the GPU,
    gives the same operator as the links the reference's reader returns for it."""
    R = _needs_reference()
    U = fund(nc)
    beta, kappa = (5.6, 0.13) if nc == 3 else (2.25, 0.18)
    R.gauge_write(rep, DIMS, fmt, tmp_path, "refcfg", 2, U, beta, kappa)
    ok, Ur = R.gauge_read(rep, DIMS, fmt, tmp_path, "refcfg", 2, beta, kappa)
    assert ok
    lat = L.Lattice(DIMS, rep)
    try:
        gid, _ = gauge_io.load_configuration(lat, fmt, tmp_path, "refcfg", 2)
        gid2 = lat.upload_fundamental(Ur)
        x = synth.gaussian_spinor(DIMS, 3, 3)
        a = L.ImprovedDiracWilsonOperator(lat, 0.13, 1.0, gamma5=False)
        a.setLattice(gid)
        b = L.ImprovedDiracWilsonOperator(lat, 0.13, 1.0, gamma5=False)
        b.setLattice(gid2)
        ya, yb = a.multiply(x), b.multiply(x)
        assert np.linalg.norm(ya - yb) <= 1e-14 * np.linalg.norm(yb)
    finally:
        lat.close()
