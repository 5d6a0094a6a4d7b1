"""The vrho restart file (src/io_module.f90:110-230 write, :300-455 read) on small grids: round
trips with and without the version tag, the grid map applied on read, and the refusals the
reference turns into stops (grid mismatch) or that a damaged file needs (bad record markers)."""
import struct

import numpy as np
import pytest

from rsdft_develop_b200 import vrho


def _sample(n=(4, 3, 2), ns=2, seed=0, versioned=True):
    rng = np.random.default_rng(seed)
    ml = n[0] * n[1] * n[2]
    return vrho.Vrho(n=n, rho=rng.random((ns, ml)), vloc=rng.normal(size=(ns, ml)), vh=rng.normal(size=ml),
                     vxc=rng.normal(size=(ns, ml)), efermi=0.25, aa=np.diag([4.0, 3.0, 2.0]),
                     atoms=np.array([[0.0, 0.0, 0.1], [0.5, 0.5, 0.5]]), ki_atom=np.array([1, 1]),
                     zn_atom=np.array([8]), versioned=versioned)


@pytest.mark.parametrize("versioned", [True, False])
@pytest.mark.parametrize("ns", [1, 2])
def test_round_trip(tmp_path, versioned, ns):
    v = _sample(ns=ns, versioned=versioned)
    path = str(tmp_path / "vrho.dat1")
    vrho.write_vrho(path, v)
    w = vrho.read_vrho(path, v.n, ns)
    assert w.versioned == versioned
    for f in ("rho", "vloc", "vh", "vxc"):
        assert np.array_equal(getattr(w, f), getattr(v, f)), f
    if versioned:
        assert w.efermi == 0.25 and np.array_equal(w.aa, v.aa) and np.array_equal(w.atoms, v.atoms)
        assert w.ki_atom.tolist() == [1, 1] and w.zn_atom.tolist() == [8]
    raw = open(path, "rb").read()
    if versioned:
        assert raw[4:4 + 29] == b"version3.0, comment_length=64"


def test_grid_map_reorders_points(tmp_path):
    v = _sample()
    n = v.n
    i3, i2, i1 = np.meshgrid(np.arange(n[2]), np.arange(n[1]), np.arange(n[0]), indexing="ij")
    ll = np.stack([i1.ravel(), i2.ravel(), i3.ravel()], axis=1)[::-1]
    path = str(tmp_path / "vrho.dat1")
    vrho.write_vrho(path, v, ll)
    raw = open(path, "rb").read()
    # the file's grid map starts with the last grid point: the file order follows ll
    w = vrho.read_vrho(path, n, 2)
    assert np.array_equal(w.rho, v.rho)
    assert struct.unpack_from("<3i", raw, (4 + 64 + 4) + (4 + 16 + 4) + 4) == tuple(ll[0])


def test_refusals(tmp_path):
    v = _sample()
    path = str(tmp_path / "vrho.dat1")
    vrho.write_vrho(path, v)
    with pytest.raises(ValueError, match="ML"):
        vrho.read_vrho(path, (4, 3, 3), 2)
    with pytest.raises(ValueError, match="grid"):
        vrho.read_vrho(path, (3, 4, 2), 2)
    with pytest.raises(ValueError, match="records"):
        vrho.read_vrho(path, v.n, 3)
    raw = bytearray(open(path, "rb").read())
    bad = str(tmp_path / "bad.dat")
    open(bad, "wb").write(bytes(raw[:-3]))
    with pytest.raises(ValueError):
        vrho.read_vrho(bad, v.n, 2)
