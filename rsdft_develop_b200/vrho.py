"""The reference's density/potential restart file (vrho.dat), read and written on the host.

write_data with OC = 2, 3, 5, 12, 13 writes it at the end of an SCF (src/io_module.f90:110-230)
and read_data with IC = 2, 3, 4, 5, 12, 13 restarts from it (:300-455).  Fortran sequential
unformatted records (a 4-byte little-endian length before and after each payload), one grid
process, in this order:

  version tag (64 characters, "version3.0, comment_length=64")
  ML, ML1, ML2, ML3                                   (4 x int32)
  LL2(1:3, 1:ML): 0-based grid coordinates of the file's points, in file order (int32)
  comment "lattice aa(3,3)";  aa(3,3)                 (real8, columns a_1, a_2, a_3)
  comment "atom: ...";  Nelement, Natom;  aa_atom(3, Natom) (reduced);  ki_atom(Natom);
  zn_atom(Nelement)
  comment "Fermi energy";  efermi
  per spin s: rho(:, s), Vloc(:, s), [Vh, for s = 1 only], Vxc(:, s)  (ML x real8 each)

A file without the version tag (the older layout) starts at ML and has no lattice, atom or Fermi
records.  Grid values are mapped through LL2 onto this library's layout (x fastest), as the
reference maps them onto its own grid.
"""
from __future__ import annotations

import dataclasses
import struct

import numpy as np

VERSION = "version3.0, comment_length=64"


@dataclasses.dataclass
class Vrho:
    n: tuple                      # (ML1, ML2, ML3)
    rho: np.ndarray               # (nspin, ML), x fastest
    vloc: np.ndarray              # (nspin, ML)
    vh: np.ndarray                # (ML,)
    vxc: np.ndarray               # (nspin, ML)
    efermi: float = 0.0
    aa: np.ndarray | None = None  # (3, 3) rows a_i (bohr)
    atoms: np.ndarray | None = None   # (natom, 3) reduced
    ki_atom: np.ndarray | None = None
    zn_atom: np.ndarray | None = None
    versioned: bool = True


def _rec(f, payload: bytes) -> None:
    f.write(struct.pack("<i", len(payload)))
    f.write(payload)
    f.write(struct.pack("<i", len(payload)))


def _text(s: str) -> bytes:
    return s.ljust(64)[:64].encode("ascii")


def write_vrho(path: str, v: Vrho, ll: np.ndarray | None = None) -> None:
    """Write v in the reference's layout; ll (ML, 3) gives the file's point order as 0-based grid
    coordinates (x fastest when None)."""
    n1, n2, n3 = v.n
    ml = n1 * n2 * n3
    if ll is None:
        i3, i2, i1 = np.meshgrid(np.arange(n3), np.arange(n2), np.arange(n1), indexing="ij")
        ll = np.stack([i1.ravel(), i2.ravel(), i3.ravel()], axis=1)
    ll = np.asarray(ll, dtype=np.int64)
    lin = ll[:, 0] + n1 * (ll[:, 1] + n2 * ll[:, 2])
    ns = v.rho.shape[0]
    aa = np.zeros((3, 3)) if v.aa is None else np.asarray(v.aa, np.float64)
    atoms = np.zeros((0, 3)) if v.atoms is None else np.asarray(v.atoms, np.float64).reshape(-1, 3)
    natom = atoms.shape[0]
    ki = np.ones(natom, np.int32) if v.ki_atom is None else np.asarray(v.ki_atom, np.int32)
    zn = np.zeros(0 if natom == 0 else int(ki.max()), np.int32) if v.zn_atom is None else np.asarray(v.zn_atom, np.int32)
    with open(path, "wb") as f:
        if v.versioned:
            _rec(f, _text(VERSION))
        _rec(f, struct.pack("<4i", ml, n1, n2, n3))
        _rec(f, np.ascontiguousarray(ll, dtype="<i4").tobytes())
        if v.versioned:
            _rec(f, _text("lattice aa(3,3)"))
            _rec(f, np.ascontiguousarray(aa.T, dtype="<f8").tobytes(order="F"))
            _rec(f, _text("atom: Nelement Natom / aa_atom / ki_atom /zn_atom"))
            _rec(f, struct.pack("<2i", zn.size, natom))
            _rec(f, np.ascontiguousarray(atoms, dtype="<f8").tobytes())
            _rec(f, np.ascontiguousarray(ki, dtype="<i4").tobytes())
            _rec(f, np.ascontiguousarray(zn, dtype="<i4").tobytes())
            _rec(f, _text("Fermi energy"))
            _rec(f, struct.pack("<d", float(v.efermi)))
        for s in range(ns):
            _rec(f, np.ascontiguousarray(v.rho[s][lin], dtype="<f8").tobytes())
            _rec(f, np.ascontiguousarray(v.vloc[s][lin], dtype="<f8").tobytes())
            if s == 0:
                _rec(f, np.ascontiguousarray(v.vh[lin], dtype="<f8").tobytes())
            _rec(f, np.ascontiguousarray(v.vxc[s][lin], dtype="<f8").tobytes())


def _records(path: str) -> list:
    out = []
    with open(path, "rb") as f:
        data = f.read()
    pos = 0
    while pos < len(data):
        if pos + 4 > len(data):
            raise ValueError(f"{path}: truncated record marker at byte {pos}")
        (m,) = struct.unpack_from("<i", data, pos)
        if m < 0 or pos + 8 + m > len(data):
            raise ValueError(f"{path}: record of {m} bytes at byte {pos} runs past the end")
        (m2,) = struct.unpack_from("<i", data, pos + 4 + m)
        if m2 != m:
            raise ValueError(f"{path}: record markers {m} and {m2} differ at byte {pos}")
        out.append(data[pos + 4:pos + 4 + m])
        pos += 8 + m
    return out


def read_vrho(path: str, n: tuple, nspin: int) -> Vrho:
    """Read a vrho file for a grid n with nspin spins (the reference stops on a grid mismatch;
    this raises ValueError)."""
    recs = _records(path)
    i = 0
    versioned = recs[0][:7] == b"version"
    if versioned:
        i = 1
    ml, n1, n2, n3 = struct.unpack("<4i", recs[i][:16])
    i += 1
    if ml != n[0] * n[1] * n[2]:
        raise ValueError(f"vrho: ML = {ml} in the file, {n[0] * n[1] * n[2]} on this grid")
    if (n1, n2, n3) != tuple(n):
        raise ValueError(f"vrho: grid {(n1, n2, n3)} in the file, {tuple(n)} here")
    ll = np.frombuffer(recs[i], dtype="<i4").reshape(ml, 3).astype(np.int64)
    i += 1
    if np.any(ll < 0) or np.any(ll >= np.array([n1, n2, n3])):
        raise ValueError("vrho: grid coordinates outside the grid")
    lin = ll[:, 0] + n1 * (ll[:, 1] + n2 * ll[:, 2])
    aa = atoms = ki = zn = None
    ef = 0.0
    if versioned:
        aa = np.frombuffer(recs[i + 1], dtype="<f8").reshape(3, 3).copy()     # rows a_i
        nel, nat = struct.unpack("<2i", recs[i + 3][:8])
        atoms = np.frombuffer(recs[i + 4], dtype="<f8").reshape(nat, 3).copy()
        ki = np.frombuffer(recs[i + 5], dtype="<i4").copy()
        zn = np.frombuffer(recs[i + 6], dtype="<i4").copy()
        (ef,) = struct.unpack("<d", recs[i + 8][:8])
        i += 9
    need = i + 3 * nspin + 1
    if len(recs) < need:
        raise ValueError(f"vrho: {len(recs)} records, {need} needed for {nspin} spins")

    def grid(rec):
        a = np.frombuffer(rec, dtype="<f8")
        if a.size != ml:
            raise ValueError(f"vrho: a grid record holds {a.size} values, ML = {ml}")
        out = np.empty(ml)
        out[lin] = a
        return out

    rho = np.zeros((nspin, ml))
    vloc = np.zeros((nspin, ml))
    vxc = np.zeros((nspin, ml))
    vh = None
    for s in range(nspin):
        rho[s] = grid(recs[i])
        vloc[s] = grid(recs[i + 1])
        i += 2
        if s == 0:
            vh = grid(recs[i])
            i += 1
        vxc[s] = grid(recs[i])
        i += 1
    return Vrho(n=(n1, n2, n3), rho=rho, vloc=vloc, vh=vh, vxc=vxc, efermi=ef, aa=aa, atoms=atoms,
                ki_atom=ki, zn_atom=zn, versioned=versioned)
