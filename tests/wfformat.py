"""Independent numpy reader/writer of the reference's wavefunction file (test infrastructure).

The layout follows write_wf_simple (src/io_write_wf_simple_module.f90:187-276) and
read_wf_simple (src/io_read_wf_simple_module.f90:80-230): Fortran sequential unformatted records
(4-byte little-endian length before and after each payload), IO_ctrl = 0, one process.
"""
import struct

import numpy as np


def _rec(f, payload: bytes):
    f.write(struct.pack("<i", len(payload)))
    f.write(payload)
    f.write(struct.pack("<i", len(payload)))


def write(path, bands, ng, oc=1, cplx=False, ll=None, occ=None, newfmt=True, mmbz=None):
    """bands[s][k] = (nb, ML) array in file point order; ll = (ML, 3) 0-based grid coordinates
    of the file's points (default: x fastest)."""
    ms, mk = len(bands), len(bands[0])
    mb = max(b.shape[0] for row in bands for b in row)
    n1, n2, n3 = ng
    ml = n1 * n2 * n3
    if ll is None:
        i3, i2, i1 = np.meshgrid(np.arange(n3), np.arange(n2), np.arange(n1), indexing="ij")
        ll = np.stack([i1.ravel(), i2.ravel(), i3.ravel()], axis=1)
    sp = oc in (4, 5)
    with open(path, "wb") as f:
        if newfmt:
            _rec(f, struct.pack("<i", -1))
        _rec(f, struct.pack("<4i", ml, n1, n2, n3))
        _rec(f, struct.pack("<3i", mb, 1, mb))
        if newfmt:
            _rec(f, struct.pack("<3i", mk, ms, mmbz or mk))
            _rec(f, struct.pack("<3i", 0, oc, 0 if cplx else 1))
        _rec(f, np.ascontiguousarray(ll, dtype="<i4").tobytes())
        o = np.zeros((mb, mk, ms)) if occ is None else occ
        _rec(f, np.asfortranarray(o, dtype="<f8").tobytes(order="F"))
        if newfmt:
            _rec(f, np.zeros(18 + 3 * mk, dtype="<f8").tobytes())
            _rec(f, np.ones(8, dtype="<i4").tobytes())
            for n in (ml, mb, mk, ms):
                _rec(f, struct.pack("<2i", 0, n))
        for s in range(ms):
            for k in range(mk):
                b = bands[s][k]
                for n in range(mb):
                    v = b[n] if n < b.shape[0] else np.zeros(ml, dtype=b.dtype)
                    if cplx:
                        v = v.astype(np.complex64 if sp else np.complex128)
                    else:
                        v = v.astype(np.float32 if sp else np.float64)
                    _rec(f, v.tobytes())


def read(path, cplx_old=False):
    """Returns dict(header..., ll=(ML,3), occ, bands[s][k] = (MB2-MB1+1, ML) in file point order).
    The old layout does not record the value type: cplx_old says whether its records are complex."""
    with open(path, "rb") as f:
        data = f.read()
    pos = 0
    recs = []
    while pos < len(data):
        (m,) = struct.unpack_from("<i", data, pos)
        recs.append(data[pos + 4:pos + 4 + m])
        (m2,) = struct.unpack_from("<i", data, pos + 4 + m)
        assert m2 == m
        pos += 8 + m
    i = 0
    newfmt = struct.unpack("<i", recs[0][:4])[0] < 0
    if newfmt:
        i = 1
    ml, n1, n2, n3 = struct.unpack("<4i", recs[i]); i += 1
    mb, mb1, mb2 = struct.unpack("<3i", recs[i]); i += 1
    mk, ms, mmbz, ioc, oc, tw = 1, 1, 1, 0, 1, 0 if cplx_old else 1
    if newfmt:
        mk, ms, mmbz = struct.unpack("<3i", recs[i]); i += 1
        ioc, oc, tw = struct.unpack("<3i", recs[i]); i += 1
    ll = np.frombuffer(recs[i], dtype="<i4").reshape(ml, 3); i += 1
    occ = np.frombuffer(recs[i], dtype="<f8").reshape((mb, mk, ms), order="F"); i += 1
    if newfmt:
        i += 6
    cplx = tw in (0, 2)
    sp = tw in (2, 3) or oc in (4, 5)
    dt = (np.complex64 if sp else np.complex128) if cplx else (np.float32 if sp else np.float64)
    bands = [[None] * mk for _ in range(ms)]
    for s in range(ms):
        for k in range(mk):
            rows = []
            for n in range(mb1, mb2 + 1):
                rows.append(np.frombuffer(recs[i], dtype=dt)); i += 1
            bands[s][k] = np.array(rows)
    return dict(ml=ml, grid=(n1, n2, n3), mb=mb, mk=mk, ms=ms, oc=oc, type_wf=tw, ll=ll, occ=occ, bands=bands,
                newfmt=newfmt)
