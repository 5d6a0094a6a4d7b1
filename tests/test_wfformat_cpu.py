"""CPU checks of the wavefunction-file support: the numpy restatement of the reference's format
round-trips (new and old layout, FP64 and FP32, real and complex), and the library's file entries
fail cleanly before rsdft_gpu_init (no device needed)."""
import ctypes as C

import numpy as np

from rsdft_develop_b200 import api
from tests import wfformat


def test_format_round_trip(tmp_path):
    rng = np.random.default_rng(3)
    ng = (4, 3, 2)
    ml = 24
    for cplx in (False, True):
        for oc, newfmt in ((1, True), (4, True), (1, False)):
            b = rng.standard_normal((2, 3, ml))
            if cplx:
                b = b + 1j * rng.standard_normal((2, 3, ml))
            bands = [[b[0], b[1][:2]]] if newfmt else [[b[0]]]
            path = str(tmp_path / f"w{int(cplx)}{oc}{int(newfmt)}")
            wfformat.write(path, bands, ng, oc=oc, cplx=cplx, newfmt=newfmt)
            d = wfformat.read(path, cplx_old=cplx)
            assert d["ml"] == ml and d["grid"] == ng and d["newfmt"] == newfmt
            tol = 1e-6 if oc == 4 else 0.0
            assert np.max(np.abs(d["bands"][0][0] - b[0])) <= tol * 10
            if newfmt:
                assert d["mb"] == 3 and d["mk"] == 2
                assert np.max(np.abs(d["bands"][0][1][:2] - b[1][:2])) <= tol * 10
                assert np.all(d["bands"][0][1][2] == 0)


def test_file_entries_before_init_fail_cleanly(tmp_path):
    lib = api.load_library()
    assert lib.rsdft_gpu_write_wf(str(tmp_path / "x").encode(), 1, None, None, None, None) == -7
    assert lib.rsdft_gpu_read_wf(str(tmp_path / "x").encode(), None) == -7
