"""Wavefunction restart files in the reference's format (write_wf_simple / read_wf_simple,
src/io_write_wf_simple_module.f90, src/io_read_wf_simple_module.f90).

The library's writer is checked against an independent numpy reader of the format
(tests/wfformat.py), and its reader against files that numpy writes: the reference's own layout
with a permuted grid map LL2 (as a file from a run with several grid ranks orders its points),
the old layout without the leading -1, FP32 records (OC 4), and complex k-point bands.  Round
trips through the library are exact in FP64 and within FP32 rounding for OC 4 files.
"""
import numpy as np
import pytest

from rsdft_develop_b200 import api, synth
from tests import wfformat

pytestmark = pytest.mark.gpu


def _natural(prob):
    n1, n2, n3 = prob.n
    i3, i2, i1 = np.meshgrid(np.arange(n3), np.arange(n2), np.arange(n1), indexing="ij")
    return np.stack([i1.ravel(), i2.ravel(), i3.ravel()], axis=1)


def test_write_matches_format_and_reads_back(tmp_path):
    prob = synth.make_problem("c0")
    path = str(tmp_path / "wf.dat1")
    occ = np.linspace(2.0, 0.0, prob.nband).reshape(prob.nband, 1, 1)
    with api.BandUpdate(prob) as g:
        g.random_wf(11)
        g.gram_schmidt()
        u = g.get_wf()
        g.write_wf(path, oc=1, occ=occ)
    d = wfformat.read(path)
    assert d["newfmt"] and d["ml"] == prob.ng and d["grid"] == tuple(prob.n)
    assert d["mb"] == prob.nband and d["mk"] == 1 and d["ms"] == 1 and d["type_wf"] == 1 and d["oc"] == 1
    assert np.array_equal(d["ll"], _natural(prob))
    assert np.array_equal(d["occ"][:, 0, 0], occ[:, 0, 0])
    assert np.array_equal(d["bands"][0][0], u)
    with api.BandUpdate(prob) as h:
        occ2 = h.read_wf(path)
        assert np.array_equal(h.get_wf(), u)
        assert np.array_equal(occ2[:, 0, 0], occ[:, 0, 0])


def test_read_permuted_grid_map_old_layout_and_fp32(tmp_path):
    prob = synth.make_problem("t0")
    rng = np.random.default_rng(5)
    u = rng.standard_normal((prob.nband, prob.ng))
    ll = _natural(prob)
    perm = rng.permutation(prob.ng)
    # file point i holds grid point ll[perm[i]]
    for newfmt, oc in ((True, 1), (False, 1), (True, 4)):
        path = str(tmp_path / f"wf_{int(newfmt)}_{oc}.dat")
        wfformat.write(path, [[u[:, perm]]], prob.n, oc=oc, ll=ll[perm], newfmt=newfmt)
        with api.BandUpdate(prob) as g:
            g.read_wf(path)
            got = g.get_wf()
        if oc == 4:
            assert np.max(np.abs(got - u)) <= 1e-6 * np.max(np.abs(u))
        else:
            assert np.array_equal(got, u)


def test_complex_kpoints_and_mixed_precision_round_trip(tmp_path):
    cfg = synth.get_config("tk", nband_range=(8, 8))
    prob = synth.make_problem(cfg)
    path = str(tmp_path / "wfz.dat")
    with api.BandUpdate(prob, precision=api.PREC_MIXED) as g:
        for k in range(prob.nk):
            g.random_wf(20 + k, k=k + 1)
        us = [g.get_wf(k=k + 1) for k in range(prob.nk)]
        g.write_wf(path, oc=4)
    d = wfformat.read(path)
    assert d["type_wf"] == 0 and d["oc"] == 4 and d["mk"] == prob.nk
    for k in range(prob.nk):
        assert np.array_equal(d["bands"][0][k].astype(np.complex128), us[k])  # FP32 bands written as is
    with api.BandUpdate(prob) as h:
        h.read_wf(path)
        for k in range(prob.nk):
            assert np.array_equal(h.get_wf(k=k + 1), us[k])


def test_mismatched_grid_is_refused(tmp_path):
    prob = synth.make_problem("t0")
    path = str(tmp_path / "wf_bad.dat")
    wfformat.write(path, [[np.zeros((prob.nband, 10 * 10 * 10))]], (10, 10, 10))
    with api.BandUpdate(prob) as g:
        with pytest.raises(api.RsdftError) as e:
            g.read_wf(path)
        assert e.value.code == -1
