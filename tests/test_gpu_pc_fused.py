"""The fused FP32 preconditioner forms inside CG against the multi-pass s-step form.

precond_hprsdft (src/conjugate_gradient/cgpc_hprsdft_module.f90:133-270) followed by the CG
dot <Pg|g> and the direction update p = Pg + beta p (src/conjugate_gradient/cg_module.f90:
254-283).  Form 2 evaluates the preconditioner's s-step chain on the fly in two
z-streamed passes and takes <Pg|g> from the moments; form 1 runs the same s-step arithmetic in
3 mloop + 3 separate passes (itself held to the FP64 recurrence of the oracle by
test_gpu_mixed.py); form 3 runs form 1's passes but lets the last one write the CG direction
p = Pg + beta p, with <Pg|g> from the Krylov moments.  Form 3 is the default; 1 and 2 are
selectable.  One CG call (Ncg = 3)
from the same start must give the same Ritz values, residuals and bands up to FP32 rounding.  The cases cover every code path of the fused kernel:
rows read from shared memory (t0, c0, tk: rows of 16, 24 and 32 reals) and by warp shuffle
(c1 grid: 64 reals, c3 / c4 grids: 128 reals), real and complex (interleaved) bands, halos that
wrap several times around a small grid (t0), a ragged last y-tile (c0), mloop 1, 2 and 3.
"""
import numpy as np
import pytest

from rsdft_develop_b200 import api, synth

pytestmark = pytest.mark.gpu


def _cg_once(prob, psis, form, mloop):
    out = []
    with api.BandUpdate(prob, precision=api.PREC_MIXED, mloop=mloop) as g:
        g.pc_form(form)
        for k, psi in enumerate(psis):
            g.set_wf(psi, k=k + 1)
            esp, res = g.conjugate_gradient(k=k + 1)
            out.append((np.asarray(esp).copy(), np.asarray(res).copy(), g.get_wf(k=k + 1)))
    return out


def _start(prob, nb, seed, nk):
    psis = []
    with api.BandUpdate(prob) as g:
        for k in range(nk):
            g.random_wf(seed, k=k + 1)
            g.gram_schmidt(k=k + 1)
            g.subspace_diag(k=k + 1)
            psis.append(g.get_wf(k=k + 1)[:nb])
    return psis


CASES = [
    ("t0", None, 1, 3), ("t0", None, 1, 1), ("c0", None, 1, 3), ("c0", None, 1, 2),
    ("tk", None, 2, 3), ("c1", 24, 1, 3), ("c3", 8, 1, 3), ("c4", 16, 2, 3),
]


@pytest.mark.parametrize("form", [2, 3])
@pytest.mark.parametrize("name,nband,nk,mloop", CASES)
def test_fused_preconditioner_cg_matches_multipass(name, nband, nk, mloop, form):
    over = {}
    if nband:
        over["nband"] = nband
        if name == "c4":
            over["nband_range"] = (nband, nband)
    cfg = synth.get_config(name, **over)
    prob = synth.make_problem(cfg)
    nb = int(prob.nband_k[0])
    psis = _start(prob, nb, 81, nk)
    ref = _cg_once(prob, psis, 1, mloop)
    fus = _cg_once(prob, psis, form, mloop)
    for k in range(nk):
        (e1, r1, u1), (e2, r2, u2) = ref[k], fus[k]
        assert np.all(np.isfinite(e2)) and np.all(np.isfinite(r2)) and np.all(np.isfinite(u2))
        scale = max(1.0, float(np.max(np.abs(e1))))
        assert np.max(np.abs(e2 - e1)) <= 2e-5 * scale, (k, np.max(np.abs(e2 - e1)))
        assert np.max(np.abs(r2 - r1)) <= 1e-3 * np.max(r1) + 1e-9, (k, r1, r2)
        du = np.max(np.abs(u2 - u1)) / np.max(np.abs(u1))
        assert du <= 2e-4, (k, du)


def test_fused_preconditioner_mixed_sweeps_converge():
    """Mixed sweeps with the fused forms reach the tolerance in about the sweeps of form 1."""
    prob = synth.make_problem("c0")
    mb = prob.nband - prob.nband // 8
    its = {}
    for form in (1, 2, 3):
        with api.BandUpdate(prob, precision=api.PREC_MIXED) as g:
            g.pc_form(form)
            g.init_sweep(mb)
            g.random_wf(82)
            g.gram_schmidt()
            it, esp, res = g.calc_sweep(400, tol=1e-8)
            assert res[0, 0, :mb].max() <= 1e-8, (form, it)
            its[form] = (it, esp[0, 0].copy())
    for form in (2, 3):
        assert abs(its[form][0] - its[1][0]) <= max(3, its[1][0] // 10), its
        assert np.max(np.abs(its[form][1][:mb] - its[1][1][:mb])) < 1e-8
