"""Drive one kernel family on the GPU for timing and ncu captures.

    python -m rsdft_develop_b200.profile_kernels gemm [m] [k] [terms] [wide|narrow]   # split-BF16 tcgen05 GEMMs
    python -m rsdft_develop_b200.profile_kernels pc|pc32 [config] [bands]   # precond_hprsdft (FP64 / FP32)
    python -m rsdft_develop_b200.profile_kernels lpc [config] [bands] [tc|fp32]  # learned preconditioner

gemm: the overlap S = A A^T (m x m, K = k) and the rotation X <- X V (m bands of k points),
each checked against cuBLAS DGEMM (the relative error is printed), with 3 (default) or 2 BF16
terms per value.  pc / lpc: one application
to `bands` seeded random bands of the configuration's grid, timed by the library's profiling
(CUDA events on its stream) after one untimed call.
"""
from __future__ import annotations

import sys

import numpy as np

from . import api, lpc_train, synth


def main(argv=None):
    argv = list(sys.argv[1:] if argv is None else argv)
    what = argv[0] if argv else "gemm"
    if what == "gemm":
        m = int(argv[1]) if len(argv) > 1 else 256
        k = int(argv[2]) if len(argv) > 2 else 262144
        terms = int(argv[3]) if len(argv) > 3 else 3
        wide = (argv[4] if len(argv) > 4 else "wide") == "wide"
        with api.BandUpdate(synth.make_problem("t0")) as g:
            g.gemm_terms(terms, terms)
            g.gemm_tile(wide)
            g.selftest_gemm(m, m, k, 0)  # untimed: module load, tensor-map encoder
            g.profile(True)
            e0 = g.selftest_gemm(m, m, k, 0)
            ms0, _, _, fl0 = g.profile_get("gemm")
            e1 = g.selftest_gemm(m, m, k, 1)
            ms, n, _, fl = g.profile_get("gemm")
            print(f"gemm m={m} k={k} terms={terms} {'wide' if wide else 'narrow'}: overlap rel.err {e0:.2e} {ms0:.3f} ms "
                  f"({fl0 / max(ms0, 1e-9) / 1e9:.0f} TFLOP/s bf16), rotation rel.err {e1:.2e} {ms - ms0:.3f} ms "
                  f"({(fl - fl0) / max(ms - ms0, 1e-9) / 1e9:.0f} TFLOP/s bf16); {n} calls")
        return
    cfg = argv[1] if len(argv) > 1 else "c1"
    prob = synth.make_problem(cfg)
    nb = int(argv[2]) if len(argv) > 2 else min(64, prob.nband)
    g_in = synth.random_wavefunctions(3, nb, prob.ng)
    if what in ("pc", "pc32"):
        f32 = what == "pc32"
        with api.BandUpdate(prob, precision=api.PREC_MIXED if f32 else api.PREC_FP64) as g:
            run = (lambda: g.precond_f32(g_in)) if f32 else (lambda: g.precond(g_in))
            run()
            g.profile(True)
            run()
            ms, n, _, _ = g.profile_get("pc")
            print(f"precond_hprsdft ({'FP32 s-step' if f32 else 'FP64'}) {cfg} bands={nb}: {ms:.3f} ms ({n} scopes)")
    elif what == "lpc":
        mode = argv[3] if len(argv) > 3 else "tc"
        with api.BandUpdate(prob, precision=api.PREC_MIXED, pc_mode=api.PC_LEARNED) as g:
            w = np.load(lpc_train.default_weights_path(prob.h))
            g.lpc_set_weights(w)
            g.lpc_inference(fp32=(mode == "fp32"))
            x = g_in.astype(np.float32)
            g.lpc_precond(x)
            g.profile(True)
            g.lpc_precond(x)
            ms, n, _, fl = g.profile_get("lpc")
            print(f"learned preconditioner ({mode}) {cfg} bands={nb}: {ms:.3f} ms, "
                  f"{fl / max(ms, 1e-9) / 1e9:.1f} TFLOP/s")
            for part in ("lpc_layer1", "lpc_mid", "lpc_layer4"):
                pms, _, pby, pfl = g.profile_get(part)
                if pms > 0:
                    print(f"  {part}: {pms:.3f} ms, {pby / pms / 1e6:.0f} GB/s, {pfl / pms / 1e9:.1f} TFLOP/s")
    else:
        raise SystemExit(f"unknown kernel family {what!r}")


if __name__ == "__main__":
    main()
