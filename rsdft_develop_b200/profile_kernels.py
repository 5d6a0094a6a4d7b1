"""Drive one kernel family on the GPU for timing and ncu captures.

    python -m rsdft_develop_b200.profile_kernels gemm [m] [k]      # split-BF16 tcgen05 GEMMs
    python -m rsdft_develop_b200.profile_kernels pc [config] [bands]   # precond_hprsdft (FP64)
    python -m rsdft_develop_b200.profile_kernels lpc [config] [bands] [tc|fp32]  # learned preconditioner

gemm: the overlap S = A A^T (m x m, K = k) and the rotation X <- X V (m bands of k points),
each checked against cuBLAS DGEMM (the relative error is printed).  pc / lpc: one application
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
        with api.BandUpdate(synth.make_problem("t0")) as g:
            g.profile(True)
            e0 = g.selftest_gemm(m, m, k, 0)
            e1 = g.selftest_gemm(m, m, k, 1)
            ms, n, _, _ = g.profile_get("gemm")
            print(f"gemm m={m} k={k}: overlap rel.err {e0:.2e}, rotation rel.err {e1:.2e}; "
                  f"{n} x3 launches {ms:.3f} ms total")
        return
    cfg = argv[1] if len(argv) > 1 else "c1"
    prob = synth.make_problem(cfg)
    nb = int(argv[2]) if len(argv) > 2 else min(64, prob.nband)
    g_in = synth.random_wavefunctions(3, nb, prob.ng)
    if what == "pc":
        with api.BandUpdate(prob) as g:
            g.precond(g_in)
            g.profile(True)
            g.precond(g_in)
            ms, n, _, _ = g.profile_get("pc")
            print(f"precond_hprsdft {cfg} bands={nb}: {ms:.3f} ms ({n} scopes)")
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
