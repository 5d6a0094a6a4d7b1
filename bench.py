"""Benchmark: seconds to band residual 1e-8 on one B200 (plus hpsi HBM GB/s).

Default workload: the 128^3 grid / 2048-band real8 problem (512 s+p atoms), mixed precision
with precond_hprsdft.  A step is one complete band-update solve through the C ABI, as a Fortran
host would drive it: set_wf from pinned host FP64 wavefunctions (host -> device), gram_schmidt,
calc_sweep (CG -> fused GS/SD per sweep, FP64 residual check) until max_n res(n) <= 1e-8 over
bands 1..mb_ref, res = dV |H psi - e psi|^2 (src/conjugate_gradient/cg_module.f90:231), then
get_wf back into pinned host memory (device -> host).  Every step starts from the same seeded
wavefunctions.

JSON line keys beyond the driver contract:
  value / ms_per_step  device time of the solve with the inputs resident (CUDA events on the
                       library stream between the end of the host->device copy and the end of
                       the last sweep), mean over the timed steps
  e2e                  wall time of the whole step, copies included (same loop)
  roofline             the hpsi stencil kernel: algorithmic bytes (read psi + write H psi per
                       band, V_loc once) over its CUDA-event time, both taken inside the library
                       on its own stream during the timed steps
  compare              one solve of the plain FP64 method (the drop-in's FP64 path with
                       precond_hprsdft) from the same input; optional mixed + learned solve
  errors               eigenvalues and subspace of the timed solve against that FP64 solve
  cpu_baseline         the CPU oracle (restatement of the reference CPU path) on the host
                       cores: a measured sweep where the problem is small, else sampled CG and
                       dense costs extrapolated to a sweep, times the FP64 method's sweeps
  clocks               nvidia-smi samples during the timed steps

--impl reference times the same CPU oracle alone (bounded sample per step) for the same config.
--kernel hpsi|gemm|pc|cg|lpc runs one kernel family on its own (timing and ncu captures).
--config o2 times the reference's own O2 sample (PSV pseudopotential, PBE, two spins, 18 bands,
48^3): a step is its sweep phase (10 sweeps), compared per sweep with the reference's logged
time(sweep), and the converged band energies are checked against the logs.
Multi-GPU runs are independent replicas (one problem per GPU): every rank solves its own copy
and the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "s to band residual 1e-8: mixed+learned vs plain FP64 on 1 GPU; hpsi HBM GB/s"
TOL = 1e-8
MAX_SWEEPS = 600
SEED = 1

# Sweeps the plain FP64 method needs from the seeded start to max res <= 1e-8 over bands
# 1..mb_ref (the same algorithm on CPU and GPU), measured with the library's FP64 path on a
# B200; the reference arm multiplies its per-sweep CPU time by these.
SWEEPS_FP64 = {"c0": 75, "c1": 43, "c2": 46, "c3": 50, "c4": 45}

# DRAM traffic of one hpsi stencil launch over its algorithmic bytes, from an ncu capture
# (dram__bytes_read.sum + dram__bytes_write.sum) of the same kernel, per (config, precision).
# c3 FP32 (k_stencil_ws): 741.30 + 498.49 MB for 64 bands against 1082 MB algorithmic (one launch);
# traffic grows with the bands, so the ratio scales to the solve's 256-band launches.
NCU_TRAFFIC_RATIO: dict = {("c3", "mixed"): 1.146}


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), float(d["bf16_tflops"]), "measured"
    return 6650.0, 1590.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle samples every 200 ms while the block runs."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) >= 9:
                    rows.append(f)
        except OSError:
            pass
        finally:
            try:
                os.unlink(self.path)
            except OSError:
                pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [num(r[1]) for r in rows]
        smax = [num(r[2]) for r in rows]
        pw = [num(r[3]) for r in rows]
        loaded = [s for s, p in zip(sm, pw) if s is not None and p is not None and p > 200.0]
        loaded = loaded or [s for s in sm if s is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        smax = [s for s in smax if s is not None]
        pw = [p for p in pw if p is not None]
        return {"sm_mhz": statistics.median(loaded) if loaded else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": reasons,
                "samples": len(rows), "power_w_max": max(pw) if pw else None}


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws <= 1:
        return None, 0, 1
    import datetime
    import torch.distributed as dist
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=3600))
    return dist, dist.get_rank(), ws


def _max_over_ranks(dist, x):
    if dist is None or x is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _barrier(dist):
    if dist is not None:
        dist.barrier()


def mb_ref_of(nband: int) -> int:
    """Convergence band set: bands 1..mb_ref, mb_ref = (nband + nocc)/2 with nocc = 3/4 nband
    (the reference's DOS driver rule max_ref_band = (nb + nocc)/2, src/dos_module.f90:64-65)."""
    return nband - nband // 8


# ----------------------------------------------------------------------------------------
# CPU oracle timing (the reference arm and cpu_baseline)
# ----------------------------------------------------------------------------------------
FULL_SWEEP_MAX = 64 ** 3 * 256  # grid points x bands up to which one whole oracle sweep is timed


def cpu_sweep_estimate(prob, nthreads: int, seed: int = 7):
    """Seconds per CG + GS + SD sweep of the oracle on `nthreads` host threads.

    Small problems: one whole sweep, timed.  Larger ones: the oracle's CG on a few bands (its
    work is independent per band, MB_d = 1) and its Gram-Schmidt + subspace diagonalisation on
    m bands (work ~ Ng m^2) are timed on the configuration's own grid and operator and scaled
    to all bands.  Returns (seconds, description, kind)."""
    from oracle import oracle as orc
    orc.build()
    orc.set_threads(nthreads)
    o = orc.Oracle(prob)
    nb, ng = prob.nband, prob.ng
    nbk = [int(x) for x in prob.nband_k]
    rng = np.random.default_rng(seed)
    if prob.nk == 1 and ng * nb <= FULL_SWEEP_MAX:
        from rsdft_develop_b200 import synth
        psi = o.gram_schmidt(synth.random_wavefunctions(seed, nb, ng))
        t0 = time.perf_counter()
        o.sweep(psi, 1)
        t = time.perf_counter() - t0
        return t, f"one whole oracle sweep (CG+GS+SD, {nb} bands)", "measured"
    ncg_b = 8
    m = min(128, nbk[0])
    psi = rng.standard_normal((m, ng))
    if prob.is_complex:
        psi = psi + 1j * rng.standard_normal((m, ng))
    t0 = time.perf_counter()
    q = o.gram_schmidt(psi)
    o.subspace_diag(q)
    t_dense = time.perf_counter() - t0
    t0 = time.perf_counter()
    o.cg(q[:ncg_b])
    t_cg = (time.perf_counter() - t0) / ncg_b
    # subspace_diag applies H to each band (work ~ Ng m): that part scales with the bands, the
    # rest of GS + SD (the Ng m^2 products) with their square
    t0 = time.perf_counter()
    o.hpsi(q[:ncg_b])
    t_h = (time.perf_counter() - t0) / ncg_b
    t_quad = max(0.0, t_dense - m * t_h)
    est = sum(n * (t_cg + t_h) + (n / m) ** 2 * t_quad for n in nbk)
    kdesc = f" per k-point, summed over {prob.nk} k-points with {nbk} bands" if prob.nk > 1 else ""
    desc = (f"extrapolated: oracle CG on {ncg_b} bands ({t_cg:.3f} s per band) and H psi ({t_h:.4f} s per band) "
            f"x the bands + oracle GS+SD products on {m} bands ({t_quad:.2f} s) x (bands/{m})^2{kdesc}")
    return est, desc, "extrapolated"


def run_reference(args, dist, rank, ws):
    """The CPU restatement of the reference path (oracle/) on the host cores, same config."""
    if rank != 0:
        return
    from rsdft_develop_b200 import synth
    prob = synth.make_problem(args.config)
    nthreads = os.cpu_count() or 1
    n_conv = SWEEPS_FP64[args.config]
    samples, desc, kind = [], "", ""
    for i in range(args.warmup + args.steps):
        per, desc, kind = cpu_sweep_estimate(prob, nthreads, seed=7 + i)
        if i >= args.warmup:
            samples.append(per)
    per = statistics.median(samples)
    val = per * n_conv
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": "s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": per * 1000.0,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded)",
        "config": {"workload": args.config, "grid": list(prob.n), "bands": prob.nband, "atoms": prob.cfg.natom,
                   "precision": "fp64", "pc": "hprsdft", "sweeps_to_tol": n_conv, "mb_ref": mb_ref_of(prob.nband)},
        "cpu_baseline": {"value": val, "unit": "s", "cores": nthreads, "kind": "port",
                         "sample": f"per step: {desc}; median {per:.2f} s per sweep on {nthreads} host threads "
                                   f"(oracle/ restatement of the reference CPU path) x {n_conv} sweeps, the "
                                   f"FP64 method's count to max res <= 1e-8 (measured on the GPU)",
                         "estimate": kind},
        "e2e": {"value": val, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------------------
# error of a solve against the FP64 solve of the same input
# ----------------------------------------------------------------------------------------
def gap_index(esp: np.ndarray, lo: int, hi: int) -> int:
    """Band count m in [lo, hi] whose gap e_{m+1} - e_m is largest (a subspace boundary)."""
    gaps = esp[lo:hi + 1] - esp[lo - 1:hi]
    return lo + int(np.argmax(gaps))


def principal_angle_max(a_host, b_host, m: int, dv: float) -> float:
    """Largest principal angle (rad) between span(a[:m]) and span(b[:m]) in the dV inner
    product; a, b are host tensors (nb, ng) of FP64 (or complex128) bands.  Evaluated on the GPU
    in FP64."""
    import torch
    A = a_host[:m].cuda()
    B = b_host[:m].cuda()
    ga = (A.conj() @ A.T) * dv
    gb = (B.conj() @ B.T) * dv
    M = (A.conj() @ B.T) * dv
    del A, B
    la = torch.linalg.cholesky(ga)
    lb = torch.linalg.cholesky(gb)
    # singular values of La^-1 M Lb^-H: the cosines of the principal angles
    X = torch.linalg.solve_triangular(la, M, upper=False)
    X = torch.linalg.solve_triangular(lb.conj(), X.T, upper=False).T
    s = torch.linalg.svdvals(X)
    smin = float(s.min().clamp(max=1.0))
    # sin(theta) = sqrt(1 - s^2), accurate for small angles
    return float(np.arcsin(min(1.0, np.sqrt(max(0.0, (1.0 - smin) * (1.0 + smin))))))


# ----------------------------------------------------------------------------------------
# our arm
# ----------------------------------------------------------------------------------------
def run_ours(args, dist, rank, ws):
    import torch
    from rsdft_develop_b200 import api, lpc_train, synth
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    prob = synth.make_problem(args.config)
    nb, ng = prob.nband, prob.ng
    mb_ref = mb_ref_of(nb)
    prec = api.PREC_MIXED if args.precision == "mixed" else api.PREC_FP64
    pc = args.pc
    wpath = lpc_train.default_weights_path(prob.h)
    pc_mode = {"learned": api.PC_LEARNED, "hprsdft": api.PC_HPRSDFT, "none": api.PC_NONE}[pc]
    terms = tuple(int(t) for t in args.gemm_terms.split(","))
    compare_arms = [a for a in args.compare.split(",") if a and a != "none"]

    # the common input: seeded FP64 (complex128 for k-points) wavefunctions in pinned host memory,
    # made by the library's device generator (bit-identical to synth.random_wavefunctions)
    nk = prob.nk
    nbk = [int(x) for x in prob.nband_k]
    dt = torch.complex128 if prob.is_complex else torch.float64
    pin_in = [torch.empty((nbk[k], ng), dtype=dt, pin_memory=True) for k in range(nk)]
    pin_out = [torch.empty((nbk[k], ng), dtype=dt, pin_memory=True) for k in range(nk)]
    with api.BandUpdate(prob, precision=api.PREC_FP64) as g0:
        for k in range(nk):
            g0.random_wf(SEED, k=k + 1)
            g0.get_wf_host(pin_in[k].data_ptr(), nbk[k], k=k + 1)
    # convergence band set: bands 1..mb_ref (one k-point), or per k-point the same 7/8 rule
    sweep_ref = mb_ref if nk == 1 else -1
    conv = [min(mb_ref, nb_) if nk == 1 else nb_ - nb_ // 8 for nb_ in nbk]

    g = api.BandUpdate(prob, precision=prec, pc_mode=pc_mode)
    g.gemm_terms(*terms)
    sched = tuple(float(x) for x in args.gemm_schedule.split(","))
    if prec == api.PREC_MIXED:
        g.gemm_schedule(*sched)
    g.pc_form(args.pc_form)
    g.stencil_form(args.stencil_form)
    if pc == "learned":
        g.lpc_set_weights(np.load(wpath))
    g.init_sweep(sweep_ref)
    stream = torch.cuda.ExternalStream(g.stream())

    def step():
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ev[0].record(stream)
        for k in range(nk):
            g.set_wf_host(pin_in[k].data_ptr(), nbk[k], k=k + 1)
        ev[1].record(stream)
        for k in range(nk):
            g.gram_schmidt(k=k + 1)
        it, esp, res = g.calc_sweep(MAX_SWEEPS, tol=TOL)
        ev[2].record(stream)
        for k in range(nk):
            g.get_wf_host(pin_out[k].data_ptr(), nbk[k], k=k + 1)
        ev[3].record(stream)
        ev[3].synchronize()
        wall = time.perf_counter() - t0
        return it, esp, res, ev[1].elapsed_time(ev[2]) / 1000.0, wall

    for _ in range(args.warmup):
        step()
    g.synchronize()
    _barrier(dist)
    torch.cuda.synchronize()
    launches0 = g.kernel_launches()
    g.profile(2)  # the hpsi stencil's own CUDA events only: no host synchronisation
    iters, solve_s, wall_s = [], [], []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            it, esp, res, ts, tw = step()
            iters.append(it)
            solve_s.append(ts)
            wall_s.append(tw)
    torch.cuda.synchronize()
    _barrier(dist)
    launches = g.kernel_launches() - launches0
    st_ms, st_n, st_bytes, _ = g.profile_get("hpsi_stencil")
    g.profile(0)
    tune = {k_: g.profile_get(k_)[0] for k_ in ("stencil_tile_y", "stencil_warps", "stencil_stages", "stencil_zchunks")}
    lpc_state = g.lpc_status()
    shares = {}
    if args.shares:  # one extra, untimed solve with every kernel family timed
        g.profile(1)
        step()
        names = ["hpsi_stencil", "nl_gather", "nl_scatter", "cg", "pc", "lpc", "gs", "gemm", "sd_gemm",
                 "sd_eig", "sd_rot", "residual"]
        shares = {n: round(g.profile_get(n)[0], 3) for n in names}
        g.profile(0)
    clocks = clk.summary()
    esp_main = [esp[0, k, :nbk[k]].copy() for k in range(nk)]
    res_max = float(max(np.max(res[0, k, :conv[k]]) for k in range(nk)))
    g.close()
    t_solve = _max_over_ranks(dist, statistics.mean(solve_s))
    e2e_val = _max_over_ranks(dist, statistics.mean(wall_s))

    # comparison solves on the same GPU and input (after the timed steps; the FP64 result
    # overwrites the input buffers, which are no longer needed)
    compare, errors = {}, None
    arms = []
    if "mixed_learned" in compare_arms and os.path.exists(wpath) and not (prec == api.PREC_MIXED and pc == "learned"):
        arms.append(("mixed_learned", api.PREC_MIXED, api.PC_LEARNED))
    if "mixed_hprsdft" in compare_arms and not (prec == api.PREC_MIXED and pc == "hprsdft"):
        arms.append(("mixed_hprsdft", api.PREC_MIXED, api.PC_HPRSDFT))
    if "fp64" in compare_arms and prec != api.PREC_FP64:
        arms.append(("fp64_hprsdft", api.PREC_FP64, api.PC_HPRSDFT))
    for name, pr, pm in arms:
        with api.BandUpdate(prob, precision=pr, pc_mode=pm) as h:
            if pm == api.PC_LEARNED:
                h.lpc_set_weights(np.load(wpath))
            h.init_sweep(sweep_ref)
            hs = torch.cuda.ExternalStream(h.stream())
            for k in range(nk):
                h.set_wf_host(pin_in[k].data_ptr(), nbk[k], k=k + 1)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(hs)
            for k in range(nk):
                h.gram_schmidt(k=k + 1)
            itc, espc, resc = h.calc_sweep(MAX_SWEEPS, tol=TOL)
            e1.record(hs)
            e1.synchronize()
            tc = _max_over_ranks(dist, e0.elapsed_time(e1) / 1000.0)
            entry = {"s": round(tc, 4), "sweeps": itc,
                     "final_res_max": float(max(np.max(resc[0, k, :conv[k]]) for k in range(nk)))}
            if pm == api.PC_LEARNED:
                entry["lpc_fallbacks"] = h.lpc_status()[2]
            if name == "fp64_hprsdft":
                for k in range(nk):
                    h.get_wf_host(pin_in[k].data_ptr(), nbk[k], k=k + 1)
                esp64 = [espc[0, k, :nbk[k]].copy() for k in range(nk)]
        compare[name] = entry
        if name == "fp64_hprsdft":
            compare["speedup_vs_fp64_hprsdft"] = round(tc / t_solve, 3)
            eig_err, ang, ms, gaps = 0.0, 0.0, [], []
            for k in range(nk):
                ck = conv[k]
                eig_err = max(eig_err, float(np.max(np.abs(esp_main[k][:ck] - esp64[k][:ck]))))
                m = gap_index(esp64[k], max(1, ck - 32), min(ck, nbk[k] - 1))
                ang = max(ang, principal_angle_max(pin_out[k], pin_in[k], m, prob.dV))
                ms.append(m)
                gaps.append(float(esp64[k][m] - esp64[k][m - 1]))
            errors = {"vs": "fp64_hprsdft solve of the same input", "eig_err_max_Ha": eig_err,
                      "principal_angle_max_rad": ang, "subspace_bands": ms if nk > 1 else ms[0],
                      "gap_Ha": gaps if nk > 1 else gaps[0]}

    hbm, bf16, peak_kind = _peaks()
    avg_ms = (st_ms / st_n) if st_n else None
    bytes_launch = (st_bytes / st_n) if st_n else None
    achieved = bytes_launch / (avg_ms * 1e-3) / 1e9 if st_n else 0.0
    ratio = NCU_TRAFFIC_RATIO.get((args.config, args.precision))
    kname = ("k_stencil_ws_c" if prob.is_complex else "k_stencil_ws") + ("<float>" if prec == api.PREC_MIXED else "<double>")
    kdesc = ("hpsi 37-point Bloch-phase stencil + V_loc (nonlocal scatter separate)" if prob.is_complex
             else "hpsi 37-point stencil + V_loc (nonlocal scatter separate)")
    roof = {"bound": "hbm", "kernel": f"{kname}: {kdesc}",
            "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s", "frac": round(achieved / hbm, 4),
            "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
            "traffic": (ratio * bytes_launch) if (ratio and bytes_launch) else None,
            "launches": st_n, "avg_launch_ms": avg_ms, "algorithmic_bytes_per_launch": bytes_launch,
            "config": tune}

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        nthreads = os.cpu_count() or 1
        per, desc, kind = cpu_sweep_estimate(prob, nthreads)
        n_conv = compare.get("fp64_hprsdft", {}).get("sweeps") or SWEEPS_FP64.get(args.config)
        cpu = {"value": per * n_conv, "unit": "s", "cores": nthreads, "kind": "port", "estimate": kind,
               "sample": f"{desc}: {per:.2f} s per sweep on {nthreads} host threads (oracle/ restatement of the "
                         f"reference CPU path) x {n_conv} sweeps of the FP64 method to max res <= 1e-8"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": t_solve, "unit": "s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_solve * 1000.0, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f32+bf16x%d/x%d+f64" % terms,
            "data": "synthetic (seeded Gaussian V_loc, Gaussian s/p projectors, seeded psi0)",
            "config": {"workload": args.config, "grid": list(prob.n), "bands": nbk if nk > 1 else nb,
                       "kpoints": nk, "storage": "complex128" if prob.is_complex else "real8", "atoms": prob.cfg.natom,
                       "projectors": prob.nzlma, "precision": args.precision, "pc": pc,
                       "lpc_fallbacks": lpc_state[2] if pc == "learned" else None,
                       "gemm_terms": list(terms) if prec == api.PREC_MIXED else None,
                       "gemm_schedule": list(sched) if prec == api.PREC_MIXED else None,
                       "pc_form": args.pc_form,
                       "mb_ref": conv if nk > 1 else mb_ref, "tol": TOL, "sweeps_to_tol": iters,
                       "final_res_max": res_max,
                       "l2": "inputs larger than L2 (psi >= 0.5 GB)", "parallelism": f"replicas x{ws}"},
            "gpu_launches": int(launches),
            "roofline": roof,
            "errors": errors,
            "compare": compare,
            "time_shares_ms": shares or None,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_val, "unit": "s", "h2d_bytes_per_step": int(sum(p.nbytes for p in pin_in)),
                    "d2h_bytes_per_step": int(sum(p.nbytes for p in pin_out) + 2 * esp.nbytes)},
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------------------
# single kernel families (timing and ncu captures)
# ----------------------------------------------------------------------------------------
# ----------------------------------------------------------------------------------------
# the reference's own O2 sample (--config o2)
# ----------------------------------------------------------------------------------------
O2_METRIC = "s per sweep phase of the reference's O2 sample (10 sweeps, 2 spins, 18 bands, 48^3, PBE)"
O2_NSWEEP = 10                   # Nsweep of the sample's input (fort.1)
O2_REF_SWEEP_S = 0.083           # fastest logged time(sweep), real8 build, 36 MPI ranks


def _o2_setup():
    from rsdft_develop_b200 import pseudo, structure
    pp = pseudo.load_npz(os.path.join(ROOT, "tests", "golden", "o_pbe_rc15_psv.npz"))
    su = structure.setup(structure.o2_molecule(pp))
    logs = json.load(open(os.path.join(ROOT, "tests", "golden", "reference_logs.json")))["o2"]
    return su, logs


def _o2_cpu_sweep(su, nthreads: int, nsweep: int = 2):
    """Oracle sweeps (FP64, both spins) on the O2 operator: seconds per sweep."""
    from oracle import oracle as orc
    from rsdft_develop_b200 import synth
    orc.set_threads(nthreads)
    t = 0.0
    for s in (1, 2):
        prob = su.problem_for_spin(s)
        o = orc.Oracle(prob)
        psi = o.gram_schmidt(synth.random_wavefunctions(SEED + s, prob.nband, prob.ng))
        t0 = time.perf_counter()
        o.sweep(psi, nsweep)
        t += time.perf_counter() - t0
    return t / nsweep


def run_o2(args, dist, rank, ws):
    """The O2 sample's sweep phase through the C ABI: per step set_wf (host -> device) of both
    spins' seeded bands, gram_schmidt, 10 sweeps of the operator of the initial density, get_wf
    (device -> host); after timing, converged band energies against the reference's logs."""
    nthreads = os.cpu_count() or 1
    su, logs = _o2_setup()
    if args.impl == "reference":
        if rank != 0:
            return
        samples = [_o2_cpu_sweep(su, nthreads) for _ in range(args.warmup + args.steps)][args.warmup:]
        per = statistics.median(samples)
        val = per * O2_NSWEEP
        print(json.dumps({
            "impl": "reference", "metric": O2_METRIC, "value": val, "unit": "s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": val * 1000.0, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": round(per / O2_REF_SWEEP_S, 4), "dtype": "f64",
            "data": "the reference's O2 sample operator (O_PBE_RC1.5.psv, initial-density PBE potential)",
            "config": {"workload": "o2", "grid": [48, 48, 48], "bands": 18, "spins": 2, "precision": "fp64"},
            "cpu_baseline": {"value": val, "unit": "s", "cores": nthreads, "kind": "port",
                             "sample": f"2 oracle sweeps per spin per step, median {per:.3f} s per sweep x {O2_NSWEEP}"},
            "e2e": {"value": val, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}), flush=True)
        return
    import torch
    from rsdft_develop_b200 import api, synth
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    prec = api.PREC_FP64 if args.precision == "fp64" else api.PREC_MIXED
    prob = su.problem_for_spin(1)
    nb, ng = prob.nband, prob.ng
    pin_in = [torch.from_numpy(synth.random_wavefunctions(SEED + s, nb, ng)).pin_memory() for s in (1, 2)]
    pin_out = [torch.empty((nb, ng), dtype=torch.float64).pin_memory() for _ in (1, 2)]
    g = api.BandUpdate(prob, precision=prec, nspin=2)
    g.set_vloc(su.vloc[1], s=2)
    g.init_sweep(7)
    stream = torch.cuda.ExternalStream(g.stream())

    def step():
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for s in (1, 2):
            g.set_wf_host(pin_in[s - 1].data_ptr(), nb, s=s)
        ev[0].record(stream)
        for s in (1, 2):
            g.gram_schmidt(s=s)
        g.calc_sweep(O2_NSWEEP)
        ev[1].record(stream)
        for s in (1, 2):
            g.get_wf_host(pin_out[s - 1].data_ptr(), nb, s=s)
        ev[2].record(stream)
        ev[2].synchronize()
        return ev[0].elapsed_time(ev[1]) / 1000.0, time.perf_counter() - t0

    for _ in range(args.warmup):
        step()
    _barrier(dist)
    torch.cuda.synchronize()
    l0 = g.kernel_launches()
    dev, wall = [], []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            d, w = step()
            dev.append(d)
            wall.append(w)
    torch.cuda.synchronize()
    _barrier(dist)
    launches = g.kernel_launches() - l0
    clocks = clk.summary()
    # converged band energies of the same start against the logged ones
    if prec == api.PREC_MIXED:
        g.calc_sweep(200, tol=1e-9)
        g.set_precision(api.PREC_FP64)
    it, esp, res = g.calc_sweep(200, tol=1e-20)
    g.close()
    err15 = err67 = 0.0
    for log in logs:
        for s in (1, 2):
            col = 2 if s == 1 else 5
            ref = np.array([r[col] for r in log["esp_scf1"][:7]])
            err15 = max(err15, float(np.max(np.abs(esp[s - 1, 0, :5] - ref[:5]))))
            err67 = max(err67, float(np.max(np.abs(esp[s - 1, 0, 5:7] - ref[5:7]))))
    val = _max_over_ranks(dist, statistics.mean(dev))
    e2e = _max_over_ranks(dist, statistics.mean(wall))
    if rank != 0:
        return
    cpu = None
    if not args.no_cpu_baseline:
        per = _o2_cpu_sweep(su, nthreads)
        cpu = {"value": per * O2_NSWEEP, "unit": "s", "cores": nthreads, "kind": "port",
               "sample": f"2 oracle sweeps per spin on {nthreads} host threads: {per:.3f} s per sweep x {O2_NSWEEP}"}
    print(json.dumps({
        "metric": O2_METRIC, "value": val, "unit": "s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": val * 1000.0, "ms_per_sweep": val * 1000.0 / O2_NSWEEP, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": round(val / O2_NSWEEP / O2_REF_SWEEP_S, 4),
        "vs_baseline_note": f"per sweep over the fastest logged reference time(sweep), {O2_REF_SWEEP_S} s "
                            "(real8 build, 36 MPI ranks, samples_for_supercomputers/ITO_KYUSHU-U)",
        "dtype": "f64" if prec == api.PREC_FP64 else "f32+bf16x3+f64",
        "data": "the reference's O2 sample operator (O_PBE_RC1.5.psv, initial-density PBE potential)",
        "config": {"workload": "o2", "grid": [48, 48, 48], "bands": nb, "spins": 2, "precision": args.precision,
                   "nsweep": O2_NSWEEP, "l2": "inputs smaller than L2 (3.2 MB of bands per spin)"},
        "errors": {"vs": "band energies printed by the reference's eight O2 logs (scf_iter 1)",
                   "bands_1_5_max_Ha": err15, "bands_6_7_max_Ha": err67, "converged_sweeps": it},
        "gpu_launches": launches, "cpu_baseline": cpu,
        "e2e": {"value": e2e, "unit": "s", "h2d_bytes_per_step": 2 * nb * ng * 8, "d2h_bytes_per_step": 2 * nb * ng * 8},
        "clocks": clocks}), flush=True)


def run_kernel(args):
    import torch
    from rsdft_develop_b200 import api, lpc_train, synth
    what = args.kernel
    reps = args.reps
    if what == "gemm":
        m, k = args.bands or 256, args.points or 262144
        terms = int(args.gemm_terms.split(",")[0])
        with api.BandUpdate(synth.make_problem("t0")) as g:
            g.gemm_terms(terms, terms)
            g.selftest_gemm(m, m, k, 0)  # untimed: module load, tensor-map encoder
            g.profile(1)
            e0 = g.selftest_gemm(m, m, k, 0)
            ms0, _, _, fl0 = g.profile_get("gemm")
            e1 = g.selftest_gemm(m, m, k, 1)
            ms, n, _, fl = g.profile_get("gemm")
            print(f"gemm m={m} k={k} terms={terms}: overlap rel.err {e0:.2e} {ms0:.3f} ms "
                  f"({fl0 / max(ms0, 1e-9) / 1e9:.0f} TFLOP/s bf16), rotation rel.err {e1:.2e} {ms - ms0:.3f} ms "
                  f"({(fl - fl0) / max(ms - ms0, 1e-9) / 1e9:.0f} TFLOP/s bf16)", flush=True)
        return
    prob = synth.make_problem(args.config)
    nb = min(args.bands or prob.nband, prob.nband)
    if what == "hpsi":
        precs = {"both": ("fp64", "fp32"), "fp64": ("fp64",), "fp32": ("fp32",)}[args.hpsi_prec]
        with api.BandUpdate(prob, nonlocal_on=not args.no_nonlocal) as g:
            g.stencil_form(args.stencil_form)
            # complex bands are interleaved (re, im): 2 ng reals each
            ncomp = 2 if prob.is_complex else 1
            x = torch.empty((nb, ncomp * prob.ng), dtype=torch.float64, device="cuda")
            x.uniform_(-1.0, 1.0)
            for name in precs:
                f32 = name == "fp32"
                a = x.float() if f32 else x
                b = torch.empty_like(a)
                g.hamiltonian_device(a.data_ptr(), b.data_ptr(), nb, fp32=f32)  # untimed first call
                g.synchronize()
                g.profile(1)
                for _ in range(reps):
                    g.hamiltonian_device(a.data_ptr(), b.data_ptr(), nb, fp32=f32)
                g.synchronize()
                ms, n, by, _ = g.profile_get("hpsi_stencil")
                gms, gn, _, _ = g.profile_get("nl_gather")
                sms, sn, _, _ = g.profile_get("nl_scatter")
                pre = "stencil" if f32 else "stencil64"
                cfg = {k: g.profile_get(f"{pre}_{k}")[0] for k in ("tile_y", "warps", "stages", "zchunks")}
                print(f"hpsi {args.config} {name} bands={nb}: stencil {ms / max(n, 1):.3f} ms "
                      f"({by / max(ms, 1e-9) / 1e6:.1f} GB/s algorithmic), gather {gms / max(gn, 1):.3f} ms, "
                      f"scatter {sms / max(sn, 1):.3f} ms; {cfg}", flush=True)
                g.profile(0)
                del a, b
        return
    if what == "cg":
        # one conjugate_gradient call (Ncg = 3) on nb bands, mixed precision with precond_hprsdft
        cfg = synth.get_config(args.config, nband=nb)
        if prob.is_complex:
            cfg = synth.get_config(args.config, nband=nb, nband_range=(nb, nb))
        pb = synth.make_problem(cfg)
        with api.BandUpdate(pb, precision=api.PREC_MIXED) as g:
            g.pc_form(args.pc_form)
            g.random_wf(5)
            g.gram_schmidt()
            g.conjugate_gradient()  # untimed first call
            g.profile(1)
            for _ in range(reps):
                g.random_wf(5)
                g.gram_schmidt()
                g.conjugate_gradient()
            g.synchronize()
            shares = {n: g.profile_get(n)[0] / reps for n in ("pc", "cg", "hpsi_stencil", "nl_gather", "nl_scatter")}
            g.profile(0)
        print(f"cg {args.config} bands={nb} pc_form={args.pc_form}: per call " +
              ", ".join(f"{k} {v:.3f} ms" for k, v in shares.items()), flush=True)
        return
    rng = np.random.default_rng(3)
    g_in = rng.standard_normal((nb, prob.ng))
    if what == "pc":
        for f32 in (False, True):
            with api.BandUpdate(prob, precision=api.PREC_MIXED if f32 else api.PREC_FP64) as g:
                run = (lambda: g.precond_f32(g_in)) if f32 else (lambda: g.precond(g_in))
                run()
                g.profile(1)
                for _ in range(reps):
                    run()
                ms, n, _, _ = g.profile_get("pc")
                print(f"precond_hprsdft ({'FP32 s-step' if f32 else 'FP64'}) {args.config} bands={nb}: "
                      f"{ms / reps:.3f} ms per application", flush=True)
    elif what == "lpc":
        with api.BandUpdate(prob, precision=api.PREC_MIXED, pc_mode=api.PC_LEARNED) as g:
            g.lpc_set_weights(np.load(lpc_train.default_weights_path(prob.h)))
            x = g_in.astype(np.float32)
            for mode in ("tc", "fp32"):
                g.lpc_inference(fp32=(mode == "fp32"))
                g.lpc_precond(x)
                g.profile(1)
                for _ in range(reps):
                    g.lpc_precond(x)
                ms, n, _, fl = g.profile_get("lpc")
                print(f"learned preconditioner ({mode}) {args.config} bands={nb}: {ms / reps:.3f} ms per "
                      f"application, {fl / max(ms, 1e-9) / 1e9:.1f} TFLOP/s", flush=True)
                for part in ("lpc_layer1", "lpc_mid", "lpc_layer4"):
                    pms, _, pby, pfl = g.profile_get(part)
                    if pms > 0:
                        print(f"  {part}: {pms / reps:.3f} ms, {pfl / pms / 1e9:.1f} TFLOP/s", flush=True)
                g.profile(0)
    else:
        raise SystemExit(f"unknown kernel family {what!r}")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c3",
                    help="workload: c0, c1, c2, c3 (real8) (default c3), c4 (complex16), o2 (the reference's O2 sample)")
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--pc", default="hprsdft", choices=["learned", "hprsdft", "none"], help="CG preconditioner")
    ap.add_argument("--compare", default="fp64",
                    help="comma list of comparison solves: fp64, mixed_hprsdft, mixed_learned, none")
    ap.add_argument("--shares", action="store_true", help="one extra untimed solve with per-kernel times")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--gemm-terms", default="3,3",
                    help="BF16 terms of the mixed overlap/Hsub and rotation contractions (2 or 3 each)")
    ap.add_argument("--pc-form", type=int, default=3, help="FP32 preconditioner form inside CG (3 s-step passes with the direction pass, 1 s-step passes, 2 fused, 0)")
    ap.add_argument("--stencil-form", type=int, default=0,
                    help="real-build hpsi stencil: 0 V_loc staged with the planes, 1 V_loc read from L2")
    ap.add_argument("--gemm-schedule", default="1e-2,1e-4",
                    help="mixed precision: two BF16 terms in overlap/Hsub, rotation while CG's residual > these")
    ap.add_argument("--kernel", default="solve", choices=["solve", "hpsi", "gemm", "pc", "cg", "lpc"],
                    help="solve (the benchmark) or one kernel family on its own")
    ap.add_argument("--bands", type=int, default=0, help="--kernel: bands (default all / 256 for gemm)")
    ap.add_argument("--points", type=int, default=0, help="--kernel gemm: K points")
    ap.add_argument("--reps", type=int, default=3, help="--kernel: timed repetitions")
    ap.add_argument("--hpsi-prec", default="both", choices=["both", "fp64", "fp32"])
    ap.add_argument("--no-nonlocal", action="store_true", help="--kernel hpsi: operator without projectors")
    args = ap.parse_args()
    if args.kernel != "solve":
        run_kernel(args)
        return
    dist, rank, ws = _dist()
    try:
        if args.config == "o2":
            run_o2(args, dist, rank, ws)
        elif args.impl == "reference":
            run_reference(args, dist, rank, ws)
        else:
            run_ours(args, dist, rank, ws)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
