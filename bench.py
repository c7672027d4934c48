"""Benchmark: MFISTA lambda-grid solves per second on B200.

Workload (every rank): a 128x128 NUFFT imaging problem with M = 8100 uv
points (10 stations x 180 hour angles, seeded synthetic sky and coverage),
solved for 64 (lambda_l1, lambda_tsv) pairs on an 8x8 log grid spanning
1e-4 .. 1 of max|A^H W^2 y|, nonnegative, zero start.  A solve counts when
its objective is within 1e-6 (relative) of F*, the FP64 optimum obtained
beforehand (untimed) with the library's FP64 batched solver run long.

One step = one batched solve of the 64 problems by the chosen method
(--method, default fp32: FP32 NUFFT/FFT operators with FP64 anchor
correction and an FP64 objective; all problems in one device-resident
CUDA-graph loop, each stopping on its own at F* (1 + 1e-6)).  The other
precision is run once more, untimed, and both forms' accuracy against F*
is reported beside the line.  The plain method (FP64, one problem per
launch) is timed on the same targets as the comparison point, and the e2e
figure repeats the chosen solve through mfista_nufft_batch from pinned host
arrays.  Side measurements (untimed for `value`): the DFT lambda grid in
FP64 and the tensor-core split-BF16 forms, the leave-one-out error of its
solutions against a numpy/LAPACK host baseline, a 48-frame movie batch and
the same frames solved as one movie with the temporal term, the FFT variant
with TV / FGP 50 in FP64 and FP32 (with the FGP kernel's rate), and the
learned warm start at 256 x 256 on held-out skies.
Multi-GPU: every rank solves its own seeded lambda grid (no collective on
the data path), value = all ranks' solves / max-over-ranks time (weak
scaling).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "solves/s at 1e-6 rel. objective, chosen vs plain GPU MFISTA; NUFFT/FGP GB/s"
NX = 128
N_STATIONS, N_HOURS = 10, 180
GRID = (8, 8)
REL_OBJ = 1e-6
FSTAR_ITERS = 20000     # FP64 iterations behind F* (tests/golden/make_fstar.py)
MAXITER_CAP = 30000     # safety cap of the timed solves
FSTAR_FILE = os.path.join(ROOT, "tests", "golden", "lambda_grid_fstar.json")
L2_FLUSH_BYTES = 512 << 20
KERNEL_NAMES = ["nufft_interp", "nufft_spread", "nufft_rows_fwd", "nufft_cols_fwd", "nufft_cols_inv",
                "nufft_rows_inv", "prox_update"]
# launches of each operator kernel per MFISTA outer iteration without
# backtracking: forward at z and at the trial point, one adjoint
KERNEL_PER_ITER = [2, 1, 2, 2, 1, 1, 1]


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--plain-sample", type=int, default=8,
                    help="problems of the grid timed with the plain FP64 one-per-launch solver")
    ap.add_argument("--method", default="fp32", choices=["fp32", "fp64"],
                    help="chosen batched form: FP32 operators with FP64 defect correction, or FP64")
    return ap.parse_args()


def workload(seed):
    from sparseimaging_b200 import synth
    return synth.lambda_grid_problem(seed=seed, nx=NX, n_stations=N_STATIONS, n_hours=N_HOURS)


def max_over_ranks(values, world, dist=None, device=None):
    """Element-wise maximum of a list of floats over all ranks (one
    all-reduce; every rank must call it at the same point)."""
    if world <= 1:
        return [float(v) for v in values]
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def weak_rate(units_per_rank, world, seconds):
    """Whole-job rate when every rank processed `units_per_rank` in at most
    `seconds` (the slowest rank's time)."""
    return world * units_per_rank / seconds


DFT_FSTAR_FILE = os.path.join(ROOT, "tests", "golden", "dft_lambda_grid_fstar.json")


def dft_lambda_grid(si):
    """Side measurement of the DFT variant: the 64-problem lambda grid of a
    64x64 image with A 8000 x 4096 (tests/golden/make_dft_fstar.py), solved
    to F*(1 + 1e-6) in one batched call per form; solve time = the library's
    comp_time (set-up and the matrix upload excluded, the same for every
    form)."""
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import make_dft_fstar as D
    if not os.path.exists(DFT_FSTAR_FILE):
        return {"unavailable": "tests/golden/dft_lambda_grid_fstar.json missing"}
    fx = json.load(open(DFT_FSTAR_FILE))
    p, gmax, lip, grid = D.dft_workload()
    if abs(fx["gmax"] - gmax) > 1e-9 * gmax:
        return {"unavailable": "F* fixture does not match the DFT workload"}
    targets = np.array(fx["fstar"]) * (1 + REL_OBJ)
    out = {"workload": f"DFT {p.nx}x{p.nx}, A {p.A.shape[0]}x{p.A.shape[1]}, 64-problem lambda grid"}
    X64 = None
    for name, prec in (("fp64", si.FP64), ("bf16x6", si.BF16X6), ("bf16x3", si.BF16X3)):
        X, R = si.dft_batch(p.y, p.A, p.nx, p.nx, D.problems(grid, lip, 30000, targets), 0.0, precision=prec)
        if X64 is None:
            X64 = X
        secs = R[0]["comp_time"]
        out[name] = {"solves_per_s": round(len(grid) / secs, 3), "solve_s": round(secs, 4),
                     "reached_1e-6": int(sum(r["finalcost"] <= t for r, t in zip(R, targets))),
                     "max_iters": int(max(r["ITER"] for r in R)),
                     # the problems that stopped above their target: which lambda,
                     # how far from F*, after how many iterations (the stop rule
                     # with eps = 0 ends a solve whose objective no longer falls)
                     "not_reached": [{"problem": b, "lambda_l1": float(grid[b][0]), "lambda_tsv": float(grid[b][1]),
                                      "rel_gap_to_fstar": float(r["finalcost"] / fx["fstar"][b] - 1), "iters": int(r["ITER"])}
                                     for b, (r, t) in enumerate(zip(R, targets)) if r["finalcost"] > t]}
    out["speedup_bf16x6_vs_fp64"] = round(out["fp64"]["solve_s"] / out["bf16x6"]["solve_s"], 2)
    out["looe"] = dft_looe_side(si, p, X64, [float(lt) for _, lt in grid])
    return out


def dft_looe_side(si, p, X, lts):
    """Leave-one-out error (the reference's c/looe_lib.c) of the 64 FP64
    lambda-grid solutions: one mfista_dft_looe call (A upload included)
    against the oracle's numpy/LAPACK restatement on the host for every 4th
    solution (scaled by 4)."""
    from oracle import looe_oracle as O
    ns = [int(np.count_nonzero(x)) for x in X]
    t = time.perf_counter()
    m, sd, pos = si.dft_looe(p.y, p.A, X, p.nx, lambda_tsv=lts)
    gpu_s = time.perf_counter() - t
    sample = list(range(0, len(X), 4))
    t = time.perf_counter()
    worst = 0.0
    for b in sample:
        st, wm, _ = O.looe(p.y, p.A, X[b], p.nx, lts[b])
        if st and pos[b]:
            worst = max(worst, abs(m[b] - wm) / abs(wm))
    cpu_s = (time.perf_counter() - t) * len(X) / len(sample)
    return {"solutions": len(X), "active_pixels": {"min": min(ns), "mean": int(np.mean(ns)), "max": max(ns)},
            "gpu_s": round(gpu_s, 4), "hessian_positive": int(pos.sum()),
            "cpu_baseline": {"seconds": round(cpu_s, 3), "kind": "port", "cores": os.cpu_count(),
                             "sample": f"numpy/LAPACK restatement on {len(sample)} of {len(X)} solutions, x{len(X) // len(sample)}"},
            "speedup_vs_cpu": round(cpu_s / gpu_s, 1), "max_rel_diff_looe_m": worst}


def movie_batch(si):
    """Side measurement of the uneven batch: 48 movie frames (128x128, M per
    frame ~1400..11700, synth.movie_problem) as L1+TSV problems in one
    batched solve with the reference stop rule (eps 1e-6), FP64 and FP32
    forms; per-frame objective and image difference of FP32 vs FP64."""
    from sparseimaging_b200 import synth
    frames = synth.movie_problem()
    nx = frames[0].nx
    probs = []
    for f in frames:
        w2 = 1 / f.vis_std ** 2
        g0 = si.nufft_adjoint(f.u_dx, f.v_dy, nx, nx, f.vis_r * w2, f.vis_i * w2)
        lam = 1e-2 * float(np.abs(g0).max())
        lip = si.nufft_lipschitz(f.u_dx, f.v_dy, f.vis_std, nx, nx, iters=10)
        probs.append(dict(lambda_l1=lam, lambda_tsv=1e-3 * lam, cinit=lip, maxiter=5000, nonneg_flag=1))
    cat = lambda a: np.concatenate([getattr(f, a) for f in frames])
    off = np.concatenate([[0], np.cumsum([f.m for f in frames])]).astype(np.int32)
    geo = (cat("u_dx"), cat("v_dy"), cat("vis_r"), cat("vis_i"), cat("vis_std"), nx, nx)
    res = {}
    for name, prec in (("fp64", si.FP64), ("fp32", si.FP32)):
        X, R = si.nufft_batch(*geo, probs, 1e-6, pt_off=off, precision=prec)
        res[name] = (X, R)
    (X64, R64), (X32, R32) = res["fp64"], res["fp32"]
    dobj = [abs(a["finalcost"] - b["finalcost"]) / b["finalcost"] for a, b in zip(R32, R64)]
    dimg = [float(np.linalg.norm(X32[k] - X64[k]) / np.linalg.norm(X64[k])) for k in range(len(frames))]
    return {"workload": f"{len(frames)} frames {nx}x{nx}, M {min(f.m for f in frames)}..{max(f.m for f in frames)}, "
                        "one uneven batch, reference stop rule eps 1e-6",
            "fp64": {"frames_per_s": round(len(frames) / R64[0]["comp_time"], 3),
                     "mean_iters": float(np.mean([r["ITER"] for r in R64]))},
            "fp32": {"frames_per_s": round(len(frames) / R32[0]["comp_time"], 3),
                     "mean_iters": float(np.mean([r["ITER"] for r in R32]))},
            "fp32_vs_fp64_rel_objective": {"median": float(np.median(dobj)), "max": float(max(dobj))},
            "fp32_vs_fp64_rel_image": {"median": float(np.median(dimg)), "max": float(max(dimg))},
            "joint": _reported(movie_joint, si, geo, off, probs)}


def dropin_calls(si):
    """Cost of the drop-in entry outside the solve: mfista_imaging_core_nufft
    on config 0 (64 x 64, tests/golden/c0_nufft.npz, 300 iterations) called
    three times: building its solver (first call), reusing the kept solver
    with new visibilities (second call), and with the cache off; wall time
    of the call against the solve time it reports (comp_time)."""
    g = np.load(os.path.join(ROOT, "tests", "golden", "c0_nufft.npz"))
    args = lambda vr: (g["u"], g["v"], vr, g["vis_i"], g["vis_std"], 64, 64, 300, 1e-5, float(g["lam1"]), 0.0,
                       float(g["lamt"]), float(g["cinit"]))
    out = {"workload": "config 0: 64x64, M = %d, 300 iterations per call" % g["u"].size}
    si.release_cache()
    for name, vr, env in (("first_call", g["vis_r"], "1"), ("same_geometry", 0.9 * g["vis_r"], "1"),
                          ("cache_off", 0.9 * g["vis_r"], "0")):
        os.environ["MFISTA_DROPIN_CACHE"] = env
        t = time.perf_counter()
        _, r = si.imaging_core_nufft(*args(vr))
        wall = time.perf_counter() - t
        out[name] = {"wall_s": round(wall, 4), "solve_s": round(r["comp_time"], 4),
                     "outside_solve_s": round(wall - r["comp_time"], 4), "iters": r["ITER"]}
    os.environ.pop("MFISTA_DROPIN_CACHE", None)
    si.release_cache()
    return out


def _reported(fn, *args):
    """fn(*args), or its error as a short record (side measurements are
    reported, not required)."""
    try:
        return fn(*args)
    except Exception as e:
        return {"error": str(e)[:200]}


def movie_joint(si, geo, off, probs):
    """The same 48 frames solved as ONE movie (mfista_nufft_movie): one
    lambda (the frames' median), temporal weight lambda_t = 5 lambda in the
    FP64 and the FP32 form, and 0 (uncoupled frames under one step size),
    1000 iterations each; time per solve, the temporal term
    sum_b |x_b - x_{b+1}|^2 it leaves, the objective, and the FP32 form's
    objective and images against the FP64 form's."""
    lam = float(np.median([q["lambda_l1"] for q in probs]))
    lip = float(max(q["cinit"] for q in probs))
    out = {"frames": len(probs), "iterations": 1000, "lambda_t_over_lambda": 5.0}
    imgs = {}
    for name, lt, prec in (("coupled", 5.0 * lam, si.FP64), ("coupled_fp32", 5.0 * lam, si.FP32),
                           ("uncoupled", 0.0, si.FP64)):
        X, R, tcost = si.nufft_movie(*geo[:5], off, geo[5], geo[6], lam, 1e-3 * lam, lt, lip, 1000, 0.0,
                                     precision=prec)
        D = X[:-1] - X[1:]
        imgs[name] = X
        out[name] = {"solve_s": round(R[0]["comp_time"], 4),
                     "iterations_per_s": round(R[0]["ITER"] / R[0]["comp_time"], 1),
                     "temporal_sum": float(np.sum(D * D)),
                     "objective": float(sum(r["finalcost"] for r in R) + tcost)}
    a, b = out["coupled_fp32"]["objective"], out["coupled"]["objective"]
    out["coupled_fp32"]["rel_objective_vs_fp64"] = abs(a - b) / b
    out["coupled_fp32"]["rel_image_vs_fp64"] = float(np.linalg.norm(imgs["coupled_fp32"] - imgs["coupled"]) /
                                                     np.linalg.norm(imgs["coupled"]))
    return out


def fft_config1(si, hbm_gbs):
    """Side measurement of the gridded (FFT) variant with the L1+TV form and
    FGP 50 (128 x 128 image, 3000 cells with their Hermitian partners, the
    config-1 fixture tests/golden/c1_fft.npz): the plain FP64 solve and the
    FP32 form (FP32 FFTs and FGP stencils, FP64-corrected spectrum and FP64
    objective), 1000 iterations each, against the reference built with
    FGPITER 50 (tests/golden/c1_tv50_1000.npz); a 16-problem lambda grid of
    the same data in both forms; the FGP prox kernel alone (CUDA events)
    for 1, 16 and 64 problems per launch against the HBM peak."""
    g = np.load(os.path.join(ROOT, "tests", "golden", "c1_fft.npz"))
    ref = np.load(os.path.join(ROOT, "tests", "golden", "c1_tv50_1000.npz"))
    data = (g["u_idx"], g["v_idx"], g["y_r"], g["y_i"], g["noise"], 128, 128)
    lam1, ltv, cinit = float(g["lam1"]), float(g["lamtv"]), float(g["cinit"])
    out = {"workload": "FFT variant 128x128, 3000 cells (+ Hermitian partners), L1+TV, FGP 50, 1000 iterations"}
    ref_cost = float(ref["res"][16])
    for name, prec in (("fp64", si.FP64), ("fp32", si.FP32)):
        probs = [dict(lambda_l1=lam1, lambda_tv=ltv, cinit=cinit, maxiter=1000, nonneg_flag=1)]
        si.fft_batch(*data, probs, 0.0, fgp_iter=50, precision=prec)  # warm
        X, R = si.fft_batch(*data, probs, 0.0, fgp_iter=50, precision=prec)
        secs = R[0]["comp_time"]
        out[name] = {"solve_s": round(secs, 4), "solves_per_s": round(1.0 / secs, 3), "iters": R[0]["ITER"],
                     "rel_err_x_vs_reference": float(np.linalg.norm(X[0] - ref["x"]) / np.linalg.norm(ref["x"])),
                     "rel_err_cost_vs_reference": abs(R[0]["finalcost"] - ref_cost) / ref_cost}
    out["reference_envelope"] = {"x": float(ref["envelope_x"]), "cost": float(ref["envelope_cost"]),
                                 "note": "the reference's own change under a 1e-15 change of one visibility"}
    scales = np.logspace(-1, 1, 16)
    for name, prec in (("fp64", si.FP64), ("fp32", si.FP32)):
        probs = [dict(lambda_l1=lam1 * s_, lambda_tv=ltv * s_, cinit=cinit, maxiter=1000, nonneg_flag=1)
                 for s_ in scales]
        _, R = si.fft_batch(*data, probs, 0.0, fgp_iter=50, precision=prec)
        out[f"grid16_{name}"] = {"solve_s": round(R[0]["comp_time"], 4),
                                 "solves_per_s": round(16 / R[0]["comp_time"], 3)}
    out["grid16_speedup_fp32"] = round(out["grid16_fp64"]["solve_s"] / out["grid16_fp32"]["solve_s"], 2)
    fgp = {}
    for name, prec in (("fp64", si.FP64), ("fp32", si.FP32)):
        for B in (1, 16, 64):
            ms, by = si.fgp_profile(128, 128, B, 50, precision=prec, reps=20)
            fgp[f"{name}_b{B}"] = {"ms": round(ms, 5), "GB/s": round(by / ms / 1e6, 1),
                                   "frac_of_hbm": round(by / ms / 1e6 / hbm_gbs, 4) if hbm_gbs else None}
    out["fgp_kernel"] = fgp
    out["fgp_kernel_note"] = ("k_fgp: 50 FGP iterations of one prox per problem inside one launch (slabs in shared "
                              "memory, DSMEM halos); compulsory bytes 24 B/pixel per prox (z, dfdx in, xnew out)")
    return out


def warmstart_config4(si, n=32):
    """Side measurement of the learned warm start at the config-4 scale
    (256 x 256, M = 19998 shared coverage; sparseimaging_b200/data/
    unet_warmstart_256.npy, trained on 1024 FP64-solved skies): n held-out
    skies solved by FP64 MFISTA to F*(1 + 1e-6) from zero and from the
    network's start; iterations, solves/s (the network's prediction and the
    choice of start included) and image error against x* (4000 FP64
    iterations)."""
    from sparseimaging_b200 import warmstart
    net = warmstart.load(256)
    try:
        ev = warmstart.evaluate(net, list(range(90000, 90000 + n)), nx=256, batch=n, fstar_iters=4000)
    finally:
        net.close()
    out = {"workload": f"256x256, M = 19998 (12 stations x 303 hour angles), {n} held-out skies, "
                       "lambda_l1 = lambda_tsv = 1e-3 max|A^H W^2 y|"}
    out.update(ev["summary"])
    return out


def workload_name(nx, m, b):
    return f"NUFFT {nx}x{nx}, M={m}, {b}-problem lambda grid (8x8 log, 1e-4..1 of max|A^H y|)"


def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {}


class ClockSampler:
    """nvidia-smi samples during the timed region (clocks and throttle reasons)."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.index)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                mx.append(float(f[1]))
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if f[4 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def lam_grid(gmax):
    from sparseimaging_b200 import synth
    return synth.lambda_grid(gmax, GRID[0], GRID[1], 1e-4, 1.0)


def problems(grid, lip, maxiter, targets=None):
    return [dict(lambda_l1=float(a), lambda_tsv=float(b), cinit=float(lip), maxiter=int(maxiter), nonneg_flag=1,
                 target_cost=0.0 if targets is None else float(targets[i])) for i, (a, b) in enumerate(grid)]


# ---------------------------------------------------------------------------
# CPU reference (compiled reference C via oracle/_ref, run on host cores)
# ---------------------------------------------------------------------------

def _ref_worker(args):
    """Times `iters` MFISTA iterations of the reference on one problem."""
    (u, v, vr, vi, vs, nx, lam1, lamt, lip, iters) = args
    import os as _os
    sys.path.insert(0, ROOT)
    from oracle import ref_ctypes as R
    fd = _os.dup(1)
    dn = _os.open(_os.devnull, _os.O_WRONLY)
    _os.dup2(dn, 1)
    try:
        t = time.perf_counter()
        R.core_nufft(u, v, vr, vi, vs, nx, nx, iters, 0.0, lam1, 0.0, lamt, lip, nonneg_flag=1)
        dt = time.perf_counter() - t
    finally:
        _os.dup2(fd, 1)
        _os.close(fd)
        _os.close(dn)
    return dt


def reference_rate(p, grid, lip, iters_needed, cores=None, sample_iters=8):
    """Solves/s of the reference C on all host cores, from a bounded sample:
    every core runs `sample_iters` iterations of one grid problem; the
    per-iteration time times the iterations each problem needs (measured by
    the FP64 GPU solver, which follows the same trajectory) gives seconds
    per solve."""
    import multiprocessing as mp
    from oracle import ref_ctypes as R
    if not R.available():
        return None
    cores = cores or os.cpu_count() or 1
    picks = [int(i) for i in np.linspace(0, len(grid) - 1, cores)]
    jobs = [(p.u_dx, p.v_dy, p.vis_r, p.vis_i, p.vis_std, p.nx, float(grid[i][0]), float(grid[i][1]), lip,
             sample_iters) for i in picks]
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(cores) as pool:
        times = pool.map(_ref_worker, jobs)
    wall = time.perf_counter() - t0
    # one extra iteration of setup/summary per call is included in each time
    t_iter = float(np.mean(times)) / sample_iters
    mean_iters = float(np.mean(iters_needed))
    rate = cores / (t_iter * mean_iters)
    return dict(value=rate, unit="solves/s", cores=cores, kind="reference",
                sample=(f"reference C (oracle/_ref, shim FFT, 1 process per core) ran {sample_iters} iterations of "
                        f"{cores} grid problems; {t_iter * 1e3:.1f} ms/iteration x {mean_iters:.0f} mean iterations "
                        f"to 1e-6 rel. objective"),
                wall_s=wall, ms_per_iter=t_iter * 1e3)


def reference_full_solves(p, grid, lip, iters_needed, cores=None):
    """Complete reference solves on the host cores: each core runs one grid
    problem for the whole number of iterations it needs to reach its
    1e-6 target (about 1000 iterations, tens of seconds), all cores at
    once.  Returns the per-iteration time measured over those complete
    solves and the grid rate it implies (cores / (time per iteration x mean
    iterations of the grid))."""
    import multiprocessing as mp
    from oracle import ref_ctypes as R
    if not R.available():
        return None
    cores = cores or os.cpu_count() or 1
    it = np.asarray(iters_needed)
    mean_it = float(it.mean())
    # the problems whose iteration counts lie closest to the grid's mean
    picks = [int(i) for i in np.argsort(np.abs(it - mean_it))[:cores]]
    jobs = [(p.u_dx, p.v_dy, p.vis_r, p.vis_i, p.vis_std, p.nx, float(grid[i][0]), float(grid[i][1]), lip,
             int(it[i])) for i in picks]
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(len(jobs)) as pool:
        times = pool.map(_ref_worker, jobs)
    wall = time.perf_counter() - t0
    n_it = float(sum(int(it[i]) for i in picks))
    ms_iter = 1e3 * float(np.sum(times)) / n_it
    return dict(solves=len(jobs), iterations=[int(it[i]) for i in picks], wall_s=round(wall, 2),
                ms_per_iter=round(ms_iter, 3), solve_s_mean=round(float(np.mean(times)), 2),
                grid_rate=cores / (ms_iter * 1e-3 * mean_it))


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

def run_ours(args):
    import torch
    import torch.distributed as dist
    os.environ.setdefault("MFISTA_QUIET", "1")
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    torch.cuda.set_device(local)
    import sparseimaging_b200 as si
    si.set_device(local)
    dev = torch.device("cuda", local)

    p = workload(seed=7 + rank)
    nx, M = p.nx, p.m
    w2 = 1 / p.vis_std ** 2
    g0 = si.nufft_adjoint(p.u_dx, p.v_dy, nx, nx, p.vis_r * w2, p.vis_i * w2)
    gmax = float(np.abs(g0).max())
    lip = si.nufft_lipschitz(p.u_dx, p.v_dy, p.vis_std, nx, nx, iters=20)
    grid = lam_grid(gmax)
    B = len(grid)
    geo = (p.u_dx, p.v_dy, p.vis_r, p.vis_i, p.vis_std, nx, nx)

    # F*: converged FP64 objectives (fixture made by tests/golden/make_fstar.py
    # for exactly this workload; recomputed, untimed, if it does not match)
    fx = json.load(open(FSTAR_FILE)) if os.path.exists(FSTAR_FILE) else None
    xstar = None
    if fx and fx["nx"] == nx and fx["M"] == M and abs(fx["gmax"] - gmax) <= 1e-9 * gmax:
        fstar = np.array(fx["fstar"])
        fstar_src = f"fixture ({fx['iters']} FP64 iterations)"
        xf = os.path.join(ROOT, "tests", "golden", fx.get("xstar_file", ""))
        if fx.get("xstar_file") and os.path.exists(xf):
            xstar = np.load(xf)["xstar"].astype(np.float64)
    else:
        t = time.perf_counter()
        _, Rs = si.nufft_batch(*geo, problems(grid, lip, FSTAR_ITERS), 0.0, precision=si.FP64)
        fstar = np.array([r["finalcost"] for r in Rs])
        fstar_src = f"computed here ({FSTAR_ITERS} FP64 iterations, {time.perf_counter() - t:.0f} s, untimed)"
    targets = fstar * (1 + REL_OBJ)

    # chosen method: batched plan, device loop
    chosen_prec = si.FP32 if args.method == "fp32" else si.FP64
    plan = si.Plan(*geo, B, precision=chosen_prec)
    # launch shapes from the library's autotuner (untimed, once per plan)
    shapes, _ = plan.tune(reps=10)
    stream = torch.cuda.ExternalStream(plan.stream, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    probs = problems(grid, lip, MAXITER_CAP, targets)

    def one_step(timed):
        plan.set_problems(probs, 0.0)
        flush.fill_(1.0)                 # evict L2 between steps (outside the events)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        plan.run()
        e1.record(stream)
        X, R = plan.fetch(want_x=timed)
        return e0.elapsed_time(e1), X, R, plan.kernel_launches

    for _ in range(args.warmup):
        one_step(False)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    ms_steps, launches = [], 0
    X = R = None
    for _ in range(args.steps):
        ms, X, R, L = one_step(True)
        ms_steps.append(ms)
        launches += L
    torch.cuda.synchronize()
    clk = clocks.stop()
    total_ms = max_over_ranks([float(np.sum(ms_steps))], world, dist, dev)[0]
    value = weak_rate(B * args.steps, world, total_ms / 1e3)
    other_prec = si.FP64 if chosen_prec == si.FP32 else si.FP32
    t = time.perf_counter()
    Xo, Ro = si.nufft_batch(*geo, probs, 0.0, precision=other_prec)
    other_s = time.perf_counter() - t
    X64 = X if chosen_prec == si.FP64 else Xo

    def xstar_errors(X):
        """relative L2 distance of every non-zero solution to the converged
        FP64 image x* of the fixture"""
        if xstar is None:
            return None
        return np.array([float(np.linalg.norm(X[b] - xstar[b]) / np.linalg.norm(xstar[b]))
                         for b in range(B) if np.linalg.norm(xstar[b]) > 0])

    def quality(X, R):
        reached = np.array([r["finalcost"] <= t for r, t in zip(R, targets)])
        relobj = (np.array([r["finalcost"] for r in R]) - fstar) / fstar
        # relative image error where the FP64 solution is not the zero image;
        # problems whose FP64 solution is zero are counted apart
        nz = [b for b in range(B) if np.linalg.norm(X64[b]) > 0]
        xerr = [float(np.linalg.norm(X[b] - X64[b]) / np.linalg.norm(X64[b])) for b in nz] or [0.0]
        zero_abs = max([float(np.abs(X[b]).max()) for b in range(B) if b not in nz] or [0.0])
        q = {"reached_1e-6": int(reached.sum()), "of": B, "max_rel_obj": float(relobj.max()),
             "max_img_err_vs_fp64": float(max(xerr)), "median_img_err_vs_fp64": float(np.median(xerr)),
             "zero_solutions": B - len(nz), "max_abs_on_zero_solutions": zero_abs,
             "mean_iters": float(np.mean([r["ITER"] for r in R])), "max_iters": int(max(r["ITER"] for r in R))}
        ex = xstar_errors(X)
        if ex is not None:
            q["max_img_err_vs_xstar"] = float(ex.max())
            q["median_img_err_vs_xstar"] = float(np.median(ex))
        return q
    q_chosen = quality(X, R)
    q_other = quality(Xo, Ro)
    e_c, e_64 = xstar_errors(X), xstar_errors(X64)
    if e_c is not None:
        # the FP64 form's own distance to x* at the same objective tolerance:
        # the image is only determined to this level at F*(1 + 1e-6)
        q_chosen["img_err_ratio_vs_fp64_form"] = {"min": float((e_c / e_64).min()),
                                                  "max": float((e_c / e_64).max())}
        q_chosen["xstar"] = "converged FP64 images (tests/golden/lambda_grid_xstar.npz)"
    q_other["wall_s"] = other_s
    iters_fp64 = [r["ITER"] for r in (R if chosen_prec == si.FP64 else Ro)]

    # plain method: FP64, one problem per launch (plan of one), same targets
    sample = [int(i) for i in np.linspace(0, B - 1, max(1, min(args.plain_sample, B)))]
    plain_ms, iters64 = [], []
    pplan = si.Plan(*geo, 1, precision=si.FP64)
    pstream = torch.cuda.ExternalStream(pplan.stream, device=dev)
    for i in sample:
        pplan.set_problems([probs[i]], 0.0)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(pstream)
        pplan.run()
        e1.record(pstream)
        _, Rp = pplan.fetch(want_x=False)
        plain_ms.append(e0.elapsed_time(e1))
        iters64.append(Rp[0]["ITER"])
    plain_rate = 1e3 / float(np.mean(plain_ms))

    # end to end through the public API: host arrays in (pinned), results out
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
    h_geo = tuple(pin(a) for a in geo[:5])
    e2e_times = []
    for k in range(max(1, min(args.steps, 2))):
        torch.cuda.synchronize()
        t = time.perf_counter()
        Xe, Re = si.nufft_batch(*h_geo, nx, nx, probs, 0.0, precision=chosen_prec)
        e2e_times.append(time.perf_counter() - t)
    e2e_s = max_over_ranks([float(np.mean(e2e_times))], world, dist, dev)[0]
    e2e_rate = weak_rate(B, world, e2e_s)
    h2d = 5 * M * 8 + B * 48
    d2h = B * nx * nx * 8 + B * 144

    # roofline: each operator kernel timed alone on the plan's stream
    prof = []
    for k in range(7):
        ms, by = plan.profile(k, 20)
        prof.append((ms, by))
    share = [prof[k][0] * KERNEL_PER_ITER[k] for k in range(7)]
    dom = int(np.argmax(share))
    pk = peaks()
    hbm = pk.get("hbm_gbs")
    achieved = prof[dom][1] / (prof[dom][0] * 1e-3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        traffic = json.load(open(tpath)).get(KERNEL_NAMES[dom])
    roofline = {"bound": "hbm", "kernel": KERNEL_NAMES[dom], "achieved": round(achieved, 1),
                "peak": hbm if hbm else 6650.0, "unit": "GB/s",
                "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs)" if hbm else "fallback",
                "frac": round(achieved / (hbm if hbm else 6650.0), 4), "traffic": traffic,
                "bytes_per_launch": prof[dom][1], "ms_per_launch": prof[dom][0],
                "note": "batch working set (64 grids, 17 MB) is L2-resident: algorithmic bytes over HBM peak",
                "kernels": {KERNEL_NAMES[k]: {"ms": round(prof[k][0], 5), "GB/s": round(prof[k][1] / prof[k][0] / 1e6, 1)}
                            for k in range(7)}}
    plan.close()
    pplan.close()

    side = {}
    if rank == 0:  # side measurements of the other configurations (rank 0 only)
        for key, fn in (("dft_lambda_grid", dft_lambda_grid), ("movie_batch", movie_batch),
                        ("fft_tv_fgp50", lambda s_: fft_config1(s_, hbm)),
                        ("warmstart_config4", warmstart_config4), ("dropin_calls", dropin_calls)):
            try:
                side[key] = fn(si)
            except Exception as e:  # reported, not required
                side[key] = {"error": str(e)[:200]}

    cpu = None
    if rank == 0 and world == 1:
        try:
            cpu = reference_rate(p, grid, lip, iters_fp64)
            full = reference_full_solves(p, grid, lip, iters_fp64, cpu["cores"]) if cpu else None
            if full:
                # the reported rate comes from complete solves; the short
                # sample's figure stays beside it
                cpu["full_solves"] = full
                cpu["sample_short"] = cpu["sample"]
                cpu["value_short"] = cpu["value"]
                cpu["value"] = full["grid_rate"]
                cpu["sample"] = (f"reference C (oracle/_ref, project FFT shim: FFTW absent) ran {full['solves']} "
                                 f"complete solves, one per core, each to its problem's 1e-6 target "
                                 f"({min(full['iterations'])}-{max(full['iterations'])} iterations, "
                                 f"{full['ms_per_iter']:.1f} ms/iteration); rate = cores / (ms/iteration x mean "
                                 f"iterations of the grid)")
                cpu["fft"] = "project Stockham FFT shim (FFTW is not installed)"
        except Exception as e:  # the baseline is reported, not required
            cpu = {"value": None, "error": str(e)[:200]}

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 operators + f64 defect correction, f64 objective" if chosen_prec == si.FP32 else "f64",
            "data": "synthetic (seeded sky + uv coverage, rank-seeded)",
            "config": {"workload": workload_name(nx, M, B),
                       "method": ("batched, FP32 NUFFT/FFT with FP64 anchor correction" if chosen_prec == si.FP32 else "batched FP64") + ", device-resident CUDA-graph loop, per-problem stop at F*(1+1e-6)",
                       "l2": "flushed between steps (512 MB write)", "fstar": fstar_src,
                       "shapes": shapes,
                       "parallelism": f"replicas x{world}"},
            "quality": q_chosen, ("fp64_batched" if chosen_prec == si.FP32 else "fp32_batched"): q_other,
            "plain_fp64": {"solves_per_s": round(plain_rate, 3), "sample": len(sample),
                           "note": "FP64, one problem per launch (plan of one), same targets"},
            "speedup_vs_plain_fp64": round(value / world / plain_rate, 2),
            "e2e": {"value": round(e2e_rate, 3), "unit": "solves/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "api": "mfista_nufft_batch (host arrays, pinned)"},
            "roofline": roofline, "cpu_baseline": cpu, "gpu_launches": int(launches), "clocks": clk,
            "side": side,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_reference(args):
    """Reference arm: the reference C on the host cores (rank 0 only)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import ref_ctypes as R
    if not R.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built (make -C oracle)"}))
        return
    from oracle import mfista_oracle as O
    p = workload(seed=7)
    plan = O.NufftPlan(p.u_dx, p.v_dy, p.nx, p.nx)
    w = 1 / p.vis_std
    g0 = plan.adjoint(p.vis_r * w * w, p.vis_i * w * w)
    lip = O.lipschitz_nufft(plan, w, iters=20)
    grid = lam_grid(float(np.abs(g0).max()))
    fx = json.load(open(FSTAR_FILE)) if os.path.exists(FSTAR_FILE) else None
    if not fx:
        print(json.dumps({"impl": "reference", "unavailable": "tests/golden/lambda_grid_fstar.json missing"}))
        return
    iters = fx["iters_to_target_fp64"]
    steps = []
    for _ in range(args.warmup):
        reference_rate(p, grid, lip, iters, sample_iters=2)
    for _ in range(args.steps):
        steps.append(reference_rate(p, grid, lip, iters, sample_iters=4))
    v = float(np.mean([s["value"] for s in steps]))
    line = {"impl": "reference", "metric": METRIC, "value": round(v, 5), "unit": "solves/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded sky + uv coverage)",
            "config": {"workload": workload_name(p.nx, p.m, len(grid)),
                       "method": "reference C MFISTA (FFTW/BLAS stand-ins), one problem per process"},
            "cpu_baseline": {"value": round(v, 5), "unit": "solves/s", "cores": steps[0]["cores"],
                             "kind": "reference", "sample": steps[0]["sample"]},
            "e2e": {"value": round(v, 5), "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)



if __name__ == "__main__":
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)
