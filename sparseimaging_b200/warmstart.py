"""Learned warm start for the NUFFT solves (no counterpart in the reference).

A U-Net (csrc/unet.cu: 4 levels, 16-32-64-128 channels, BF16 weights, FP32
accumulation, trained on the GPU by the library's own kernels) maps the
dirty image A^H W^2 y and the dirty beam A^H W^2 1 of a problem to an
initial image.  MFISTA then runs from that image with the reference's own
stopping rule, which alone decides when it stops; per problem the start is used
only when its objective is below that of the zero image (zero init is the
fallback, `choose_starts`).

Input scaling: both maps are divided by the beam's peak (a unit point
source then has peak 1 in the dirty image), and the dirty image and the
target solution by the dirty image's peak, so the network sees O(1) values;
its output is scaled back.

    python -m sparseimaging_b200.warmstart --train   (on a GPU: makes the
        training set with the FP64 solver and writes WEIGHTS)
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import time

import numpy as np

from . import MfistaError, nufft_adjoint, synth
from . import lib as _lib_loader

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS = os.path.join(HERE, "data", "unet_warmstart_128.npy")
WEIGHTS_256 = os.path.join(HERE, "data", "unet_warmstart_256.npy")  # config 4 (config4_main)
TRAIN_LAMBDA = 1e-3  # training targets: lambda_l1 = lambda_tsv = 1e-3 max|A^H W^2 y|

_bound = False


def _lib():
    global _bound
    L = _lib_loader()
    if not _bound:
        vp, fp = C.c_void_p, C.POINTER(C.c_float)
        L.mfista_unet_create.restype = vp
        L.mfista_unet_create.argtypes = [C.c_int, C.c_int, C.c_int]
        L.mfista_unet_destroy.restype = None
        L.mfista_unet_destroy.argtypes = [vp]
        L.mfista_unet_param_count.restype = C.c_long
        L.mfista_unet_param_count.argtypes = [vp]
        L.mfista_unet_get_params.restype = C.c_int
        L.mfista_unet_get_params.argtypes = [vp, fp]
        L.mfista_unet_set_params.restype = C.c_int
        L.mfista_unet_set_params.argtypes = [vp, fp]
        L.mfista_unet_forward.restype = C.c_int
        L.mfista_unet_forward.argtypes = [vp, fp, C.c_int, fp]
        L.mfista_unet_grad.restype = C.c_int
        L.mfista_unet_grad.argtypes = [vp, fp, fp, C.c_int, fp, fp]
        L.mfista_unet_train_step.restype = C.c_int
        L.mfista_unet_train_step.argtypes = [vp, fp, fp, C.c_int, C.c_float, fp]
        L.mfista_unet_last_status.restype = C.c_int
        L.mfista_unet_last_error.restype = C.c_char_p
        _bound = True
    return L


def _f(a):
    return np.ascontiguousarray(a, np.float32)


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _ok(st):
    if st != 0:
        raise MfistaError(st, _lib().mfista_unet_last_error().decode())


class UNet:
    """The GPU U-Net: forward, gradients and Adam steps."""

    def __init__(self, H, W, batch_max=8):
        L = _lib()
        self.H, self.W, self.batch_max = H, W, batch_max
        self.h = L.mfista_unet_create(H, W, batch_max)
        if not self.h:
            _ok(L.mfista_unet_last_status() or 1)
        self.n = int(L.mfista_unet_param_count(self.h))

    def params(self):
        out = np.zeros(self.n, np.float32)
        _ok(_lib().mfista_unet_get_params(self.h, _fp(out)))
        return out

    def set_params(self, p):
        p = _f(p)
        if p.size != self.n:
            raise ValueError(f"expected {self.n} parameters, got {p.size}")
        _ok(_lib().mfista_unet_set_params(self.h, _fp(p)))

    def forward(self, x):
        """Initial images [n][H][W] (clamped >= 0) for inputs [n][2][H][W]."""
        x = _f(x).reshape(-1, 2, self.H, self.W)
        out = np.zeros((x.shape[0], self.H, self.W), np.float32)
        for i in range(0, x.shape[0], self.batch_max):
            xb = np.ascontiguousarray(x[i:i + self.batch_max])
            ob = np.zeros((xb.shape[0], self.H, self.W), np.float32)
            _ok(_lib().mfista_unet_forward(self.h, _fp(xb), xb.shape[0], _fp(ob)))
            out[i:i + xb.shape[0]] = ob
        return out

    def grad(self, x, t):
        x, t = _f(x), _f(t)
        loss = C.c_float(0)
        g = np.zeros(self.n, np.float32)
        _ok(_lib().mfista_unet_grad(self.h, _fp(x), _fp(t), x.shape[0], C.byref(loss), _fp(g)))
        return float(loss.value), g

    def train_step(self, x, t, lr):
        x, t = _f(x), _f(t)
        loss = C.c_float(0)
        _ok(_lib().mfista_unet_train_step(self.h, _fp(x), _fp(t), x.shape[0], lr, C.byref(loss)))
        return float(loss.value)

    def close(self):
        if getattr(self, "h", None):
            _lib().mfista_unet_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


def dirty_inputs(u_dx, v_dy, vis_r, vis_i, vis_std, nx):
    """(network input [2][nx][nx], scale): dirty image and dirty beam over
    the beam's peak, the image also over its own peak (= scale)."""
    w2 = 1.0 / np.asarray(vis_std, np.float64) ** 2
    dirty = nufft_adjoint(u_dx, v_dy, nx, nx, np.asarray(vis_r) * w2, np.asarray(vis_i) * w2)
    beam = nufft_adjoint(u_dx, v_dy, nx, nx, w2, np.zeros_like(w2))
    peak = beam.max()
    dirty, beam = dirty / peak, beam / peak
    scale = max(float(np.abs(dirty).max()), 1e-30)
    x = np.stack([dirty.reshape(nx, nx) / scale, beam.reshape(nx, nx)])
    return x.astype(np.float32), scale


def predict(net, u_dx, v_dy, vis_r, vis_i, vis_std, nx):
    """Initial image [nx*nx] (>= 0) for one problem."""
    x, scale = dirty_inputs(u_dx, v_dy, vis_r, vis_i, vis_std, nx)
    return net.forward(x[None])[0].reshape(-1).astype(np.float64) * scale


def choose_starts(geo, problems, x_warm, precision=None):
    """Per problem, x_warm where its objective is below the zero image's,
    else zero (each objective from one evaluation at the start, no
    iteration).  geo = (u, v, vis_r, vis_i, vis_std, nx, ny).  Returns
    ([B * N] starts, [B] bool used)."""
    from . import FP64, nufft_batch
    B = len(problems)
    at0 = [dict(p, maxiter=0, target_cost=0.0) for p in problems]
    prec = FP64 if precision is None else precision
    _, Rw = nufft_batch(*geo, at0, 0.0, xinit=np.tile(x_warm, B), precision=prec)
    _, Rz = nufft_batch(*geo, at0, 0.0, precision=prec)
    used = np.array([rw["finalcost"] < rz["finalcost"] for rw, rz in zip(Rw, Rz)])
    starts = np.where(used[:, None], np.asarray(x_warm)[None, :], 0.0).reshape(-1)
    return starts, used


def load(nx=128, batch_max=8, path=None):
    """The trained network (raises if the weights file is absent): the
    128 x 128 lambda-grid weights, or for nx = 256 the config-4 weights."""
    net = UNet(nx, nx, batch_max)
    net.set_params(np.load(path or (WEIGHTS_256 if nx == 256 else WEIGHTS)))
    return net


# ---------------------------------------------------------------------------
# training set: seeded synthetic skies solved by the FP64 solver
# ---------------------------------------------------------------------------
def training_problem(seed, nx=128):
    """A seeded sky and uv coverage shaped like the benchmark's (8-12
    stations, 180 hour angles), different per seed."""
    rng = np.random.default_rng(seed)
    return synth.lambda_grid_problem(seed=seed, nx=nx, n_stations=int(rng.integers(8, 13)), n_hours=180)


_C4 = {}


def config4_geometry(nx=256):
    """The uv coverage of the learned-warm-start configuration, shared by
    all its skies: 12 stations (seeded) over 303 hour angles, 66 baselines,
    M = 19998 points; with the Lipschitz constant of A^H A (unit weights),
    and the network's dirty-beam channel (the beam over its peak), which a
    shared coverage with uniform weights makes the same for every sky."""
    if nx not in _C4:
        from . import nufft_lipschitz
        u, v = synth.earth_rotation_uv(12, 303, seed=4)
        u_dx, v_dy = synth.scale_uv_to_radians(u, v, nx, synth.safe_kmax(nx))
        ones = np.ones(u_dx.size)
        lip1 = nufft_lipschitz(u_dx, v_dy, ones, nx, nx, iters=30)
        beam = nufft_adjoint(u_dx, v_dy, nx, nx, ones, np.zeros_like(ones))
        _C4[nx] = (u_dx, v_dy, lip1, (beam / beam.max()).reshape(nx, nx))
    return _C4[nx]


def config4_problem(seed, nx=256):
    """A config-4 problem: the seeded training sky (3-12 blobs, sigma 1-10
    px, a ring or crescent with probability 0.5, flux 1) seen through the
    shared coverage (config4_geometry), visibilities from this library's
    FP64 NUFFT (~1e-12 of the exact DFT) plus complex noise of 1 % of
    max|V|."""
    from . import nufft_forward
    u_dx, v_dy, _, _ = config4_geometry(nx)
    sky = synth.sky_training(nx, seed)
    fr, fi = nufft_forward(u_dx, v_dy, nx, nx, sky.ravel())
    vis = fr + 1j * fi
    sigma = 0.01 * float(np.abs(vis).max())
    rng = np.random.default_rng(seed + 7777)
    vis = vis + sigma * (rng.standard_normal(vis.size) + 1j * rng.standard_normal(vis.size))
    return synth.NufftProblem(u_dx, v_dy, vis.real.copy(), vis.imag.copy(), np.full(vis.size, sigma), nx, nx, sky)


def _batch_setup(ps, nx, lam_rel):
    """Network inputs, scales and MFISTA parameters of config-4 problems
    (shared coverage, uniform weights per problem: cinit = L_unit / sigma^2)."""
    _, _, lip1, beam = config4_geometry(nx)
    X, scales, problems = [], [], []
    for p in ps:
        sig = float(p.vis_std[0])
        w2 = 1.0 / sig ** 2
        g0 = nufft_adjoint(p.u_dx, p.v_dy, nx, nx, p.vis_r * w2, p.vis_i * w2)
        lam = lam_rel * float(np.abs(g0).max())
        # dirty image over the beam's peak (M w^2), then over its own peak
        dirty = g0.reshape(nx, nx) / (p.m * w2)
        scale = max(float(np.abs(dirty).max()), 1e-30)
        X.append(np.stack([dirty / scale, beam]).astype(np.float32))
        scales.append(scale)
        problems.append(dict(lambda_l1=lam, lambda_tsv=lam, cinit=lip1 * w2, nonneg_flag=1))
    cat = lambda f: np.concatenate([getattr(p, f) for p in ps])
    off = np.concatenate([[0], np.cumsum([p.m for p in ps])]).astype(np.int32)
    geo = (cat("u_dx"), cat("v_dy"), cat("vis_r"), cat("vis_i"), cat("vis_std"), nx, nx)
    return X, scales, problems, geo, off


def make_training_set(seeds, nx=128, iters=1500, batch=32, lam_rel=TRAIN_LAMBDA, problem=None, eps=1e-7):
    """(inputs [n][2][nx][nx], targets [n][nx][nx]) for the given seeds: the
    targets are FP64 MFISTA solutions (at most `iters` iterations, the
    reference's stopping rule with `eps`) at
    lambda_l1 = lambda_tsv = lam_rel * max|A^H W^2 y|."""
    from . import FP64, nufft_batch, nufft_lipschitz
    if problem is not None:
        X, T = [], []
        for i in range(0, len(seeds), batch):
            ps = [problem(s) for s in seeds[i:i + batch]]
            Xb, scales, problems, geo, off = _batch_setup(ps, nx, lam_rel)
            for q in problems:
                q["maxiter"] = iters
            Xs, _ = nufft_batch(*geo, problems, eps, pt_off=off, precision=FP64)
            X += Xb
            T += [(Xs[k].reshape(nx, nx) / sc).astype(np.float32) for k, sc in enumerate(scales)]
        return np.stack(X), np.stack(T)
    X, T = [], []
    for i in range(0, len(seeds), batch):
        ps = [training_problem(s, nx) for s in seeds[i:i + batch]]
        cat = lambda f: np.concatenate([getattr(p, f) for p in ps])
        off = np.concatenate([[0], np.cumsum([p.m for p in ps])]).astype(np.int32)
        problems, scales = [], []
        for p in ps:
            x, scale = dirty_inputs(p.u_dx, p.v_dy, p.vis_r, p.vis_i, p.vis_std, nx)
            w2 = 1 / p.vis_std ** 2
            g0 = nufft_adjoint(p.u_dx, p.v_dy, nx, nx, p.vis_r * w2, p.vis_i * w2)
            lam = lam_rel * float(np.abs(g0).max())
            lip = nufft_lipschitz(p.u_dx, p.v_dy, p.vis_std, nx, nx, iters=20)
            problems.append(dict(lambda_l1=lam, lambda_tsv=lam, cinit=lip, maxiter=iters, nonneg_flag=1))
            X.append(x)
            scales.append(scale)
        Xs, _ = nufft_batch(cat("u_dx"), cat("v_dy"), cat("vis_r"), cat("vis_i"), cat("vis_std"), nx, nx,
                            problems, 1e-7, pt_off=off, precision=FP64)
        for k, s in enumerate(scales):
            T.append((Xs[k].reshape(nx, nx) / s).astype(np.float32))
    return np.stack(X), np.stack(T)


def train(X, T, steps=400, batch=8, lr=1e-3, seed=0, net=None, log=None):
    """Adam on random minibatches (learning rate / 10 for the last 20 %);
    returns the network and the loss history."""
    net = net or UNet(X.shape[-2], X.shape[-1], batch)
    rng = np.random.default_rng(seed)
    hist = []
    for s in range(steps):
        idx = rng.choice(X.shape[0], size=min(batch, X.shape[0]), replace=False)
        hist.append(net.train_step(X[idx], T[idx], lr * (0.1 if s >= int(0.8 * steps) else 1.0)))
        if log and (s % 100 == 0 or s == steps - 1):
            log(f"step {s} loss {hist[-1]:.4g}")
    return net, hist


def evaluate(net, seeds, nx=256, batch=64, lam_rel=TRAIN_LAMBDA, fstar_iters=6000, precision=None,
             problem=None):
    """Held-out evaluation: per seed, F* and x* from a long FP64 solve
    (`fstar_iters` iterations, stopping rule off), then MFISTA to
    F*(1 + 1e-6) from zero and from the network's start (where its objective
    is below the zero image's, choose_starts).  Returns per-problem
    iterations, batch solve times and relative image errors against x*."""
    from . import FP64, nufft_batch
    problem = problem or config4_problem
    prec = FP64 if precision is None else precision
    out = {"iters_zero": [], "iters_warm": [], "err_zero": [], "err_warm": [], "used": [], "s_zero": 0.0,
           "s_warm": 0.0, "s_predict": 0.0, "reached_zero": 0, "reached_warm": 0}
    for i in range(0, len(seeds), batch):
        ps = [problem(s) for s in seeds[i:i + batch]]
        X, scales, problems, geo, off = _batch_setup(ps, nx, lam_rel)
        long = [dict(q, maxiter=fstar_iters) for q in problems]
        Xs, Rs = nufft_batch(*geo, long, 0.0, pt_off=off, precision=FP64)
        targets = [r["finalcost"] * (1 + 1e-6) for r in Rs]
        timed = [dict(q, maxiter=fstar_iters, target_cost=t) for q, t in zip(problems, targets)]
        t0 = time.perf_counter()
        Xz, Rz = nufft_batch(*geo, timed, 0.0, pt_off=off, precision=prec)
        out["s_zero"] += time.perf_counter() - t0
        t0 = time.perf_counter()
        pred = net.forward(np.stack(X))
        x0 = np.concatenate([pred[k].reshape(-1).astype(np.float64) * sc for k, sc in enumerate(scales)])
        # per problem, the start whose objective is lower (one evaluation each)
        at0 = [dict(q, maxiter=0, target_cost=0.0) for q in problems]
        _, Rw0 = nufft_batch(*geo, at0, 0.0, pt_off=off, precision=prec, xinit=x0)
        _, Rz0 = nufft_batch(*geo, at0, 0.0, pt_off=off, precision=prec)
        used = np.array([a["finalcost"] < b["finalcost"] for a, b in zip(Rw0, Rz0)])
        starts = np.where(used[:, None], x0.reshape(len(ps), -1), 0.0).reshape(-1)
        out["s_predict"] += time.perf_counter() - t0
        t0 = time.perf_counter()
        Xw, Rw = nufft_batch(*geo, timed, 0.0, pt_off=off, precision=prec, xinit=starts)
        out["s_warm"] += time.perf_counter() - t0
        for k in range(len(ps)):
            nrm = max(np.linalg.norm(Xs[k]), 1e-300)
            out["err_zero"].append(float(np.linalg.norm(Xz[k] - Xs[k]) / nrm))
            out["err_warm"].append(float(np.linalg.norm(Xw[k] - Xs[k]) / nrm))
        out["iters_zero"] += [r["ITER"] for r in Rz]
        out["iters_warm"] += [r["ITER"] for r in Rw]
        out["reached_zero"] += int(sum(r["finalcost"] <= t for r, t in zip(Rz, targets)))
        out["reached_warm"] += int(sum(r["finalcost"] <= t for r, t in zip(Rw, targets)))
        out["used"] += used.tolist()
    n = len(out["iters_zero"])
    out["summary"] = {
        "problems": n, "used_start": int(sum(out["used"])),
        "mean_iters_zero": float(np.mean(out["iters_zero"])), "mean_iters_warm": float(np.mean(out["iters_warm"])),
        "median_iters_zero": float(np.median(out["iters_zero"])),
        "median_iters_warm": float(np.median(out["iters_warm"])),
        "solves_per_s_zero": n / out["s_zero"], "solves_per_s_warm": n / (out["s_warm"] + out["s_predict"]),
        "median_img_err_zero": float(np.median(out["err_zero"])),
        "median_img_err_warm": float(np.median(out["err_warm"])),
        "reached_zero": out["reached_zero"], "reached_warm": out["reached_warm"]}
    return out


def config4_main(n_train, n_eval, steps, out_weights, out_json, train_iters=5000):
    """Config 4 end to end on one GPU: training set (FP64 solves, reference
    stopping rule at eps 1e-6), training, held-out evaluation."""
    t0 = time.time()
    seeds_train = list(range(20000, 20000 + n_train))
    seeds_eval = list(range(90000, 90000 + n_eval))
    X, T = make_training_set(seeds_train, nx=256, iters=train_iters, batch=64, problem=config4_problem, eps=1e-6)
    t1 = time.time()
    net, hist = train(X, T, steps=steps, batch=8, log=print)
    t2 = time.time()
    os.makedirs(os.path.dirname(os.path.abspath(out_weights)), exist_ok=True)
    np.save(out_weights, net.params())
    ev = evaluate(net, seeds_eval, nx=256)
    t3 = time.time()
    res = {"config": "256x256, M = 19998 (12 stations x 303 hour angles), lambda_l1 = lambda_tsv = "
                     f"{TRAIN_LAMBDA} max|A^H W^2 y|, targets: FP64 MFISTA to eps 1e-6",
           "n_train": n_train, "n_eval": n_eval, "steps": steps, "data_s": t1 - t0, "train_s": t2 - t1,
           "eval_s": t3 - t2, "loss_first": hist[0], "loss_last": float(np.mean(hist[-50:])),
           "eval": ev["summary"],
           "per_problem": {k: ev[k] for k in ("iters_zero", "iters_warm", "err_zero", "err_warm", "used")}}
    json.dump(res, open(out_json, "w"), indent=1)
    print(json.dumps({k: v for k, v in res.items() if k != "per_problem"}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", action="store_true")
    ap.add_argument("--n-train", type=int, default=256)
    ap.add_argument("--steps", type=int, default=1500)
    ap.add_argument("--out", default=WEIGHTS)
    ap.add_argument("--iters", type=int, default=1500, help="FP64 MFISTA iterations per training target")
    ap.add_argument("--lam", type=float, default=TRAIN_LAMBDA, help="training lambdas relative to max|A^H W^2 y|")
    ap.add_argument("--config4", action="store_true",
                    help="256x256 / M = 19998 configuration: training set, training and held-out evaluation")
    ap.add_argument("--n-eval", type=int, default=256)
    ap.add_argument("--json", default="warmstart_config4.json")
    a = ap.parse_args()
    os.environ.setdefault("MFISTA_QUIET", "1")
    if a.config4:
        out = a.out if a.out != WEIGHTS else WEIGHTS_256
        config4_main(a.n_train, a.n_eval, a.steps, out, a.json)
        return
    if not a.train:
        ap.print_help()
        return
    t0 = time.time()
    X, T = make_training_set(list(range(1000, 1000 + a.n_train)), iters=a.iters, lam_rel=a.lam)
    t1 = time.time()
    net, hist = train(X, T, steps=a.steps, log=print)
    t2 = time.time()
    os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
    np.save(a.out, net.params())
    print(json.dumps({"n_train": a.n_train, "steps": a.steps, "iters": a.iters, "lam": a.lam,
                      "data_s": t1 - t0, "train_s": t2 - t1,
                      "loss_first": hist[0], "loss_last": float(np.mean(hist[-50:]))}))


if __name__ == "__main__":
    main()
