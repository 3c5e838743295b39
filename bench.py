"""Benchmark: ms per fractional step of the 1,004,000-node lid-driven cavity.

Workload (the plain-FP64 single-GPU configuration): unit-square cavity,
1000 x 1000 interior nodes at ((i+1/2)h, (j+1/2)h) jittered by +/-0.2h
(Philox seed 20261203) plus 4000 boundary nodes; PHS r^3 with a degree-3
polynomial, 20-node stencils; operators ELL FP64 width 20; pressure by BiCGSTAB
with the smoothed-aggregation multigrid preconditioner to ||r||/||b|| <= 1e-8;
Re = 100 (rho 1, mu 0.01), Adams-Bashforth 2; dt from the reference's calc_dt
rule with Courant 0.25 (the configured dt = 1e-3 is explicitly unstable on
this cloud; dt is rounded to 6 significant digits so that both arms step with
the same value).  A "step" is one FRACTIONAL_STEP_1 timestep, graph-launched.

`value` (and the reference arm's): the flow starts from rest, runs `--warmup`
untimed steps, then `--steps` timed ones, each pressure solve from the previous
pressure (the reference's solveWithGuess(rhs, p_old)) to 1e-8.  The variants
(FP32 multigrid storage, FP32 Krylov with FP64 refinement, extrapolated,
projected and learned initial guesses, learned + FP32 multigrid as
`learned_mixed`) are timed after `--spinup` untimed steps from rest (100, the
configuration's run length), during which the learned guess records its
training samples and after which it is trained, against a plain FP64 run over
the same steps (`variants.plain_fp64`).

Printed (rank 0, one JSON line): `value`, the variants, the end-to-end ms/step
through mp_fs1_single_timestep with pinned host buffers, the SpMV roofline, the
CPU oracle baseline, the batched uneven stencils, the 3D mixed-precision cube
(2,195,456 nodes, per-field error against FP64) and the learned-guess channel
(1,004,010 nodes, network trained on 500 plain-solver steps, each initial guess
timed from the same state).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--nx NX]
"""
from __future__ import annotations

import argparse
import json
import os
import re
import signal
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

FALLBACK_HBM_GBS = 6650.0
METRIC = "ms/fractional-step at 1M pts (learned+mixed vs plain FP64 GPU); SpMV HBM GB/s"
# pressure-solve iterations per step allowed to the reference's BiCGSTAB + ILUT in the
# reference arm: it does not reach 1e-8 on the 1M-node cavity (relres 1e-3 to 0.3 after
# 1000 iterations), so it runs to this limit and reports the residual it reached
REF_MAXIT = 100


def bench_dt(dt: float) -> float:
    """calc_dt's step rounded to 6 significant digits: both arms compute the
    eigenvalues independently (GPU Arnoldi / ARPACK, agreeing to ~1e-10) and step
    with the same value."""
    return float(f"{dt:.6g}")


def bench_config(nx, nv, K, dt, courant):
    """The workload, identical in both arms."""
    return {"workload": f"cavity_2d {nx}x{nx} jittered + {4 * nx} boundary = {nv} nodes, "
                        "FRACTIONAL_STEP_1 (AB2), pressure solve from the previous pressure "
                        "to relres 1e-8, steps from rest",
            "nodes": nv, "stencil": K, "phs": 3, "poly_deg": 3, "dt": dt, "courant": courant,
            "re": 100, "temporal_order": 2, "start": "rest",
            "l2": f"one ELL operator {nv * (12 * K + 16) / 1e6:.0f} MB, four per step plus the "
                  "solver's; 126 MB of L2"}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nx", type=int, default=1000)
    ap.add_argument("--courant", type=float, default=0.25)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--no-graph", action="store_true",
                    help="launch the step's kernels one by one instead of as a CUDA graph")
    ap.add_argument("--spinup", type=int, default=100,
                    help="untimed timesteps from rest before the timed ones (the 100 steps of "
                         "the 1M-node configuration); the learned guess trains on their solves")
    ap.add_argument("--samples", type=int, default=16384,
                    help="nodes whose features and solved increments are recorded per step")
    ap.add_argument("--epochs", type=int, default=10)
    ap.add_argument("--batched", type=int, default=4_000_000,
                    help="independent uneven stencil systems per dimension in the batched "
                         "weights measurement (0 skips it)")
    ap.add_argument("--no-cube", action="store_true",
                    help="skip the 3D mixed-precision cube (2,195,456 nodes)")
    ap.add_argument("--cube-n", type=int, default=128)
    ap.add_argument("--integrator-steps", type=int, default=3,
                    help="timed steps of each other time integrator at the headline size (0: skip)")
    ap.add_argument("--cube-spinup", type=int, default=10)
    ap.add_argument("--no-channel", action="store_true",
                    help="skip the learned-guess channel (1,004,010 nodes)")
    ap.add_argument("--channel-h", type=float, default=2.828e-3)
    ap.add_argument("--channel-train-steps", type=int, default=500)
    ap.add_argument("--channel-samples", type=int, default=4096)
    ap.add_argument("--inner-tol", type=float, default=1e-3,
                    help="mixed precision: relative reduction of each FP32 refinement solve")
    ap.add_argument("--profile", default=None,
                    choices=["steps", "spmv", "stencil", "cloud", "sis", "fsf", "train"],
                    help="set up, warm up, then run `--steps` steps (SpMV launches, stencil-weight "
                         "computations, cloud builds, semi-implicit or Fourier-z steps, training "
                         "epochs) inside a profiler capture range and exit (for ncu "
                         "--profile-from-start off)")
    ap.add_argument("--variant", default="plain",
                    choices=["plain", "mg32", "extrapolated_mg32", "projected_mg32",
                             "learned_mg32"],
                    help="solver configuration of --profile steps")
    return ap.parse_args()


def dist_setup(args=None, timeout_s: int = 120):
    """One process per GPU (torchrun env).  The replicas share no data: the process
    group carries only the start barrier and the max-over-ranks of the timings
    (NCCL on GPUs, gloo where there is no GPU)."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
        pg = dist
    return ws, rank, local, pg


def barrier(pg):
    if pg is not None:
        pg.barrier()


def max_over_ranks(pg, v: float) -> float:
    if pg is None:
        return v
    import torch
    dev = "cuda" if torch.cuda.is_available() and pg.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region.

    The sampler starts before the region and the region starts only once its first
    sample is written; the samples counted are those written between the region's
    start and end (every 50 ms).  A region shorter than the interval keeps the first
    sample after it and says so (`after_region`)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    INTERVAL_MS = 50

    def __init__(self, index: int):
        self.index = index
        self.p = None
        self.path = os.path.join(tempfile.gettempdir(), f"memphys_clocks_{os.getpid()}_{index}.csv")
        self.n0 = self.n1 = 0
        self.after = False

    def _lines(self):
        try:
            with open(self.path) as f:
                return [ln for ln in f if ln.count(",") >= 8]
        except OSError:
            return []

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits",
                                       "-lms", str(self.INTERVAL_MS)],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
            t_end = time.time() + 5.0
            while not self._lines() and time.time() < t_end and self.p.poll() is None:
                time.sleep(0.01)
            self.n0 = len(self._lines())
        except Exception:
            self.p = None
        return self

    def __exit__(self, *exc):
        if self.p is not None:
            self.n1 = len(self._lines())
            if self.n1 <= self.n0:  # region shorter than the interval: the next sample
                t_end = time.time() + 1.0
                while len(self._lines()) <= self.n0 and time.time() < t_end:
                    time.sleep(0.005)
                self.n1 = min(len(self._lines()), self.n0 + 1)
                self.after = True
            self.p.send_signal(signal.SIGTERM)
            try:
                self.p.wait(timeout=5)
            except Exception:
                self.p.kill()
            self.f.close()
        return False

    def summary(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        rows = [[x.strip() for x in ln.split(",")] for ln in self._lines()[self.n0:self.n1]]
        try:
            os.remove(self.path)
        except OSError:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k] == "Active"})
        out = {"sm_mhz": float(np.median(sm)) if sm else None,
               "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows),
               "interval_ms": self.INTERVAL_MS}
        if self.after:
            out["after_region"] = True
        return out


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        j = json.load(open(p))
        return float(j["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def profile_traffic():
    """dram bytes per SpMV launch from the committed ncu summary, if present."""
    p = os.path.join(ROOT, "profiles", "spmv_fp64_cavity1m.md")
    try:
        m = re.search(r"traffic_bytes_per_launch:\s*([0-9.eE+]+)", open(p).read())
        return float(m.group(1)) if m else None
    except Exception:
        return None


# ----------------------------------------------------------------- our arm
def run_ours(args, ws, rank, local, pg):
    from memphys_b200 import capi, clouds, meshless
    L = capi.lib()
    capi.check(L.mp_set_device(local), "mp_set_device")
    capi.device_info()
    nx = args.nx
    cl = clouds.cavity_2d(nx)
    nv = cl.nv
    prm = meshless.PARAMETERS(solver_type="cuda_bicgstab_amg", solver_tolerance=1e-8, n_iter=2000)
    prm.rho, prm.mu = 1.0, 0.01
    pts = meshless.POINTS(cl)
    t0 = time.time()
    cld = meshless.CLOUD(pts, prm, compute_cond=False)
    t_cloud = time.time() - t0
    prm.dt = bench_dt(meshless.calc_dt(cld, 1.0, 1.0, 0.0, prm.mu / prm.rho, args.courant))

    def make(**cfg):
        return meshless.FRACTIONAL_STEP_1(pts, cld, prm, cl.u_dirichlet, cl.v_dirichlet,
                                          cl.p_dirichlet, 2, use_graph=not args.no_graph, **cfg)

    stream = capi.Stream()
    vel0 = [cl.vel_bc[0].copy(), cl.vel_bc[1].copy()]
    t0 = time.time()
    fs = make()
    t_setup = time.time() - t0
    ns = fs.system_size
    p0 = np.zeros(ns)
    if args.profile:
        return profile_range(args, cl, cld, make, fs, vel0, p0, stream, pts, prm)
    import ctypes as C

    # headline: plain FP64 from rest, `--warmup` untimed steps, `--steps` timed steps
    # (the steps the reference arm times)
    fs.set_state(vel0, p0, 0)
    for _ in range(args.warmup):
        fs.step(1, stream.handle)
    stream.sync()
    barrier(pg)
    stream.sync()
    with Clocks(local) as clk:
        with capi.Timer(stream.handle) as tm:
            for _ in range(args.steps):
                fs.step(1, stream.handle)
    clocks = clk.summary()
    ms64_max = max_over_ranks(pg, tm.ms / args.steps)
    log64 = fs.log(args.warmup, args.steps)
    fixed, per_sweep, per_ref = C.c_int(), C.c_int(), C.c_int()
    capi.check(L.mp_fs1_kernel_counts(fs.handle, C.byref(fixed), C.byref(per_sweep),
                                      C.byref(per_ref)), "mp_fs1_kernel_counts")
    iters64 = log64[:, 0]
    launches = int(args.steps * fixed.value + np.ceil(iters64).sum() * per_sweep.value)
    vel_h, p_h64 = fs.get_state()

    # spin-up from rest, untimed, recording the learned guess's training samples
    # (features and solved increments of `--samples` fixed nodes at every step);
    # the network is trained on them before any variant is timed
    spin = make()
    net = meshless.MLP(seed=7)
    meshless.attach_mlp(spin, net, sample_nodes=min(args.samples, nv),
                        capacity_steps=max(args.spinup, 1))
    spin.set_state(vel0, p0, 0)
    spin.step(args.spinup, stream.handle)
    stream.sync()
    t0 = time.time()
    train_loss = None
    if args.spinup >= 3:
        train_loss = meshless.train_mlp(spin, epochs=args.epochs, batch=1024, lr=1e-3)
    t_train = time.time() - t0
    del spin

    def timed_steps(f, K, W):
        # every variant repeats the spin-up from rest (untimed), so its Adams-Bashforth
        # and pressure histories are its own, then warms up and times K steps
        f.set_state(vel0, p0, 0)
        f.step(args.spinup, stream.handle)
        for _ in range(W):
            f.step(1, stream.handle)
        stream.sync()
        barrier(pg)
        stream.sync()
        with capi.Timer(stream.handle) as tm:
            for _ in range(K):
                f.step(1, stream.handle)
        return tm.ms / K

    base = {}

    def variant(guess=capi.MP_GUESS_PREVIOUS, **cfg):
        """Time the steps after the spin-up with a solver configuration; errors and
        speed-up against the plain FP64 run over the same steps."""
        f = make(**cfg)
        if guess == capi.MP_GUESS_LEARNED:
            meshless.attach_mlp(f, net, sample_nodes=1, capacity_steps=1, collect=False)
        if guess != capi.MP_GUESS_PREVIOUS:
            meshless.set_guess(f, guess)
        ms = max_over_ranks(pg, timed_steps(f, args.steps, args.warmup))
        lg = f.log(args.spinup + args.warmup, args.steps)
        vv, pp = f.get_state()
        out = {"ms_per_step": round(ms, 4), "iters_per_step": float(np.mean(lg[:, 0])),
               "relres0_mean": float(np.mean(lg[:, 4])), "max_relres": float(lg[:, 1].max())}
        if not base:
            base.update(ms=ms, vel=vv, p=pp)
            return out
        err = [float(np.abs(vv[d] - base["vel"][d]).max() / np.abs(base["vel"][d]).max())
               for d in range(2)]
        perr = float(np.abs((pp - base["p"])[:nv]).max() / np.abs(base["p"][:nv]).max())
        if guess == capi.MP_GUESS_LEARNED:
            out["learned_weight_mean"] = float(np.mean(lg[:, 6]))
        if cfg.get("precision") == capi.MP_FP32:
            out["refinements_per_step"] = float(np.mean(lg[:, 5]))
        out["speedup_vs_plain_fp64"] = round(base["ms"] / ms, 3)
        out["rel_err_vs_fp64"] = {"u": err[0], "v": err[1], "p": perr}
        return out

    variants = {}
    if not args.no_mixed:
        variants["plain_fp64"] = variant()
        # FP64 BiCGSTAB, multigrid operators stored in FP32 (difference form)
        variants["mg32"] = variant(precision=capi.MP_MG32)
        # FP32 BiCGSTAB + multigrid under FP64 iterative refinement
        variants["fp32_refined"] = variant(precision=capi.MP_FP32, inner_tol=args.inner_tol)
        variants["extrapolated_guess"] = variant(guess=capi.MP_GUESS_EXTRAPOLATE)
        variants["projected_guess"] = variant(guess=capi.MP_GUESS_PROJECT)
        variants["projected_mg32"] = variant(guess=capi.MP_GUESS_PROJECT, precision=capi.MP_MG32)
        variants["learned_guess"] = variant(guess=capi.MP_GUESS_LEARNED)
        variants["learned_mg32"] = variant(guess=capi.MP_GUESS_LEARNED, precision=capi.MP_MG32)

    # end to end through the C ABI drop-in with pinned host buffers, continuing the
    # headline run from its state after the timed steps
    u_h = capi.PinnedArray((nv,))
    v_h = capi.PinnedArray((nv,))
    p_h = capi.PinnedArray((ns,))
    un_h = capi.PinnedArray((nv,))
    vn_h = capi.PinnedArray((nv,))
    pn_h = capi.PinnedArray((ns,))
    u_h.array[:] = vel_h[0]
    v_h.array[:] = vel_h[1]
    p_h.array[:] = p_h64
    vo = (C.c_void_p * 2)(u_h.ptr, v_h.ptr)
    vn = (C.c_void_p * 2)(un_h.ptr, vn_h.ptr)
    step0 = args.warmup + args.steps
    barrier(pg)
    with capi.Timer(stream.handle) as tm:
        for k in range(args.steps):
            capi.check(L.mp_fs1_single_timestep(fs.handle, vn if k % 2 == 0 else vo,
                                                C.c_void_p(pn_h.ptr if k % 2 == 0 else p_h.ptr),
                                                vo if k % 2 == 0 else vn,
                                                C.c_void_p(p_h.ptr if k % 2 == 0 else pn_h.ptr),
                                                step0 + k, stream.handle), "single_timestep")
    e2e_ms = max_over_ranks(pg, tm.ms / args.steps)
    e2e_bytes = (2 * nv + ns) * 8

    # SpMV roofline: the FP64 Laplacian at this size, CUDA events on its stream
    op = cld.operator(capi.MP_LAPLACIAN)
    x = capi.DeviceArray.from_host(np.random.default_rng(0).standard_normal(nv))
    y = capi.DeviceArray((nv,))
    for _ in range(5):
        op.apply(x, y, stream=stream.handle)
    reps = 50
    with capi.Timer(stream.handle) as tm:
        for _ in range(reps):
            op.apply(x, y, stream=stream.handle)
    spmv_ms = tm.ms / reps
    K = cld.n
    alg_bytes = nv * (12 * K + 16)
    achieved = alg_bytes / (spmv_ms * 1e-3) / 1e9
    peak, peak_kind = measured_peak()
    lm = variants.get("learned_mg32") or {}
    lg_ = variants.get("learned_guess") or {}
    pj = variants.get("projected_guess") or {}
    out = {
        "metric": METRIC,
        "value": round(ms64_max, 4), "unit": "ms/step", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms64_max, 4), "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": bench_config(nx, nv, cld.n, prm.dt, args.courant),
        "solver": "BiCGSTAB + smoothed-aggregation multigrid on the GPU, FP64",
        "pressure_iters_per_step": float(iters64.mean()),
        "max_relres": float(log64[:, 1].max()),
        # learned + mixed precision against plain FP64, after the spin-up (variants: every
        # configuration)
        "learned_mixed_speedup_vs_plain_fp64": lm.get("speedup_vs_plain_fp64"),
        "learned_vs_projected": (round(pj["ms_per_step"] / lg_["ms_per_step"], 3)
                                 if pj and lg_ else None),
        "learned_weight_mean": lg_.get("learned_weight_mean"),
        "e2e": {"value": round(e2e_ms, 4), "unit": "ms/step", "h2d_bytes_per_step": e2e_bytes,
                "d2h_bytes_per_step": e2e_bytes},
        "roofline": {"kernel": "ell_spmv_kernel<double> (laplacian, width 20)", "bound": "hbm",
                     "achieved": round(achieved, 1), "peak": peak, "peak_kind": peak_kind,
                     "unit": "GB/s", "frac": round(achieved / peak, 4),
                     "traffic": profile_traffic(), "algorithmic_bytes": alg_bytes,
                     "launch_ms": round(spmv_ms, 5)},
        "gpu_launches": launches,
        "clocks": clocks,
        "learned_mixed": variants.get("learned_mg32"),
        "variants": variants,
        "learned_training": training_summary(min(args.samples, nv) * max(args.spinup - 2, 0),
                                             args.epochs, train_loss, t_train,
                                             spinup_steps=args.spinup,
                                             sample_nodes=min(args.samples, nv)),
        "setup_s": {"cloud": round(t_cloud, 2), "fs1_and_multigrid": round(t_setup, 2)},
    }
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(cl, cld, prm.dt)
    # supplementary workloads: a failure in one is reported in its own field and
    # does not cost the headline line; a failure that leaves the CUDA context broken
    # (a sticky error) stops the rest and is reported as context_error
    legs = []
    if args.batched > 0:
        legs.append(("batched_stencils", lambda: batched_stencils(args.batched, stream)))
    if ws == 1 and not args.no_cube:
        legs.append(("cube3d_mixed", lambda: cube_mixed(args, stream)))
    if ws == 1 and not args.no_channel:
        legs.append(("channel_learned", lambda: channel_learned(args, stream)))
    if ws == 1 and args.integrator_steps > 0:
        legs.append(("integrators", lambda: integrators(args, cl, cld, prm, pts)))
    for name, run in legs:
        try:
            out[name] = run()
        except Exception as e:  # noqa: BLE001 -- any failure is reported, not raised
            out[name] = {"error": f"{type(e).__name__}: {e}"[:400]}
            if L.mp_stream_sync(None) != capi.MP_OK:
                out["context_error"] = f"{name}: {capi.last_error()}"[:400]
                break
    return out


def training_summary(samples, epochs, loss, secs, **extra):
    """Training throughput of the network: forward + backward ~ 3 x 82,176 flop per
    sample and epoch (the 41,088 multiply-adds of the forward, twice that backward),
    against the measured sustained BF16 tensor peak (training runs for seconds)."""
    flops = 3.0 * 82176.0 * samples * epochs
    tf = flops / secs / 1e12 if secs > 0 else None
    try:
        peak = float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["bf16_tflops_sustained"])
    except Exception:
        peak = 1400.0
    return {**extra, "samples": samples, "epochs": epochs, "final_loss": loss,
            "train_s": round(secs, 2), "train_tflops": round(tf, 2) if tf else None,
            "train_frac_of_bf16_sustained": round(tf / peak, 5) if tf else None}


def steps_timed(f, stream, first, warmup, steps):
    """`warmup` untimed steps, then `steps` steps between CUDA events; returns the
    ms per step and the solver log of the timed steps (first = the step index the
    state was set to)."""
    from memphys_b200 import capi
    for _ in range(warmup):
        f.step(1, stream.handle)
    stream.sync()
    with capi.Timer(stream.handle) as tm:
        for _ in range(steps):
            f.step(1, stream.handle)
    return tm.ms / steps, f.log(first + warmup, steps)


def integrators(args, cl, cld, prm, pts):
    """The other time integrators on the headline's 1,004,000-node cavity and dt, each
    end to end through its entry point with host arrays in and out (CUDA events on the
    default stream, which those calls use; every call ends synchronised).

    SEMI_IMPLICIT_SPLIT_SOLVER as the reference's own driver sets it up
    (eccentric_couette_flow_batch_ml.cpp:61-72: 5 outer iterations, iterative
    tolerance 1e-4): Jacobi-BiCGSTAB velocity solves and the multigrid pressure
    correction, to 1e-8, from rest.  IMPLICIT_SCALAR_TRANSPORT_SOLVER: one heated-lid
    scalar step per call in the resulting velocity (the driver's closing call, :93-94).
    FRACTIONAL_STEP_FOURIER: the cavity extruded over 2 nw + 1 = 5 planes of period 1,
    5,020,000 unknowns per field."""
    from memphys_b200 import capi, meshless
    nv = cl.nv
    K = max(1, args.integrator_steps)
    out = {"nodes": nv, "dt": prm.dt}
    state = {}

    def semi_implicit():
        t0 = time.time()
        sis = meshless.SEMI_IMPLICIT_SPLIT_SOLVER(pts, cld, prm, cl.u_dirichlet, cl.v_dirichlet,
                                                  cl.p_dirichlet, 5, 1e-4, 10000)
        t_setup = time.time() - t0
        ns = sis.system_size
        u, v, p = cl.vel_bc[0].copy(), cl.vel_bc[1].copy(), np.zeros(ns)
        logs = []
        un, vn, pn = np.zeros(nv), np.zeros(nv), np.zeros(ns)
        sis.single_timestep_2d(un, vn, pn, u, v, p, 0)  # BDF1 step, untimed
        u, v, p = un.copy(), vn.copy(), pn.copy()
        with capi.Timer(None) as tm:
            for k in range(K):
                logs.append(sis.single_timestep_2d(un, vn, pn, u, v, p, 1 + k))
                u, v, p = un.copy(), vn.copy(), pn.copy()
        state["vel"] = (u, v)
        return {"ms_per_step": round(tm.ms / K, 3), "steps": K,
                "outer_iters_per_step": float(np.mean([l[0] for l in logs])),
                "last_l1_change": logs[-1][1], "setup_s": round(t_setup, 2),
                "config": "n_outer_iter 5, iterative_tolerance 1e-4, solves to 1e-8, "
                          "BDF2 steps after one BDF1 step from rest"}

    def scalar_transport():
        # a transient step: the unsteady coefficient is 1 / dt (the reference multiplies
        # it by the BDF factor only), convection 1, diffusion 0.01; the velocity is the
        # semi-implicit run's (the lid's where that run failed)
        u, v = state.get("vel", (cl.vel_bc[0], cl.vel_bc[1]))
        ist = meshless.IMPLICIT_SCALAR_TRANSPORT_SOLVER(pts, cld, prm, cl.boundary, 10000,
                                                        1.0 / prm.dt, 1.0, -0.01)
        phi = np.where(cl.boundary & (cl.vel_bc[0] != 0), 1.0, 0.0)
        phn = np.zeros(nv)
        ist.single_timestep_2d(phn, phi, u, v, 0)
        phi = phn.copy()
        its = []
        with capi.Timer(None) as tm:
            for k in range(K):
                n_it, rr = ist.single_timestep_2d(phn, phi, u, v, 1 + k)
                its.append(n_it)
                phi = phn.copy()
        return {"ms_per_step": round(tm.ms / K, 3), "steps": K,
                "iters_per_step": float(np.mean(its)), "last_relres": rr}

    def fourier_z():
        nw, N = 2, 5
        t0 = time.time()
        fsf = meshless.FRACTIONAL_STEP_FOURIER(pts, cld, prm, cl.u_dirichlet, cl.v_dirichlet,
                                               cl.u_dirichlet, cl.p_dirichlet, 1.0, nw, 2)
        t_setup = time.time() - t0
        z = np.arange(N) / N
        x, y = cl.xyz[:, 0], cl.xyz[:, 1]
        g = [np.repeat(cl.vel_bc[0][:, None], N, 1), np.zeros((nv, N)),
             np.where(cl.boundary[:, None], 0.0,
                      0.05 * (np.sin(np.pi * x) * np.sin(np.pi * y))[:, None]
                      * np.cos(2 * np.pi * z)[None, :]), np.zeros((nv, N))]
        o = [np.zeros((nv, N)) for _ in range(4)]
        fsf.single_timestep(*o, *g, 0)
        g = [a.copy() for a in o]
        # end to end through the Python mirror: host (nv, N) arrays, node-major, which
        # the library transposes to its plane-contiguous layout and back on the device
        with capi.Timer(None) as tm:
            for k in range(K):
                fsf.single_timestep(*o, *g, 1 + k)
                g = [a.copy() for a in o]
        e2e_ms = tm.ms / K
        # device-resident through the C ABI: plane-contiguous device fields, ping-pong
        import ctypes as C
        L = capi.lib()
        capi.check(L.mp_fsf_set_layout(fsf.handle, 0), "mp_fsf_set_layout")
        stream = capi.Stream()
        dev = [[capi.DeviceArray.from_host(np.ascontiguousarray(a.T)) for a in g],
               [capi.DeviceArray((N, nv)) for _ in range(4)]]

        def dstep(k, a, b):
            vo = (C.c_void_p * 3)(*[dev[a][i].ptr for i in range(3)])
            vn = (C.c_void_p * 3)(*[dev[b][i].ptr for i in range(3)])
            capi.check(L.mp_fsf_single_timestep(fsf.handle, vo, C.c_void_p(dev[a][3].ptr), vn,
                                                C.c_void_p(dev[b][3].ptr), k, stream.handle),
                       "mp_fsf_single_timestep")
        dstep(1 + K, 0, 1)
        with capi.Timer(stream.handle) as tm:
            for k in range(K):
                dstep(2 + K + k, (k + 1) % 2, k % 2)
        return {"ms_per_step": round(tm.ms / K, 3), "steps": K, "planes": N,
                "unknowns_per_field": nv * N, "setup_s": round(t_setup, 2),
                "ms_per_step_host_arrays": round(e2e_ms, 3),
                "timing": "device fields through mp_fsf_single_timestep (ms_per_step); host "
                          "(nv, N) node-major arrays through the Python mirror, copied in and "
                          "out and transposed on the device (ms_per_step_host_arrays)",
                "w_max": float(np.abs(g[2]).max())}

    for name, fn in (("semi_implicit", semi_implicit), ("scalar_transport", scalar_transport),
                     ("fourier_z", fourier_z)):
        try:
            out[name] = fn()
        except capi.MemphysError as e:
            out[name] = {"error": str(e)[:300]}
            if capi.lib().mp_stream_sync(None) != capi.MP_OK:
                raise
    return out


def cube_mixed(args, stream):
    """The 3D mixed-precision configuration: unit-cube lid-driven cavity, 128^3
    jittered interior + 6 * 128^2 face nodes, PHS r^3 + degree 3 (20 monomials),
    40-node stencils, Re = 100.  From rest, `--cube-spinup` untimed steps, then the
    bench's warm-up and timed steps, for FP64, FP32 Krylov + FP64 refinement
    (MP_FP32) and FP32 multigrid storage (MP_MG32); the error of each field after
    the same steps is stated against the FP64 run."""
    from memphys_b200 import capi, clouds, meshless
    t0 = time.time()
    cl = clouds.cube_3d(args.cube_n)
    prm = meshless.PARAMETERS(solver_type="cuda_bicgstab_amg", solver_tolerance=1e-8, n_iter=2000)
    prm.rho, prm.mu = 1.0, 0.01
    pts = meshless.POINTS(cl)
    cld = meshless.CLOUD(pts, prm, compute_cond=False)
    t_cloud = time.time() - t0
    prm.dt = meshless.calc_dt(cld, 1.0, 1.0, 1.0, prm.mu / prm.rho, args.courant)
    vel0 = [cl.vel_bc[d].copy() for d in range(3)]
    res, states = {}, {}
    for name, cfg in (("fp64", {}),
                      ("fp32_refined", {"precision": capi.MP_FP32, "inner_tol": args.inner_tol}),
                      ("mg32", {"precision": capi.MP_MG32})):
        t0 = time.time()
        f = meshless.FRACTIONAL_STEP_1(pts, cld, prm, cl.u_dirichlet, cl.v_dirichlet,
                                       cl.p_dirichlet, 2, w_dirichlet_flag=cl.w_dirichlet, **cfg)
        t_setup = time.time() - t0
        f.set_state(vel0, np.zeros(f.system_size), 0)
        f.step(args.cube_spinup, stream.handle)
        ms, lg = steps_timed(f, stream, args.cube_spinup, args.warmup, args.steps)
        states[name] = f.get_state()
        res[name] = {"ms_per_step": round(ms, 3), "iters_per_step": float(lg[:, 0].mean()),
                     "refinements_per_step": float(lg[:, 5].mean()),
                     "max_relres": float(lg[:, 1].max()), "setup_s": round(t_setup, 2)}
        del f
    v64, p64 = states["fp64"]
    for name in ("fp32_refined", "mg32"):
        vv, pp = states[name]
        err = {c: float(np.abs(vv[d] - v64[d]).max() / max(np.abs(v64[d]).max(), 1e-300))
               for d, c in enumerate("uvw")}
        err["p"] = float(np.abs((pp - p64)[:cl.nv]).max() / np.abs(p64[:cl.nv]).max())
        res[name]["rel_err_vs_fp64"] = err
        res[name]["speedup_vs_fp64"] = round(res["fp64"]["ms_per_step"] / res[name]["ms_per_step"], 3)
    return {"workload": f"cube_3d {args.cube_n}^3 jittered + faces = {cl.nv} nodes, 40-node "
                        "stencils, BiCGSTAB + SA multigrid to 1e-8",
            "nodes": cl.nv, "dt": prm.dt, "spinup_steps": args.cube_spinup,
            "cloud_s": round(t_cloud, 2), **res}


def channel_learned(args, stream):
    """The learned-guess configuration: channel [0,8] x [0,1] with a cylinder of
    radius 0.1 at (1, 0.5), Re = 200, h = `--channel-h` (1,004,010 nodes), 20-node
    stencils, outlet p-Dirichlet.  The plain solver runs `--channel-train-steps`
    steps from rest while the network records its samples; the network is trained
    on them; then, from that state, each initial guess times the same steps
    (iterations and ms/step; the configuration's comparison is learned against
    zero).  The size of the second temporal difference that the network predicts,
    relative to the increment and to the pressure, is stated beside it."""
    from memphys_b200 import capi, clouds, meshless
    cl = clouds.channel_2d(args.channel_h)
    prm = meshless.PARAMETERS(solver_type="cuda_bicgstab_amg", solver_tolerance=1e-8, n_iter=4000)
    prm.rho, prm.mu = 1.0, 0.2 / 200.0
    pts = meshless.POINTS(cl)
    cld = meshless.CLOUD(pts, prm, compute_cond=False)
    prm.dt = meshless.calc_dt(cld, 1.5, 1.0, 0.0, prm.mu / prm.rho, args.courant)
    f = meshless.FRACTIONAL_STEP_1(pts, cld, prm, cl.u_dirichlet, cl.v_dirichlet, cl.p_dirichlet,
                                   2, w_dirichlet_flag=cl.w_dirichlet)
    T = max(args.channel_train_steps, 4)
    net = meshless.MLP(seed=11)
    ns_ = min(args.channel_samples, cl.nv)
    meshless.attach_mlp(f, net, sample_nodes=ns_, capacity_steps=T)
    f.set_state([cl.vel_bc[0], cl.vel_bc[1]], np.zeros(f.system_size), 0)
    t0 = time.time()
    f.step(T - 2, stream.handle)
    p1 = f.get_state()[1][:cl.nv]
    f.step(1, stream.handle)
    p2 = f.get_state()[1][:cl.nv]
    f.step(1, stream.handle)
    vel, p = f.get_state()
    t_spin = time.time() - t0
    plain = f.log(T - 100, 100) if T > 100 else f.log(0, T)
    rms = lambda a: float(np.sqrt(np.mean(a * a)))
    inc, d2 = p[:cl.nv] - p2, (p[:cl.nv] - p2) - (p2 - p1)
    t0 = time.time()
    loss = meshless.train_mlp(f, epochs=args.epochs, batch=1024, lr=1e-3)
    t_train = time.time() - t0
    meshless.attach_mlp(f, net, sample_nodes=1, capacity_steps=1, collect=False)
    res = {}
    for name, g in (("zero", capi.MP_GUESS_ZERO), ("previous", capi.MP_GUESS_PREVIOUS),
                    ("extrapolated", capi.MP_GUESS_EXTRAPOLATE),
                    ("projected", capi.MP_GUESS_PROJECT), ("learned", capi.MP_GUESS_LEARNED)):
        meshless.set_guess(f, g)
        f.set_state(vel, p, T + 1)
        ms, lg = steps_timed(f, stream, T + 1, args.warmup, args.steps)
        res[name] = {"ms_per_step": round(ms, 3), "iters_per_step": float(lg[:, 0].mean()),
                     "relres0_median": float(np.median(lg[:, 4])),
                     "max_relres": float(lg[:, 1].max())}
        if g == capi.MP_GUESS_LEARNED:
            res[name]["learned_weight_mean"] = float(np.mean(lg[:, 6]))
    res["learned"]["speedup_vs_zero_guess"] = round(res["zero"]["ms_per_step"] /
                                                    res["learned"]["ms_per_step"], 3)
    return {"workload": f"channel_2d h={args.channel_h} with cylinder, {cl.nv} nodes, Re 200, "
                        "BiCGSTAB + SA multigrid to 1e-8",
            "nodes": cl.nv, "dt": prm.dt,
            "training": training_summary(ns_ * (T - 2), args.epochs, loss, t_train,
                                         plain_steps=T, sample_nodes=ns_,
                                         spinup_s=round(t_spin, 2),
                                         plain_iters_last_steps=float(plain[:, 0].mean())),
            "second_difference_over_increment": rms(d2) / rms(inc),
            "increment_over_pressure": rms(inc) / rms(p[:cl.nv]),
            "guesses": res}


FP64_PEAK_TFLOPS = 37.0  # B200 datasheet FP64 (non-tensor) per GPU; no measured FP64 peak


def batched_stencils(nsys: int, stream):
    """The batched uneven stencil workload: nsys independent augmented PHS r^3 +
    degree-3 systems per dimension; 90 % interior stencils with n drawn from {20, 30},
    10 % boundary stencils with n from {40, 60}; offsets uniform in the unit ball
    scaled by h in [1e-3, 1e-2], node 0 the centre.  A plan classifies the systems
    once (host); each run is the persistent size-class kernels on the stream, timed
    with CUDA events over `reps` runs after one untimed run (which also tunes the CTA
    shapes).  FLOPs on the algorithmic basis (2/3) s^3 + 2 (dim + 1) s^2 per system,
    s = n + m (LU and the triangular solves; the kernel's Gauss-Jordan does more).
    The weights of this workload are checked against per-stencil LAPACK in the GPU
    tests (tests/test_gpu_parity.py), not here."""
    import ctypes as C
    from memphys_b200 import capi
    L = capi.lib()
    res = {}
    reps = 3
    for dim, m in ((2, 10), (3, 20)):
        rng = np.random.default_rng(20261203 + dim)
        bnd = rng.random(nsys) < 0.1
        sizes = np.where(bnd, rng.choice([40, 60], size=nsys),
                         rng.choice([20, 30], size=nsys)).astype(np.int32)
        off = np.zeros(nsys, np.int64)
        off[1:] = np.cumsum(sizes[:-1], dtype=np.int64)
        total = int(sizes.sum(dtype=np.int64))
        pts = rng.normal(size=(total, dim))
        pts /= np.linalg.norm(pts, axis=1, keepdims=True)
        pts *= rng.random((total, 1)) ** (1.0 / dim)
        pts *= np.repeat(rng.uniform(1e-3, 1e-2, nsys), sizes)[:, None]
        pts[off] = 0.0  # the centre node first
        d_sizes = capi.DeviceArray.from_host(sizes)
        d_off = capi.DeviceArray.from_host(off)
        d_pts = capi.DeviceArray.from_host(np.ascontiguousarray(pts))
        d_w = capi.DeviceArray(((dim + 1) * total,))
        del pts
        plan = C.c_void_p()
        t0 = time.time()
        capi.check(L.mp_stencil_plan_create(nsys, capi.ptr(d_sizes), capi.ptr(d_off), dim, 3,
                                            C.byref(plan)), "mp_stencil_plan_create")
        t_plan = time.time() - t0
        try:
            def run():
                capi.check(L.mp_stencil_plan_run(plan, capi.ptr(d_pts), 3, capi.ptr(d_w), None,
                                                 stream.handle), "mp_stencil_plan_run")
            run()  # untimed: tunes the CTA shapes of each class on its first run
            bad = C.c_int()
            capi.check(L.mp_stencil_plan_singular(plan, C.byref(bad), stream.handle))
            with capi.Timer(stream.handle) as tm:
                for _ in range(reps):
                    run()
            secs = tm.ms / reps / 1e3
            counts = (C.c_int * 7)()
            shapes = (C.c_int * 7)()
            capi.check(L.mp_stencil_plan_info(plan, counts, shapes))
        finally:
            L.mp_stencil_plan_destroy(plan)
        s_ = sizes.astype(np.float64) + m
        flops = float(np.sum(2.0 / 3.0 * s_ ** 3 + 2.0 * (dim + 1) * s_ ** 2))
        tf = flops / secs / 1e12
        res[f"{dim}d"] = {"systems": nsys, "monomials": m, "seconds": round(secs, 5),
                          "systems_per_s": round(nsys / secs), "tflops_fp64_algorithmic": round(tf, 3),
                          "frac_of_fp64_datasheet": round(tf / FP64_PEAK_TFLOPS, 4),
                          "singular": bad.value, "plan_s": round(t_plan, 2),
                          "class_systems": list(counts), "class_systems_per_cta": list(shapes)}
        del d_w, d_pts
    res["fp64_peak_tflops"] = f"{FP64_PEAK_TFLOPS} (B200 datasheet, FP64 non-tensor; not measured)"
    return res


def profile_range(args, cl, cld, make, fs, vel0, p0, stream, pts, prm):
    """Warm-up outside, `--steps` steps (SpMV launches, weight computations) inside the
    capture range."""
    from memphys_b200 import capi, meshless
    L = capi.lib()
    nv = cld.nv

    def in_range(run):
        for _ in range(args.warmup):
            run(False)
        L.mp_stream_sync(None)
        stream.sync()
        capi.check(L.mp_profiler(1))
        for k in range(args.steps):
            run(True)
        L.mp_stream_sync(None)
        stream.sync()
        capi.check(L.mp_profiler(0))

    if args.profile == "cloud":
        # kNN stencils, PHS-RBF-FD weights and condition numbers of the whole cloud
        in_range(lambda timed: meshless.CLOUD(pts, prm, compute_cond=True))
        return {"profile": "cloud", "builds": args.steps, "nodes": nv}
    if args.profile == "sis":
        # --no-graph: kernels inside graphs with conditional nodes cannot be profiled
        sis = meshless.SEMI_IMPLICIT_SPLIT_SOLVER(pts, cld, prm, cl.u_dirichlet, cl.v_dirichlet,
                                                  cl.p_dirichlet, 5, 1e-4, 10000,
                                                  use_graph=not args.no_graph)
        st = {"u": cl.vel_bc[0].copy(), "v": cl.vel_bc[1].copy(), "p": np.zeros(sis.system_size),
              "it": 0}

        def sis_step(timed):
            un, vn, pn = np.zeros(nv), np.zeros(nv), np.zeros(sis.system_size)
            sis.single_timestep_2d(un, vn, pn, st["u"], st["v"], st["p"], st["it"])
            st.update(u=un, v=vn, p=pn, it=st["it"] + 1)
        in_range(sis_step)
        return {"profile": "sis", "steps": args.steps, "nodes": nv}
    if args.profile == "fsf":
        N = 5
        fsf = meshless.FRACTIONAL_STEP_FOURIER(pts, cld, prm, cl.u_dirichlet, cl.v_dirichlet,
                                               cl.u_dirichlet, cl.p_dirichlet, 1.0, 2, 2)
        st = {"g": [np.repeat(cl.vel_bc[0][:, None], N, 1)] + [np.zeros((nv, N))] * 3, "it": 0}

        def fsf_step(timed):
            o = [np.zeros((nv, N)) for _ in range(4)]
            fsf.single_timestep(*o, *st["g"], st["it"])
            st.update(g=o, it=st["it"] + 1)
        in_range(fsf_step)
        return {"profile": "fsf", "steps": args.steps, "nodes": nv, "planes": N}
    if args.profile == "train":
        # samples from a short spin-up, then training epochs in the range
        net = meshless.MLP(seed=7)
        meshless.attach_mlp(fs, net, sample_nodes=min(args.samples, nv),
                            capacity_steps=max(args.spinup, 3))
        fs.set_state(vel0, p0, 0)
        fs.step(max(args.spinup, 3), stream.handle)
        stream.sync()
        in_range(lambda timed: meshless.train_mlp(fs, epochs=1, batch=1024, lr=1e-3))
        return {"profile": "train", "epochs": args.steps,
                "samples": min(args.samples, nv) * max(args.spinup - 2, 1)}
    if args.profile == "steps":
        if args.variant != "plain":
            fs = make(precision=capi.MP_MG32)
            if args.variant == "learned_mg32":
                # train on a short spin-up first (outside the capture range)
                net = meshless.MLP(seed=7)
                meshless.attach_mlp(fs, net, sample_nodes=min(args.samples, nv),
                                    capacity_steps=max(args.spinup, 3))
                fs.set_state(vel0, p0, 0)
                fs.step(max(args.spinup, 3), stream.handle)
                stream.sync()
                meshless.train_mlp(fs, epochs=args.epochs, batch=1024, lr=1e-3)
                meshless.attach_mlp(fs, net, sample_nodes=1, capacity_steps=1, collect=False)
                meshless.set_guess(fs, capi.MP_GUESS_LEARNED)
            elif args.variant == "extrapolated_mg32":
                meshless.set_guess(fs, capi.MP_GUESS_EXTRAPOLATE)
            elif args.variant == "projected_mg32":
                meshless.set_guess(fs, capi.MP_GUESS_PROJECT)
        fs.set_state(vel0, p0, 0)
        fs.step(args.spinup + args.warmup, stream.handle)
        stream.sync()
        capi.check(L.mp_profiler(1))
        fs.step(args.steps, stream.handle)
        stream.sync()
        capi.check(L.mp_profiler(0))
        log = fs.log(args.spinup + args.warmup, args.steps)
        return {"profile": "steps", "variant": args.variant, "iters": log[:, 0].tolist()}
    if args.profile == "stencil":
        # the cloud's PHS-RBF-FD weights from its own stencils, device in and out
        cld.fetch()
        nb = cld.nb_points_col
        n = nb.shape[1]
        dx = capi.DeviceArray.from_host(np.ascontiguousarray(cl.xyz, np.float64))
        dn = capi.DeviceArray.from_host(np.ascontiguousarray(nb, np.int32))
        w = [capi.DeviceArray((nv, n)) for _ in range(3)]

        def weights():
            capi.check(L.mp_stencil_weights(capi.ptr(dx), nv, cl.dim, capi.ptr(dn), n, 3, 3,
                                            capi.ptr(w[0]), capi.ptr(w[1]), None,
                                            capi.ptr(w[2]), None, stream.handle),
                       "mp_stencil_weights")
        for _ in range(args.warmup):
            weights()
        stream.sync()
        capi.check(L.mp_profiler(1))
        for _ in range(args.steps):
            weights()
        stream.sync()
        capi.check(L.mp_profiler(0))
        return {"profile": "stencil", "launches": args.steps, "stencils": nv, "n": n}
    op = cld.operator(capi.MP_LAPLACIAN)
    x = capi.DeviceArray.from_host(np.random.default_rng(0).standard_normal(nv))
    y = capi.DeviceArray((nv,))
    for _ in range(args.warmup):
        op.apply(x, y, stream=stream.handle)
    stream.sync()
    capi.check(L.mp_profiler(1))
    for _ in range(args.steps):
        op.apply(x, y, stream=stream.handle)
    stream.sync()
    capi.check(L.mp_profiler(0))
    return {"profile": "spmv", "launches": args.steps, "nodes": nv}


def cpu_baseline(cl, cld, dt, max_iters=40):
    """The CPU oracle (C restatement of the reference's FS1 step with BiCGSTAB+ILUT),
    one thread, the first timestep from rest of the same cloud with the pressure solve
    capped."""
    import oracle
    cld.fetch()
    w = {"gx": cld.grad_x_coeff, "gy": cld.grad_y_coeff, "lap": cld.laplacian_coeff}
    t0 = time.time()
    f = oracle.FS1(cl, cld.nb_points_col, w, 1.0, 0.01, dt, 2, 1e-8, max_iters, 1e-6, 50)
    t_setup = time.time() - t0
    vel = [cl.vel_bc[0].copy(), cl.vel_bc[1].copy()]
    p = np.zeros(f.nsys)
    prev = oracle.set_threads(1)  # the reference's own semantics: one thread
    t0 = time.time()
    iters, rr = f.step(vel, p, 0)
    secs = time.time() - t0
    oracle.set_threads(prev)
    return {"value": round(secs * 1e3, 1), "unit": "ms/step", "cores": 1, "kind": "port",
            "sample": f"the first timestep from rest of the same {cl.nv}-node cavity, one "
                      f"thread; BiCGSTAB + ILUT(1e-6, 50) capped at {max_iters} iterations "
                      f"({iters} run, relres {rr:.1e}"
                      + ("; the reference's solver does not reach 1e-8 at this size"
                         if rr > 1e-8 else "") + f"); ILUT setup {t_setup:.1f} s excluded"}


def reference_dt(cl, nb, w, courant):
    """PARAMETERS::calc_dt (parameters.cpp:269-296) with the largest-magnitude
    eigenvalues from ARPACK (scipy), the counterpart of the reference's Spectra
    Arnoldi (general_functions.cpp:4-24)."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as sla
    nv, n = nb.shape
    rows = np.repeat(np.arange(nv), n)
    ev = 0.0
    for key, coef in (("gx", 1.0), ("gy", 1.0), ("lap", 0.01)):
        A = sp.csr_matrix((w[key].ravel(), (rows, nb.ravel())), shape=(nv, nv))
        lam = sla.eigs(A, k=1, which="LM", ncv=30, tol=1e-10, v0=np.ones(nv),
                       return_eigenvectors=False)[0]
        ev += coef * abs(lam)
    return bench_dt(courant * 2.0 / ev)


# ----------------------------------------------------------- reference arm
def run_reference(args, ws, rank):
    """The reference's CPU path (the oracle's C restatement of FRACTIONAL_STEP_1 with
    SOLVER eigen_ilu_bicgstab: Eigen/HYPRE are not installable here) on the host cores,
    over the same steps as `value`: from rest, `--warmup` untimed steps, `--steps`
    timed ones, dt from calc_dt with ARPACK eigenvalues.  Each pressure solve runs
    BiCGSTAB + ILUT(1e-6, 50) from the previous pressure to 1e-8 or REF_MAXIT
    iterations, whichever comes first; the iterations and residuals reached are
    reported."""
    import oracle
    from memphys_b200 import clouds
    cl = clouds.cavity_2d(args.nx)
    n = oracle.cloud_size(2, 3, 2.0)
    cores = os.cpu_count() or 1
    oracle.set_threads(cores)  # every host thread for the row-parallel loops
    t0 = time.time()
    nb = oracle.knn_stencils(cl.xyz, cl.boundary, n)
    w = parallel_weights(cl.xyz, nb)
    dt = reference_dt(cl, nb, w, args.courant)
    t_setup = time.time() - t0
    f = oracle.FS1(cl, nb, w, 1.0, 0.01, dt, 2, 1e-8, REF_MAXIT, 1e-6, 50)
    vel = [cl.vel_bc[0].copy(), cl.vel_bc[1].copy()]
    p = np.zeros(f.nsys)
    for it in range(args.warmup):
        f.step(vel, p, it)
    iters, res = [], []
    t0 = time.time()
    for it in range(args.steps):
        k, rr = f.step(vel, p, args.warmup + it)
        iters.append(k)
        res.append(rr)
    ms = (time.time() - t0) * 1e3 / args.steps
    sample = (f"{args.steps} timesteps (after {args.warmup} untimed) of the {cl.nv}-node cavity "
              f"from rest: C restatement of FRACTIONAL_STEP_1 + SOLVER eigen_ilu_bicgstab, "
              f"BiCGSTAB + ILUT(1e-6, 50) to 1e-8 or {REF_MAXIT} iterations per step (mean "
              f"{np.mean(iters):.0f} run, relres reached {min(res):.1e} to {max(res):.1e}"
              + (": the reference's solver does not reach 1e-8 at this size, so this is a lower "
                 "bound of its converged step" if max(res) > 1e-8 else "") +
              f"); SpMV rows and fractional-step row loops on {cores} "
              f"threads, vector updates, dot products and ILUT solves serial as in Eigen; "
              f"setup (stencils, weights, ARPACK dt) {t_setup:.0f} s")
    return {"metric": METRIC, "impl": "reference", "value": round(ms, 2), "unit": "ms/step",
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 2),
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": bench_config(args.nx, cl.nv, n, dt, args.courant),
            "solver": f"BiCGSTAB + ILUT(1e-6, 50) on the CPU (C restatement), FP64, at most "
                      f"{REF_MAXIT} iterations per step",
            "pressure_iters_per_step": float(np.mean(iters)),
            "max_relres": float(max(res)),
            "cpu_baseline": {"value": round(ms, 2), "unit": "ms/step", "cores": cores,
                             "kind": "port", "sample": sample},
            "e2e": {"value": round(ms, 2), "unit": "ms/step", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def parallel_weights(xyz, nb):
    """Oracle weights over stencil chunks on all host cores (ctypes releases the GIL)."""
    import concurrent.futures as cf
    import oracle
    nthreads = max(1, os.cpu_count() or 1)
    chunks = [c for c in np.array_split(np.arange(len(nb)), nthreads) if len(c)]
    with cf.ThreadPoolExecutor(nthreads) as ex:
        parts = list(ex.map(lambda c: oracle.cloud_weights(xyz, nb[c], 3, 3, cond=False), chunks))
    # each chunk's stencils index the full cloud, so the rows are already global
    return {k: np.concatenate([p[k] for p in parts]) for k in ("gx", "gy", "lap")}


def main():
    args = parse()
    if args.impl == "reference":
        # rank 0 alone times the CPU path; other ranks exit without work
        ws = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        if rank == 0:
            print(json.dumps(run_reference(args, ws, rank)), flush=True)
        return
    ws, rank, local, pg = dist_setup(args)
    out = run_ours(args, ws, rank, local, pg)
    if rank == 0:
        print(json.dumps(out), flush=True)
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()
    if "context_error" in out:
        sys.exit(1)


if __name__ == "__main__":
    main()
