#!/usr/bin/env python
"""SART + FISTA + FGP-TV iterations/s on the 512^3 / 1024-view CBCT scan.

One step = one outer iteration of the reference's FISTA loop
(V63/main_recon.cu:344-430): a SART pass over all 1024 views (Siddon FP
correction + gather BP update per view, in order), the FGP-TV prox with 20
inner iterations, the FISTA momentum and the objective (a forward
projection of all views plus the TV norm).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Each rank reconstructs its own copy of the scan (replicas: the path has no
data exchange between scans), so ``value`` is the sum over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SCAN = dict(nx=512, ny=512, nz=512, vx=0.5, nu=1024, nv=768, du=0.4, dso=1000.0, dod=-500.0, n_views=1024)
# The SART relaxation of the FISTA loop is the reference's own step,
# step_size = 2/Lip_con with Lip_con = 32 (V63/main_recon.cu:58,161).  (A
# relaxation of 0.8, right for plain SART, makes FISTA over SART diverge after
# a few iterations at these sizes.)
BETA, LAMBDA_TV, FGP_ITERS = 2.0 / 32.0, 2e-4, 20
METRIC = "SART-FISTA-TV iter/s & voxel-updates/s, 512^3 x 1024 views, mixed vs FP32, 1 B200"
# 16 views spread evenly over the scan, off the axis-aligned angles (views
# 0, 256, 512, 768 at 1024 views): the CPU arms time their SART and
# objective projections on these, and the measurement noise is scaled to
# their largest ray sum
SAMPLE_VIEWS = [17 + 64 * k for k in range(16)]
NOISE = 0.005          # Gaussian noise sigma, relative to the largest ray sum of the sample views
SCAN_SEED = 2024


def scan_config(world):
    """The workload's description, shared by both arms of the benchmark."""
    return {"workload": "SART+FISTA+FGP-TV (20 inner) iteration with objective, 512^3 x 0.5 mm, "
                        "1024 views, 1024x768 detector x 0.4 mm, DSO 1000 mm, DOD -500 mm",
            "phantom": "40 ellipsoids + 200 spheres (seeded), Siddon projections + 0.5% noise",
            "parallelism": f"replicas x{world}", "l2": "inputs > L2 (512 MB+ volume)",
            "relaxation": BETA, "lambda_tv": LAMBDA_TV, "fgp_iters": FGP_ITERS}


def refine_note(args):
    """The refinement solver's correction volume, as the bench lines name it."""
    return "FP32 correction volume" if args.refine == 2 else "16-bit correction volume"


def view_noise(view, n, seed):
    """Unit Gaussian noise of one view (CPU generator seeded per view, so the
    CPU arm can draw its sample views' noise without the others)."""
    import torch
    gen = torch.Generator().manual_seed(seed * 1000003 + view)
    return torch.randn(n, generator=gen, dtype=torch.float32)


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=6)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--mixed", choices=["f16", "bf16"], default="f16")
    p.add_argument("--large-plain", action="store_true",
                   help="large: also run plain FP16 storage (no refinement) against the FP64 reference")
    p.add_argument("--refine", type=int, choices=[1, 2], default=2,
                   help="the 16-bit runs' refinement solver: 1 keeps the correction volume in the 16-bit type, "
                        "2 in FP32")
    p.add_argument("--fast-sums", action="store_true",
                   help="the mixed-precision run (and --profile-views) with fused ray sums (CTR_GEOM_FAST_SUMS); "
                        "the default")
    p.add_argument("--exact-sums", action="store_true",
                   help="the mixed-precision run (and --profile-views) with the reference's ray-sum sequence "
                        "instead of fused ray sums")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--profile-views", type=int, default=0,
                   help="profiling mode: set up the scan, run a SART update of this many views, print timings, exit")
    p.add_argument("--profile-iteration", action="store_true",
                   help="with --profile-views: also run two FP16 solver iterations (the second in steady state)")
    p.add_argument("--profile-refbp", action="store_true",
                   help="with --profile-views: the SART updates with the reference backprojector's arithmetic")
    p.add_argument("--profile-obj", action="store_true",
                   help="short run for ncu: two FP16 solver iterations on an 8-view subset of the 512^3 scan "
                        "(the second projects the first's objective in its SART traversal)")
    p.add_argument("--profile-slabs", type=int, default=0,
                   help="short run for ncu: N views of the 4-slab SART (the reference's default 4-device build) "
                        "on the 512^3 scan, FP32, its backprojection arithmetic, tiled")
    p.add_argument("--profile-fdk", type=int, default=0,
                   help="profiling mode: FDK of the 512^3 scan restricted to this many views (weighting, ramp "
                        "and backprojection), print timings, exit")
    p.add_argument("--profile-tune", action="store_true",
                   help="with --profile-views: also print the tuner's time for every launch shape")
    p.add_argument("--workload", choices=["scan512", "batched", "large", "tbct"], default="scan512",
                   help="scan512: the 512^3 / 1024-view scan (default); batched: 48 uneven scans in one graph; "
                        "large: 1024^3 / 1024 views / 1024^2 detector in FP32, BF16 and FP16; tbct: the "
                        "tetrahedron-beam program's scan (512^3, 64 sources x 16 rows x 1024, 360 views)")
    p.add_argument("--scans", type=int, default=48, help="batched: number of scans")
    p.add_argument("--no-tune", action="store_true", help="batched: keep the default launch shapes")
    p.add_argument("--no-sr", action="store_true", help="batched: BF16 updates rounded to nearest instead of "
                                                        "stochastically")
    args = p.parse_args()
    # the mixed-precision run is not the reference's sum sequence in any case
    # (refinement), so it takes the fused sums unless asked otherwise; the
    # FP32 run always keeps the reference's sequence, and --profile-views
    # takes the fused sums only when --fast-sums is given
    args.profile_fast_sums = args.fast_sums
    args.fast_sums = not args.exact_sums
    return args


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


# Replicas: every rank reconstructs its own scan (seeded by its rank); the
# only collectives are the barriers around the timed regions and the maximum
# of the per-rank times.  NCCL on the GPUs; the same calls run over gloo on
# the CPU in the tests.
def init_replicas(world, backend="nccl", timeout_s=600):
    import torch.distributed as dist
    if world > 1 and not dist.is_initialized():
        from datetime import timedelta
        dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s))


def max_over_ranks(x, world, device):
    """The largest of the ranks' values of x (a time in ms): the job's time."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(ms_max, world):
    """Whole-job iterations/s: every rank completes one iteration per step,
    the job's step time is the slowest rank's."""
    return world * 1000.0 / ms_max


def phantom_params(seed=2024):
    """40 ellipsoids (semi-axes 3-100 mm, 0.005-0.04 /mm) + 200 spheres (r 1-3 mm, 0.05 /mm)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    n1, n2 = 40, 200
    p = np.zeros((n1 + n2, 10))
    p[:n1, 0:2] = rng.uniform(-60, 60, (n1, 2))
    p[:n1, 2] = rng.uniform(-60, 60, n1)
    p[:n1, 3:6] = rng.uniform(3, 100, (n1, 3))
    p[:n1, 6:9] = rng.uniform(0, 2 * np.pi, (n1, 3))
    p[:n1, 9] = rng.uniform(0.005, 0.04, n1)
    r = rng.uniform(1, 3, n2)
    ang = rng.uniform(0, 2 * np.pi, n2)
    rad = 100 * np.sqrt(rng.uniform(0, 1, n2))
    p[n1:, 0], p[n1:, 1] = rad * np.cos(ang), rad * np.sin(ang)
    p[n1:, 2] = rng.uniform(-90, 90, n2)
    p[n1:, 3:6] = r[:, None]
    p[n1:, 9] = 0.05
    return p


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                self.rows.append(f)

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": len(self.rows)}
        if not self.rows:
            return out
        import statistics
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        out["sm_mhz"] = statistics.median(sm) if sm else None
        out["sm_max_mhz"] = max(mx) if mx else None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for k, n in enumerate(names):
                if r[5 + k].lower().startswith("active"):
                    reasons.add(n)
        out["reasons"] = sorted(reasons)
        return out


def measured_peak_hbm():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profiled_traffic(name="roofline_traffic.json"):
    """Per-launch DRAM bytes and warp instructions of the backprojector from
    the committed ncu summary."""
    try:
        with open(os.path.join(ROOT, "profiles", name)) as f:
            return json.load(f)
    except (OSError, ValueError):
        return None


def issue_roofline(traffic, launch_ms, sm_mhz, dev):
    """The bound that applies to the projectors: warp instructions issued per
    second (the launch's instruction count from the ncu capture over its live
    CUDA-event duration) against the issue peak, one warp instruction per
    cycle on each of the 4 schedulers of every SM at the sampled SM clock."""
    import torch
    if not traffic or "warp_instructions_per_launch" not in traffic or not sm_mhz:
        return None
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    achieved = traffic["warp_instructions_per_launch"] / (launch_ms * 1e-3) / 1e9
    peak = sms * 4 * sm_mhz * 1e6 / 1e9
    return {"achieved": achieved, "peak": peak, "unit": "G warp-instructions/s", "frac": achieved / peak,
            "instructions_per_launch": traffic["warp_instructions_per_launch"], "sms": sms, "sm_mhz": sm_mhz}


class CpuScan:
    """The reference's own kernels compiled for the CPU (oracle/_ref) on the
    benchmark's scan: the same seeded phantom (the oracle's voxelizer, whose
    sums are the device voxelizer's), and the measured views of SAMPLE_VIEWS
    made as the GPU arm makes them (the projector's ray sums plus the seeded
    noise of each view).  The estimate starts at zero, as the solver's."""

    def __init__(self, seed=SCAN_SEED):
        import numpy as np

        from oracle import ctoracle
        d = ctoracle.make_desc(SCAN["nx"], SCAN["ny"], SCAN["nz"], SCAN["nu"], SCAN["nv"], SCAN["n_views"],
                               SCAN["vx"], SCAN["du"], SCAN["dso"], SCAN["dod"])
        self.ref = ctoracle.RefOracle(d)
        truth = ctoracle.Oracle(d).phantom(phantom_params(seed))
        self.ref._set()
        clean = {}
        for j in SAMPLE_VIEWS:
            s, c = self.ref.trig(j)
            out = np.zeros(self.ref.view_shape, np.float32)
            self.ref.lib.ref_forward_view(truth, out, None, s, c, 0)
            clean[j] = out
        sigma = NOISE * max(float(v.max()) for v in clean.values())
        P = SCAN["nu"] * SCAN["nv"]
        self.b = {j: (clean[j] + sigma * view_noise(j, P, seed).numpy().reshape(self.ref.view_shape)).astype(np.float32)
                  for j in SAMPLE_VIEWS}
        self.vol = np.zeros(self.ref.vol_shape, np.float32)
        del truth

    def sart_view(self, j):
        """Seconds of one SART view: the projection with correction, then the update."""
        import numpy as np
        self.ref._set()
        s, c = self.ref.trig(j)
        corr = np.zeros(self.ref.view_shape, np.float32)
        t0 = time.perf_counter()
        self.ref.lib.ref_forward_view(self.vol, corr, self.b[j].ctypes.data, s, c, 1)
        self.ref.lib.ref_backproject_view(self.vol, corr, BETA, s, c, 1)
        return time.perf_counter() - t0

    def objective_view(self, j):
        """Seconds of the objective's forward projection of one view."""
        import numpy as np
        self.ref._set()
        s, c = self.ref.trig(j)
        fp = np.zeros(self.ref.view_shape, np.float32)
        t0 = time.perf_counter()
        self.ref.lib.ref_forward_view(self.vol, fp, None, s, c, 0)
        return time.perf_counter() - t0

    def iteration(self, views):
        """One iteration's time estimated from a sample: the SART pass and the
        objective's projection from `views` (x n_views/len(views)), FGP from 2
        of its 20 inner iterations (x 10), the TV norm."""
        sart = [self.sart_view(j) for j in views]
        obj = [self.objective_view(j) for j in views]
        t0 = time.perf_counter()
        self.ref.fgp(self.vol, BETA * LAMBDA_TV, 2)
        t_fgp = (time.perf_counter() - t0) * FGP_ITERS / 2.0
        t0 = time.perf_counter()
        self.ref.tv_norm(self.vol)
        t_tv = time.perf_counter() - t0
        n = SCAN["n_views"]
        t_sart, t_obj = sum(sart) / len(views) * n, sum(obj) / len(views) * n
        return {"seconds_per_iter": t_sart + t_obj + t_fgp + t_tv,
                "parts_s": {"sart": t_sart, "objective_fp": t_obj, "fgp": t_fgp, "tv": t_tv},
                "per_view_s": {"views": list(views), "sart": sart, "objective_fp": obj}}


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count()


def cpu_sample_text(cores, per_step):
    n = SCAN["n_views"]
    return (f"reference kernels compiled for the CPU (OpenMP, {cores} threads) on the benchmark scan (same seeded "
            f"phantom and noise): SART and the objective forward projection timed on views 17+64k, k=0..15 "
            f"(16 of {n}, evenly spaced, off the axis angles; {per_step} per step), scaled x{n}/{per_step}; "
            f"2 of {FGP_ITERS} FGP inner iterations (x{FGP_ITERS // 2}); TV norm; 512^3 volume, 1024x768 detector")


def cpu_baseline():
    """The CPU reference timed once on all 16 sample views."""
    scan = CpuScan()
    r = scan.iteration(SAMPLE_VIEWS)
    cores = host_cores()
    sv = r["per_view_s"]["sart"]
    return {"value": 1.0 / r["seconds_per_iter"], "unit": "iter/s", "cores": cores, "kind": "reference",
            "sample": cpu_sample_text(cores, len(SAMPLE_VIEWS)), "seconds_per_iter": r["seconds_per_iter"],
            "parts_s": r["parts_s"], "sart_view_s": {"min": min(sv), "max": max(sv), "mean": sum(sv) / len(sv)}}


def run_reference(args):
    """The reference's CPU implementation on the same scan: each step times 2
    of the 16 sample views in turn (the steps' samples cycle through all 16),
    so that the run stays within a few minutes."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    scan = CpuScan()
    per_step = 2
    times, sart_view = [], {}
    for it in range(args.warmup + args.steps):
        views = [SAMPLE_VIEWS[(per_step * it + i) % len(SAMPLE_VIEWS)] for i in range(per_step)]
        r = scan.iteration(views)
        if it >= args.warmup:
            times.append(r["seconds_per_iter"])
            for j, t in zip(views, r["per_view_s"]["sart"]):
                sart_view.setdefault(j, []).append(t)
    ms = 1000.0 * sum(times) / len(times)
    value = 1000.0 / ms
    cores = host_cores()
    per_view = {j: sum(t) / len(t) for j, t in sorted(sart_view.items())}
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "iter/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": scan_config(world),
        "cpu_baseline": {"value": value, "unit": "iter/s", "cores": cores, "kind": "reference",
                         "sample": cpu_sample_text(cores, per_step)},
        "e2e": {"value": value, "unit": "iter/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "voxel_updates_per_s": value * SCAN["nx"] * SCAN["ny"] * SCAN["nz"] * SCAN["n_views"],
        "sart_view_s": {"per_view": per_view, "min": min(per_view.values()), "max": max(per_view.values())},
    }
    print(json.dumps(line), flush=True)


def profile_fdk(args):
    """A short run for ncu: FDK on the 512^3 scan's geometry restricted to the
    first --profile-fdk views of its 1024 (same angles, the full-circle
    scale factor): cosine weight + ramp of those views through ctr_fdk on a
    geometry of that many views, and the backprojection of the filtered
    views through ctr_fdk_backproject on the 1024-view geometry, twice."""
    import torch

    import gpu_b200
    n = args.profile_fdk
    S = SCAN
    geom = gpu_b200.Geometry(gpu_b200.make_desc(S["nx"], S["ny"], S["nz"], S["vx"], S["nu"], S["nv"], S["du"],
                                                S["dso"], S["dod"], S["n_views"]))
    small = gpu_b200.Geometry(gpu_b200.make_desc(S["nx"], S["ny"], S["nz"], S["vx"], S["nu"], S["nv"], S["du"],
                                                 S["dso"], S["dod"], n, us_rate=360.0 / S["n_views"]))
    truth = torch.zeros(geom.vol_shape, device="cuda")
    geom.phantom_voxelize(phantom_params(2024), truth)
    sino = torch.zeros((n,) + geom.view_shape, device="cuda")
    geom.forward(truth, sino, 0, n)
    vol = torch.zeros(geom.vol_shape, device="cuda")
    e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    e[0].record()
    small.fdk(sino, vol)                            # weighting, ramp, backprojection of n views
    e[1].record()
    filt = sino.clone()                             # any FP32 views serve for timing the backprojection
    e[2].record()
    geom.fdk_backproject(filt, vol, 0, n)
    geom.fdk_backproject(filt, vol, 0, n)
    e[3].record()
    torch.cuda.synchronize()
    print(json.dumps({"profile_fdk": n, "fdk_small_ms": e[0].elapsed_time(e[1]),
                      "backprojection_ms_per_view": e[2].elapsed_time(e[3]) / (2 * n)}), flush=True)


def profile_obj(args):
    """A short run for ncu: the FP16 solver (FISTA, FGP-TV, objective) on the
    512^3 scan restricted to its first 8 views (same angles), two
    iterations: the first's SART forward projections are the plain kind, the
    second's also project the first's objective (the fused kind)."""
    import torch

    import gpu_b200
    n = 8
    geom = gpu_b200.Geometry(gpu_b200.make_desc(SCAN["nx"], SCAN["ny"], SCAN["nz"], SCAN["vx"], SCAN["nu"], SCAN["nv"],
                                                SCAN["du"], SCAN["dso"], SCAN["dod"], n,
                                                us_rate=360.0 / SCAN["n_views"]))
    truth = torch.zeros(geom.vol_shape, device="cuda")
    geom.phantom_voxelize(phantom_params(2024), truth)
    sino = torch.zeros((n,) + geom.view_shape, device="cuda", dtype=torch.float16)
    geom.forward(truth, sino, 0, n)
    del truth
    solver = gpu_b200.Solver(geom, gpu_b200.F16, beta=BETA, lambda_tv=LAMBDA_TV, fgp_iters=FGP_ITERS)
    solver.set_sinogram(sino)
    solver.set_volume(None)
    e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    e[0].record()
    solver.iterate(1, objectives=False)
    e[1].record()
    solver.iterate(1, objectives=False)
    e[2].record()
    torch.cuda.synchronize()
    print(json.dumps({"profile_obj": n, "first_iteration_ms": e[0].elapsed_time(e[1]),
                      "second_iteration_ms": e[1].elapsed_time(e[2])}), flush=True)
    solver.close()


def profile_slabs(args):
    """A short run for ncu: --profile-slabs views of the 4-slab SART pass on the
    512^3 scan (per view 4 partial projections, the ordered combination, 4
    slab updates), FP32, the reference backprojector's arithmetic, tiled;
    after 2 warm-up views."""
    import torch

    import gpu_b200
    n = args.profile_slabs
    geom = gpu_b200.Geometry(gpu_b200.make_desc(SCAN["nx"], SCAN["ny"], SCAN["nz"], SCAN["vx"], SCAN["nu"], SCAN["nv"],
                                                SCAN["du"], SCAN["dso"], SCAN["dod"], SCAN["n_views"]))
    truth = torch.zeros(geom.vol_shape, device="cuda")
    geom.phantom_voxelize(phantom_params(2024), truth)
    sino = torch.zeros((n + 2,) + geom.view_shape, device="cuda")
    geom.forward(truth, sino, 0, n + 2)
    vol = torch.zeros(geom.vol_shape, device="cuda")
    fl = gpu_b200.SART_TILED | gpu_b200.SART_REFERENCE_BP
    geom.sart_pass_slabs(vol, sino, BETA, 4, 0, 2, flags=fl)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    geom.sart_pass_slabs(vol, sino, BETA, 4, 2, n, flags=fl)
    e1.record()
    torch.cuda.synchronize()
    print(json.dumps({"profile_slabs": n, "ms_per_view": e0.elapsed_time(e1) / n}), flush=True)


def profile_views(args):
    """A short run for ncu on the benchmark scan: SART updates of the first
    --profile-views views (one forward + one backprojection launch each) in
    FP32 and FP16, then, with --profile-iteration, one FP16 solver iteration.
    Only the profiled views' sinogram is kept on the device unless the
    iteration needs all of it."""
    import torch

    import gpu_b200
    n = args.profile_views
    tbct = args.workload == "tbct"
    if tbct:     # the tetrahedron-beam scan: its geometry, phantom and relaxation
        geom, ph = tbct_geometry(0)
        n_views, beta, lam = TBCT_SCAN["n_views"], TBCT_BETA, 0.0
    else:
        geom = gpu_b200.Geometry(gpu_b200.make_desc(SCAN["nx"], SCAN["ny"], SCAN["nz"], SCAN["vx"], SCAN["nu"],
                                                    SCAN["nv"], SCAN["du"], SCAN["dso"], SCAN["dod"],
                                                    SCAN["n_views"], fast_sums=args.profile_fast_sums))
        ph = phantom_params(2024)
        n_views, beta, lam = SCAN["n_views"], BETA, LAMBDA_TV
    truth = torch.zeros(geom.vol_shape, device="cuda")
    geom.phantom_voxelize(ph, truth)
    nv = n_views if args.profile_iteration else n
    sino16 = torch.zeros((nv,) + geom.view_shape, device="cuda", dtype=torch.float16)
    geom.forward(truth, sino16, 0, nv)
    sino32 = sino16[:n].float()
    out = {}
    if args.profile_tune:
        out["tune_f16"] = geom.autotune(gpu_b200.F16, n_views=4)
        out["tune_f32"] = geom.autotune(gpu_b200.F32, n_views=4)
        geom.set_shapes(1, 1)
    for name, s in (("f32", sino32), ("f16", sino16)):
        vol = torch.zeros(geom.vol_shape, device="cuda", dtype=s.dtype)
        fl = gpu_b200.SART_TILED | (gpu_b200.SART_REFERENCE_BP if args.profile_refbp else 0)
        fp, bp = geom.sart_views(vol, s, beta, 0, n, flags=fl, timed=True)
        out[name] = {"fp_ms_per_view": fp / n, "bp_ms_per_view": bp / n}
        del vol
    del truth
    if args.profile_iteration:
        # the benchmark's mixed-precision form: the refinement solver
        solver = gpu_b200.Solver(geom, gpu_b200.F16, beta=beta, lambda_tv=lam, fgp_iters=FGP_ITERS,
                                 refine=args.refine)
        solver.set_sinogram(sino16)
        solver.set_volume(None)
        t0 = time.perf_counter()
        solver.iterate(1, objectives=False)     # first iteration: its objective stays pending
        t1 = time.perf_counter()
        solver.iterate(1, objectives=False)     # steady state: projects the previous objective in its SART pass
        out["iteration_s"] = time.perf_counter() - t1
        out["first_iteration_s"] = t1 - t0
        solver.close()
    print(json.dumps({"profile_views": n, "workload": "tbct" if tbct else "scan512", **out}), flush=True)


def batched_scans(n, seed=4):
    """n independent scans: volume edge from {64, 96, 128, 192, 256} over a
    128 mm field of view, 90-720 views, square detector of 96-384 pixels
    covering the magnified volume, source-to-isocentre 600-1200 mm (detector
    at 1.5x that from the source), each with 5-30 seeded ellipsoids (centres
    within 40 mm, semi-axes 5-40 mm, 0.01-0.03 /mm)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        m = int(rng.choice([64, 96, 128, 192, 256]))
        views = int(rng.integers(90, 721))
        det = int(rng.integers(96, 385))
        dso = float(rng.uniform(600.0, 1200.0))
        k = int(rng.integers(5, 31))
        p = np.zeros((k, 10))
        r = 40.0 * np.cbrt(rng.uniform(0, 1, k))
        d = rng.normal(size=(k, 3))
        p[:, 0:3] = r[:, None] * d / np.linalg.norm(d, axis=1, keepdims=True)
        p[:, 3:6] = rng.uniform(5.0, 40.0, (k, 3))
        p[:, 6:9] = rng.uniform(0, 2 * np.pi, (k, 3))
        p[:, 9] = rng.uniform(0.01, 0.03, k)
        fov = 128.0
        half = fov * np.sqrt(2.0) / 2.0
        mag = 1.5 * dso / (dso - half)
        out.append(dict(nx=m, ny=m, nz=m, vx=fov / m, nu=det, nv=det, du=2.0 * half * mag * 1.05 / det, dso=dso,
                        dod=-0.5 * dso, n_views=views, phantom=p))
    return out


def sampling_split(specs, errs):
    """The per-scan errors split by the detector pixel's width at the
    isocentre in voxels: at most one voxel (every voxel met by rays of
    positive chord in every view) or wider (a voxel may meet one ray of a view
    at a grazing chord, and whether the voxel-driven update takes it depends
    on the chord's last bits)."""
    fine, coarse = [], []
    for sp, e in zip(specs, errs):
        pixel_at_iso = sp["du"] * sp["dso"] / (sp["dso"] - sp["dod"])
        (fine if pixel_at_iso <= sp["vx"] else coarse).append(e)
    summ = lambda v: {"scans": len(v), "rmse_max": max(v) if v else None,
                      "rmse_median": sorted(v)[len(v) // 2] if v else None}
    return {"pixel_at_most_one_voxel": summ(fine), "pixel_wider_than_a_voxel": summ(coarse)}


def run_batched(args):
    """Aggregate voxel-updates/s of a batch of uneven scans with BF16 volumes
    (the refinement solver: BF16 copies for the projectors and a BF16
    correction per pass with stochastic rounding, FP32 FISTA state; FP16
    measured data), every iteration of every scan one CUDA graph launch;
    per-scan RMSE and maximum error against the FP64 reference solver on the
    same data after the same iterations, relative to the scan's phantom
    maximum."""
    import torch

    import gpu_b200
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    specs = batched_scans(args.scans, seed=4 + rank)
    geoms, sinos, mus = [], [], []
    for sp in specs:
        g = gpu_b200.Geometry(gpu_b200.make_desc(sp["nx"], sp["ny"], sp["nz"], sp["vx"], sp["nu"], sp["nv"],
                                                 sp["du"], sp["dso"], sp["dod"], sp["n_views"]))
        truth = torch.zeros(g.vol_shape, device=dev)
        g.phantom_voxelize(sp["phantom"], truth)
        mus.append(float(truth.max()))
        sino = torch.zeros((sp["n_views"],) + g.view_shape, device=dev)
        g.forward(truth, sino)
        geoms.append(g)
        sinos.append(sino.to(torch.float16))
        del truth, sino
        if not args.no_tune:
            g.autotune(gpu_b200.BF16, n_views=2)
    flags = 0 if args.no_sr else gpu_b200.SART_STOCHASTIC_ROUND
    batch = gpu_b200.Batch(geoms, gpu_b200.BF16, beta=BETA, lambda_tv=LAMBDA_TV, fgp_iters=FGP_ITERS,
                           sart_flags=flags, refine=args.refine)
    for i, s in enumerate(sinos):
        batch.set_sinogram(i, s)
    iters = args.steps
    stream = torch.cuda.current_stream()
    # the per-view form (one kernel per view and scan, the scans as parallel
    # graph branches), then the persistent pass (every scan's views in one
    # launch per iteration); both give the same bits, the faster is the
    # headline; the volumes compared below are the persistent run's
    timed = {}
    for mode in ("graph_branches", "persistent"):
        batch.set_persistent(mode == "persistent")
        batch.reset()
        batch.iterate(args.warmup)
        batch.reset()
        torch.cuda.synchronize()
        clocks = ClockSampler(local)
        clocks.start()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        objs = batch.iterate(iters)
        e1.record(stream)
        torch.cuda.synchronize()
        timed[mode] = (e0.elapsed_time(e1) / iters, clocks.stop())
    form = min(timed, key=lambda m: timed[m][0])
    ms, clk = timed[form]
    updates = sum(sp["nx"] * sp["ny"] * sp["nz"] * sp["n_views"] for sp in specs)
    # accuracy: the same iterations through the FP64 reference solver on the
    # same (FP16-stored) data, per scan, relative to the scan's phantom maximum
    # The fidelity's trend over the timed iterations (last / first) of this
    # run and of the FP64 solver: a scan whose fidelity grows in FP64 too is
    # one where FISTA over SART diverges at this step, and its error against
    # the FP64 run measures that divergence, not the arithmetic.
    errs, maxs, trend, trend64 = [], [], [], []
    for i, (sp, g) in enumerate(zip(specs, geoms)):
        got = torch.zeros(g.vol_shape, device=dev)
        batch.get_volume_f32(i, got)
        s64 = gpu_b200.Solver(g, gpu_b200.F64, beta=BETA, lambda_tv=LAMBDA_TV, fgp_iters=FGP_ITERS, objective=True)
        s64.set_sinogram(sinos[i])
        s64.set_volume(None)
        o64 = s64.iterate(iters)
        trend.append(float(objs[i][-1][1] / objs[i][0][1]))
        trend64.append(float(o64[-1][1] / o64[0][1]))
        want = torch.zeros(g.vol_shape, device=dev, dtype=torch.float64)
        s64.get_volume(want)
        s64.close()
        dlt = got.double() - want
        errs.append(float(torch.sqrt(torch.mean(dlt * dlt))) / mus[i])
        maxs.append(float(dlt.abs().max()) / mus[i])
        del got, want, dlt
    # per scan and step: the pass's FISTA factor, d = 0, the sum y_k + d, FGP
    # (2 per inner step), the final prox with the rotation; from the second
    # step the previous objective fused (TV + reduce, 2-level reduce); after
    # the last step the objective (FP, 2 reduce, TV, reduce); plus, per step,
    # the one persistent launch of every scan's views, or per view and scan a
    # forward and a walk launch
    launches = sum((2 + 2 * FGP_ITERS) * iters + 4 * (iters - 1) + 5 for sp in specs)
    launches += iters if form == "persistent" else sum(2 * sp["n_views"] * iters for sp in specs)
    other = "graph_branches" if form == "persistent" else "persistent"
    notes = {"graph_branches": "one kernel per view and scan, the scans as parallel graph branches",
             "persistent": "every scan's SART views in one persistent launch per iteration, its blocks handed "
                           "out as a data flow over the scans' phases"}
    line = {
        "metric": "batched SART-FISTA-TV voxel-updates/s", "value": updates * 1000.0 / ms,
        "unit": "voxel-updates/s", "n_gpus": 1, "steps": iters, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": f"bf16 storage for the projectors (refinement: FP32 FISTA state, {refine_note(args)}, FP16 "
                 f"sinogram), f32 arithmetic"
                 + ("" if args.no_sr or args.refine == 2 else ", stochastic rounding of the correction's updates"),
        "data": "synthetic",
        "config": {"workload": f"{len(specs)} uneven scans (volumes 64-256^3, 90-720 views, 96^2-384^2 detectors, "
                               f"DSO 600-1200 mm), one CUDA graph launch per iteration of all scans",
                   "form": f"{form}: {notes[form]}",
                   "scans": [{k: sp[k] for k in ("nx", "n_views", "nu", "dso")} for sp in specs],
                   "l2": "inputs > L2 (sum of the scans' volumes and sinograms)"},
        "iter_per_s": 1000.0 / ms,
        other: {"ms_per_step": timed[other][0], "voxel_updates_per_s": updates * 1000.0 / timed[other][0],
                "note": notes[other]},
        "error_vs_fp64": {"rmse": {"max": max(errs), "median": sorted(errs)[len(errs) // 2]},
                          "max_abs": {"max": max(maxs), "median": sorted(maxs)[len(maxs) // 2]},
                          "per_scan_rmse": errs, "iterations": iters,
                          "relative_to": "each scan's phantom maximum, against the FP64 reference solver",
                          "fidelity_last_over_first": {"this_run": trend, "fp64": trend64},
                          "diverging_in_fp64": [i for i, t in enumerate(trend64) if t > 1.0],
                          "by_sampling": sampling_split(specs, errs)},
        "clocks": clk, "gpu_launches": launches,
        "launch_shapes": [g.shapes() for g in geoms],
    }
    batch.close()
    print(json.dumps(line), flush=True)


LARGE = dict(nx=1024, ny=1024, nz=1024, vx=0.25, nu=1024, nv=1024, du=0.3, dso=1000.0, dod=-500.0, n_views=1024)


def run_large(args):
    """1024^3 (0.25 mm) / 1024 views / 1024x1024 detector (0.3 mm): iterations/s
    of FP32 and of the BF16 / FP16 refinement solver on a seeded 100-ellipsoid
    phantom, and the RMSE and maximum error of every reconstruction against
    the FP64 reference solver after the same iterations (relative to the
    phantom's maximum).  --large-plain adds plain FP16 storage (no
    refinement), whose error grows with the iterations."""
    import numpy as np
    import torch

    import gpu_b200
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    L = LARGE
    geom = gpu_b200.Geometry(gpu_b200.make_desc(L["nx"], L["ny"], L["nz"], L["vx"], L["nu"], L["nv"], L["du"],
                                                L["dso"], L["dod"], L["n_views"]))
    rng = np.random.default_rng(1024)
    k = 100
    ph = np.zeros((k, 10))
    r = 40.0 * np.cbrt(rng.uniform(0, 1, k))
    d = rng.normal(size=(k, 3))
    ph[:, 0:3] = r[:, None] * d / np.linalg.norm(d, axis=1, keepdims=True)
    ph[:, 3:6] = rng.uniform(5.0, 40.0, (k, 3))
    ph[:, 6:9] = rng.uniform(0, 2 * np.pi, (k, 3))
    ph[:, 9] = rng.uniform(0.01, 0.03, k)
    truth = torch.zeros(geom.vol_shape, device=dev)
    geom.phantom_voxelize(ph, truth)
    mu_max = float(truth.max())
    sino32 = torch.zeros((L["n_views"],) + geom.view_shape, device=dev)
    geom.forward(truth, sino32)
    del truth
    stream = torch.cuda.current_stream()
    out = {}
    vols = {}
    sino16 = sino32.to(torch.float16)
    # BF16 and FP16: the refinement solver (16-bit copies, FP32 FISTA state,
    # FP16 measured data); a 16-bit correction takes stochastic rounding in
    # BF16.  f16_plain: FP16 storage without refinement.
    modes = [("f32", gpu_b200.F32, torch.float32), ("bf16", gpu_b200.BF16, torch.bfloat16),
             ("f16", gpu_b200.F16, torch.float16)]
    if args.large_plain:
        modes.append(("f16_plain", gpu_b200.F16, torch.float16))
    for mode, vdt, tdt in modes:
        sino = sino32 if tdt == torch.float32 else sino16
        tuned = geom.autotune(vdt, n_views=2)
        flags = gpu_b200.SART_STOCHASTIC_ROUND if mode == "bf16" else 0
        solver = gpu_b200.Solver(geom, vdt, beta=BETA, lambda_tv=LAMBDA_TV, fgp_iters=FGP_ITERS, sart_flags=flags,
                                 refine=0 if mode in ("f32", "f16_plain") else args.refine)
        solver.set_sinogram(sino)
        solver.set_volume(None)
        for _ in range(args.warmup):
            solver.iterate(1)
        solver.set_volume(None)
        torch.cuda.synchronize()
        clocks = ClockSampler(local)
        clocks.start()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        solver.iterate(args.steps)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        vol = torch.zeros(geom.vol_shape, device=dev)
        solver.get_volume_f32(vol)
        solver.close()
        vols[mode] = vol
        out[mode] = {"ms_per_step": ms, "iter_per_s": 1000.0 / ms, "clocks": clocks.stop(),
                     "launch_shapes": [tuned["fp_shape"], tuned["bp_shape"]],
                     "voxel_updates_per_s": 1000.0 / ms * L["nx"] * L["ny"] * L["nz"] * L["n_views"]}
    del sino16
    # the FP64 reference solver on the same (FP32) data for the same iterations
    f64 = gpu_b200.Solver(geom, gpu_b200.F64, beta=BETA, lambda_tv=LAMBDA_TV, fgp_iters=FGP_ITERS, objective=False)
    f64.set_sinogram(sino32)
    f64.set_volume(None)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    f64.iterate(args.steps, objectives=False)
    e1.record(stream)
    torch.cuda.synchronize()
    ref = f64.get_volume(torch.zeros(geom.vol_shape, device=dev, dtype=torch.float64))
    f64.close()
    for mode in vols:
        dlt = vols[mode].double() - ref
        out[mode]["rmse_vs_fp64"] = float(torch.sqrt(torch.mean(dlt * dlt))) / mu_max
        out[mode]["max_err_vs_fp64"] = float(dlt.abs().max()) / mu_max
        out[mode]["speedup_vs_f32"] = out["f32"]["ms_per_step"] / out[mode]["ms_per_step"]
        # where the largest error sits: voxel, distance from the axis relative
        # to the reconstruction cylinder's radius, and the two values there
        q = int(dlt.abs().argmax())
        k, rem = divmod(q, L["nx"] * L["ny"])
        j, i = divmod(rem, L["nx"])
        r = float(np.hypot(i - (L["nx"] / 2 - 0.5), j - (L["ny"] / 2 - 0.5))) / (L["nx"] / 2 - 0.5)
        out[mode]["max_err_at"] = {"ijk": [i, j, k], "r_over_fov": r, "value": float(vols[mode].view(-1)[q]),
                                   "fp64": float(ref.view(-1)[q])}
        del dlt
    line = {"metric": "SART-FISTA-TV iter/s, 1024^3 x 1024 views, BF16/FP16 vs FP32", "value": out["bf16"]["iter_per_s"],
            "unit": "iter/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": out["bf16"]["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None,
            "dtype": f"bf16 storage for the projectors (refinement: FP32 FISTA state, {refine_note(args)}, FP16 "
                     f"sinogram" + (", stochastic rounding" if args.refine == 1 else "") + "), f32 arithmetic",
            "data": "synthetic",
            "config": {"workload": "1024^3 x 0.25 mm, 1024 views, 1024x1024 detector x 0.3 mm, DSO 1000 mm, "
                                   "DOD -500 mm, 100 seeded ellipsoids, noiseless Siddon sinogram",
                       "l2": "inputs > L2"},
            "modes": out, "phantom_max": mu_max, "fp64_ms_per_iteration": e0.elapsed_time(e1) / args.steps,
            "errors_relative_to": "the phantom's maximum attenuation, against the FP64 reference solver after the "
                                  "same iterations"}
    print(json.dumps(line), flush=True)


# The tetrahedron-beam program's own configuration (T42/main_recon.cu:41-120)
# in millimetres: 512^3 voxels of 0.1 mm, 64 sources stacked along z, each
# with a band of 16 detector rows x 1024 columns of 0.12 mm, DSO 200 mm,
# DOD -200 mm, 360 views 1 degree apart; relaxation 2/Lip_con = 2/32 and
# lambda_TV = 0 (SART + FISTA, no TV prox), the objective every iteration.
TBCT_SCAN = dict(nx=512, ny=512, nz=512, vx=0.1, nu=1024, nv=16, n_sources=64, du=0.12, dso=200.0, dod=-200.0,
                 n_views=360, us_rate=1.0)
TBCT_BETA = 2.0 / 32.0   # T42/main_recon.cu's Lip_con = 32, as the cone-beam loop's


def tbct_geometry(seed):
    """The tetrahedron-beam geometry on the current device and its phantom:
    the 512^3 scan's ellipsoids scaled to the 51.2 mm volume (attenuation
    scaled up alike)."""
    import gpu_b200
    T = TBCT_SCAN
    desc = gpu_b200.make_desc(T["nx"], T["ny"], T["nz"], T["vx"], T["nu"], T["nv"], T["du"], T["dso"], T["dod"],
                              T["n_views"], us_rate=T["us_rate"], ct_style=3, n_sources=T["n_sources"])
    ph = phantom_params(2024 + seed)
    ph[:, 0:6] *= 0.2
    ph[:, 9] *= 5.0
    return gpu_b200.Geometry(desc), ph


def tbct_desc_oracle():
    from oracle import ctoracle
    T = TBCT_SCAN
    return ctoracle.make_desc(T["nx"], T["ny"], T["nz"], T["nu"], T["nv"], T["n_views"], T["vx"], T["du"], T["dso"],
                              T["dod"], us_rate=T["us_rate"], ct_style=3, n_sources=T["n_sources"])


def cpu_baseline_tbct(budget_s=20.0):
    """The tetrahedron-beam program's kernels compiled for the CPU
    (oracle/_ref/libctref_tbct.so) on this host's cores, on a bounded sample
    of one iteration scaled to a full one: S views of the SART pass (forward
    projection of all 64 sources' rays, backprojection, update) and of the
    objective's forward projection (x 360/S).  The FISTA step and the norms
    are host loops over the volume and are left out (a few hundred ms)."""
    import numpy as np

    from oracle import ctoracle
    ref = ctoracle.RefOracle(tbct_desc_oracle())
    nviews = TBCT_SCAN["n_views"]
    rng = np.random.default_rng(0)
    vol = rng.uniform(0.0, 0.02, ref.vol_shape).astype(np.float32)
    b_view = rng.uniform(0.0, 1.0, ref.view_shape).astype(np.float32)
    ref._set()

    def sart_view(j):
        s, c = ref.trig(j)
        corr = np.zeros(ref.view_shape, np.float32)
        ref.lib.ref_forward_view(vol, corr, b_view.ctypes.data, s, c, 1)
        ref.lib.ref_backproject_view(vol, corr, TBCT_BETA, s, c, 1)

    # the first sampled view also sizes the sample to the budget
    t0 = time.perf_counter()
    sart_view(nviews // 2)
    t_one = time.perf_counter() - t0
    s_views = max(1, min(16, int(0.8 * budget_s / max(t_one, 1e-3))))
    views = [nviews // 2] + [int((q + 0.5) * nviews / s_views) for q in range(1, s_views)]
    t0 = time.perf_counter()
    for j in views[1:]:
        sart_view(j)
    t_sart = (time.perf_counter() - t0 + t_one) / len(views) * nviews
    t0 = time.perf_counter()
    for j in views:
        s, c = ref.trig(j)
        fp = np.zeros(ref.view_shape, np.float32)
        ref.lib.ref_forward_view(vol, fp, None, s, c, 0)
    t_obj = (time.perf_counter() - t0) / len(views) * nviews
    t_iter = t_sart + t_obj
    cores = os.cpu_count()
    try:
        cores = len(os.sched_getaffinity(0))
    except AttributeError:
        pass
    return {
        "value": 1.0 / t_iter, "unit": "iter/s", "cores": cores, "kind": "reference",
        "sample": (f"the tetrahedron-beam program's kernels compiled for the CPU (OpenMP, {cores} threads): SART on "
                   f"{len(views)} of {nviews} views and the objective forward projection on the same views (scaled "
                   f"x{nviews}/{len(views)}); 512^3 volume, 64 sources x 16 x 1024 detector"),
        "seconds_per_iter": t_iter, "parts_s": {"sart": t_sart, "objective_fp": t_obj},
    }


def run_tbct(args):
    """The tetrahedron-beam scan: SART + FISTA iterations/s (FP32 and FP16
    storage) with the objective, end to end with host buffers, the SART
    update kernel against the HBM roofline, and the CPU reference beside it."""
    import torch

    import gpu_b200
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    T = TBCT_SCAN
    geom, ph = tbct_geometry(rank)
    vshape, sshape = geom.vol_shape, (T["n_views"],) + geom.view_shape
    V = T["nx"] * T["ny"] * T["nz"]
    P = geom.view_shape[0] * geom.view_shape[1]
    truth = torch.zeros(vshape, device=dev)
    geom.phantom_voxelize(ph, truth)
    sino32 = torch.zeros(sshape, device=dev)
    geom.forward(truth, sino32)
    gen = torch.Generator(device=dev).manual_seed(77 + rank)
    sino32 += 0.005 * sino32.max() * torch.randn(sshape, device=dev, generator=gen)
    del truth
    stream = torch.cuda.current_stream()
    runs, tuned = {}, {}
    for mode, vdt, sdt in (("f32", gpu_b200.F32, torch.float32), ("f16", gpu_b200.F16, torch.float16)):
        tuned[mode] = geom.autotune(vdt, n_views=4)
        sino = sino32 if sdt == torch.float32 else sino32.to(sdt)
        solver = gpu_b200.Solver(geom, vdt, beta=TBCT_BETA, lambda_tv=0.0, fgp_iters=0, fista=True,
                                 objective=True, use_graph=True)
        solver.set_sinogram(sino)
        solver.set_volume(None)
        solver.iterate(args.warmup)
        torch.cuda.synchronize()
        clocks = ClockSampler(local)
        clocks.start()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        objs = solver.iterate(args.steps).tolist()
        e1.record(stream)
        torch.cuda.synchronize()
        runs[mode] = {"ms": e0.elapsed_time(e1) / args.steps, "clocks": clocks.stop(), "objective_last": objs[-1],
                      "solver": solver, "sino": sino}

    # end to end with host buffers (FP16 storage): sinogram in, one iteration,
    # volume out, every step; the objectives read at the end
    geom.set_shapes(tuned["f16"]["fp_shape"], tuned["f16"]["bp_shape"])
    solver, sino = runs["f16"]["solver"], runs["f16"]["sino"]
    h_sino = sino.cpu().pin_memory()
    h_vol = torch.empty(vshape, dtype=torch.float16).pin_memory()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    k0 = solver.iteration
    for _ in range(args.steps):
        sino.copy_(h_sino, non_blocking=True)
        solver.iterate(1, objectives=False)
        solver.get_volume(h_vol)
    solver.objectives(k0 + 1, args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / args.steps
    h2d = h_sino.numel() * h_sino.element_size()
    d2h = h_vol.numel() * h_vol.element_size() + 3 * 8

    # T42's own backprojection arithmetic (CTR_SART_REFERENCE_BP: the SART pass
    # equals the tetrahedron-beam program's bit for bit), FP32 as the reference
    geom.set_shapes(tuned["f32"]["fp_shape"], tuned["f32"]["bp_shape"])
    refbp = gpu_b200.Solver(geom, gpu_b200.F32, beta=TBCT_BETA, lambda_tv=0.0, fgp_iters=0, fista=True,
                            objective=True, use_graph=True, sart_flags=gpu_b200.SART_REFERENCE_BP)
    refbp.set_sinogram(runs["f32"]["sino"])
    refbp.set_volume(None)
    refbp.iterate(1)
    torch.cuda.synchronize()
    e0.record(stream)
    refbp.iterate(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    refbp_ms = e0.elapsed_time(e1) / args.steps
    refbp.close()
    # the program's default build (Number_of_Devices 4, T42/main_recon.cu:17): its
    # slab SART and row-split objective projector, bit-exact with it
    dflt = gpu_b200.Solver(geom, gpu_b200.F32, beta=TBCT_BETA, lambda_tv=0.0, fgp_iters=0, fista=True,
                           objective=True, use_graph=True, sart_flags=gpu_b200.SART_REFERENCE_BP)
    dflt.set_slabs(4)
    dflt.set_sinogram(runs["f32"]["sino"])
    dflt.set_volume(None)
    dflt.iterate(1)
    torch.cuda.synchronize()
    e0.record(stream)
    dflt.iterate(2)
    e1.record(stream)
    torch.cuda.synchronize()
    dflt_ms = e0.elapsed_time(e1) / 2
    dflt.close()

    # per-kernel times of the SART projectors (32 views spread over the scan)
    kern = {}
    for mode in ("f32", "f16"):
        geom.set_shapes(tuned[mode]["fp_shape"], tuned[mode]["bp_shape"])
        vol = torch.zeros(vshape, device=dev, dtype=torch.float32 if mode == "f32" else torch.float16)
        geom.sart_views(vol, runs[mode]["sino"], TBCT_BETA, 0, 4, flags=gpu_b200.SART_TILED)
        fp_t = bp_t = 0.0
        nt = 32
        for j in range(nt):
            f_ms, b_ms = geom.sart_views(vol, runs[mode]["sino"], TBCT_BETA, (j * 97) % T["n_views"], 1,
                                         flags=gpu_b200.SART_TILED, timed=True)
            fp_t += f_ms
            bp_t += b_ms
        kern[mode] = {"fp_ms": fp_t / nt, "bp_ms": bp_t / nt}
        del vol
    for m in runs.values():
        m["solver"].close()

    peak, peak_kind = measured_peak_hbm()
    bp_bytes = 2 * V * 2 + 4 * P            # SART update of one view, FP16 volume: volume in + out, the FP32 correction
    achieved = bp_bytes / (kern["f16"]["bp_ms"] * 1e-3) / 1e9
    traffic = profiled_traffic("roofline_traffic_tbct.json")
    value = 1000.0 / runs["f16"]["ms"]
    line = {
        "metric": "TBCT SART-FISTA iter/s & voxel-updates/s, 512^3 x 360 views x 64 sources, FP16 vs FP32, 1 B200",
        "value": value, "unit": "iter/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": runs["f16"]["ms"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f16 storage, f32 arithmetic", "data": "synthetic",
        "config": {"workload": "tetrahedron-beam SART+FISTA iteration with objective (lambda_TV 0), 512^3 x 0.1 mm, "
                               "360 views, 64 sources x 16 rows x 1024 columns x 0.12 mm, DSO 200 mm, DOD -200 mm",
                   "phantom": "40 ellipsoids + 200 spheres (seeded, scaled to the volume), Siddon projections "
                              "+ 0.5% noise", "l2": "inputs > L2 (1.5 GB sinogram)"},
        "voxel_updates_per_s": value * V * T["n_views"],
        "f32": {"iter_per_s": 1000.0 / runs["f32"]["ms"], "ms_per_step": runs["f32"]["ms"],
                "voxel_updates_per_s": 1000.0 / runs["f32"]["ms"] * V * T["n_views"]},
        "f16_over_f32": runs["f32"]["ms"] / runs["f16"]["ms"],
        "reference_bp_f32": {"iter_per_s": 1000.0 / refbp_ms, "ms_per_step": refbp_ms,
                             "note": "CTR_SART_REFERENCE_BP: the tetrahedron-beam program's backprojection "
                                     "arithmetic, SART pass bit-exact with it"},
        "reference_default_build_f32": {"iter_per_s": 1000.0 / dflt_ms, "ms_per_step": dflt_ms,
                                        "note": "the program's default Number_of_Devices=4 build's SART + FISTA "
                                                "loop with its objective, bit-exact with it, on one B200 "
                                                "(ctr_solver_set_slabs(4), CTR_SART_REFERENCE_BP, FP32); 2 timed "
                                                "iterations after 1"},
        "objective_last": {m: runs[m]["objective_last"] for m in runs},
        "e2e": {"value": 1000.0 / e2e_ms, "unit": "iter/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "roofline": {"bound": "hbm", "kernel": "k_sart_walk, tetrahedron beam (SART update, f16 volume, tiled)",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind, "traffic": (traffic or {}).get("bytes_per_launch"),
                     "algorithmic_bytes_per_launch": bp_bytes, "launch_ms": kern["f16"]["bp_ms"],
                     "issue": issue_roofline(traffic, kern["f16"]["bp_ms"], runs["f16"]["clocks"]["sm_mhz"], dev)},
        "kernels_ms": kern, "launch_shapes": tuned, "clocks": runs["f16"]["clocks"],
        "clocks_f32": runs["f32"]["clocks"],
        # per step: tile, FP + BP per view, untile, FISTA momentum; objectives fused as in the 512^3 scan
        "gpu_launches": (2 + 2 * T["n_views"] + 1) * args.steps + 5 * (args.steps - 1) + 6,
    }
    if not args.no_cpu_baseline:
        try:
            cb = cpu_baseline_tbct()
            line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
            line["cpu_baseline_parts_s"] = cb["parts_s"]
        except Exception as e:  # the CPU leg must not hide the GPU result
            line["cpu_baseline"] = {"value": None, "error": str(e)[:200]}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.profile_views:
        return profile_views(args)
    if args.profile_fdk:
        return profile_fdk(args)
    if args.profile_slabs:
        return profile_slabs(args)
    if args.profile_obj:
        return profile_obj(args)
    if args.workload == "batched":
        return run_batched(args)
    if args.workload == "large":
        return run_large(args)
    if args.workload == "tbct":
        return run_tbct(args)
    import numpy as np
    import torch
    import torch.distributed as dist

    import gpu_b200
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    init_replicas(world, "nccl")
    dev = torch.device("cuda", local)
    desc = gpu_b200.make_desc(SCAN["nx"], SCAN["ny"], SCAN["nz"], SCAN["vx"], SCAN["nu"], SCAN["nv"], SCAN["du"],
                              SCAN["dso"], SCAN["dod"], SCAN["n_views"])
    geom = gpu_b200.Geometry(desc)
    # the mixed-precision run's projections with fused ray sums
    # (CTR_GEOM_FAST_SUMS) unless --exact-sums; the FP32 run keeps the
    # reference's sequence
    geoms = {"f32": geom, "mixed": geom}
    if args.fast_sums:
        geoms["mixed"] = gpu_b200.Geometry(gpu_b200.make_desc(
            SCAN["nx"], SCAN["ny"], SCAN["nz"], SCAN["vx"], SCAN["nu"], SCAN["nv"], SCAN["du"], SCAN["dso"],
            SCAN["dod"], SCAN["n_views"], fast_sums=True))
    vshape, sshape = geom.vol_shape, (SCAN["n_views"],) + geom.view_shape
    V = SCAN["nx"] * SCAN["ny"] * SCAN["nz"]
    P = SCAN["nu"] * SCAN["nv"]

    # synthetic scan: seeded phantom, its Siddon projections + Gaussian noise of
    # 0.5% of the largest ray sum of the sample views, drawn per view from a
    # seeded CPU generator (the CPU arm draws the same noise for its views)
    seed = SCAN_SEED + rank
    truth = torch.zeros(vshape, device=dev)
    geom.phantom_voxelize(phantom_params(seed), truth)
    truth_max = float(truth.max())
    sino32 = torch.zeros(sshape, device=dev)
    geom.forward(truth, sino32)
    sigma = NOISE * float(sino32[SAMPLE_VIEWS].max())
    for j in range(SCAN["n_views"]):
        sino32[j] += sigma * view_noise(j, P, seed).to(dev).view(sshape[1:])
    del truth
    mixed_dt = torch.float16 if args.mixed == "f16" else torch.bfloat16
    mixed_code = gpu_b200.F16 if args.mixed == "f16" else gpu_b200.BF16
    # the measured data are stored in FP16 for either 16-bit volume type (BF16's
    # 8-bit mantissa would change the data by itself)
    sino16 = sino32.to(torch.float16)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    def job_ms(x):
        return max_over_ranks(x, world, dev)

    runs = {}
    stream = torch.cuda.current_stream()
    tuned = {}
    # mixed precision: the refinement solver (FP32 FISTA state, 16-bit copies
    # for the projectors, each pass accumulated into a 16-bit correction
    # against the FP32 residual), the form that meets the accuracy bar
    for mode, vdt, sino in (("f32", gpu_b200.F32, sino32), ("mixed", mixed_code, sino16)):
        tuned[mode] = geoms[mode].autotune(vdt, n_views=4)   # launch shapes; results do not depend on them
        solver = gpu_b200.Solver(geoms[mode], vdt, beta=BETA, lambda_tv=LAMBDA_TV, fgp_iters=FGP_ITERS, fista=True,
                                 objective=True, use_graph=True, refine=args.refine if mode == "mixed" else 0,
                                 sart_flags=gpu_b200.SART_STOCHASTIC_ROUND if vdt == gpu_b200.BF16 else 0)
        solver.set_sinogram(sino)
        solver.set_volume(None)
        solver.iterate(args.warmup)
        barrier()
        clocks = ClockSampler(local)
        clocks.start()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        # the K steps in one call, as a driver runs its iterations: the
        # objective of each iteration but the last rides on the next SART pass
        objs = solver.iterate(args.steps).tolist()
        e1.record(stream)
        barrier()
        ms = e0.elapsed_time(e1) / args.steps
        runs[mode] = {"ms": job_ms(ms), "clocks": clocks.stop(), "objective_last": objs[-1]}
        runs[mode]["solver"] = solver
        runs[mode]["sino"] = sino

    # accuracy (outside the timed regions): the FP64 reference solver on the
    # same scan (FP32 measured data) for the same number of iterations; the
    # errors of the mixed-precision estimate (its FP32 x_k) and of the FP32
    # run, relative to the phantom's maximum attenuation.  The FP64 run's
    # state after 5 iterations also scores the FP64 ray-box entry variant.
    n_acc = args.warmup + args.steps
    n_early = min(5, n_acc)
    acc, entry64 = {}, {}
    try:
        def err(v, ref):
            d = v.double() - ref
            return {"rmse": float(torch.sqrt(torch.mean(d * d))) / truth_max,
                    "max_abs": float(d.abs().max()) / truth_max}

        f64 = gpu_b200.Solver(geom, gpu_b200.F64, beta=BETA, lambda_tv=LAMBDA_TV, fgp_iters=FGP_ITERS, fista=True,
                              objective=False)
        f64.set_sinogram(sino32)
        f64.set_volume(None)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        f64.iterate(n_early, objectives=False)
        e1.record(stream)
        torch.cuda.synchronize()
        f64_ms = e0.elapsed_time(e1) / n_early
        ref_early = f64.get_volume(torch.empty(vshape, device=dev, dtype=torch.float64))
        if n_acc > n_early:
            f64.iterate(n_acc - n_early, objectives=False)
        ref = f64.get_volume(torch.empty(vshape, device=dev, dtype=torch.float64))
        f64.close()
        for mode in ("mixed", "f32"):
            acc[mode] = err(runs[mode]["solver"].get_volume_f32(torch.empty(vshape, device=dev)), ref)
        mixed_acc = {"rmse": acc["mixed"]["rmse"], "max_abs": acc["mixed"]["max_abs"], "f32": acc["f32"],
                     "relative_to": "the phantom's maximum attenuation, against the FP64 reference solver",
                     "iterations": n_acc, "fp64_ms_per_iteration": f64_ms, "bar": 1e-3,
                     "meets_bar": acc["mixed"]["rmse"] <= 1e-3}
        del ref
        # CTR_GEOM_ENTRY_F64: the ray-box entry/exit in FP64 (the traversal in
        # FP32); kernel times per view and the FP32 solver's error after
        # n_early iterations, beside the default FP32 entry
        d64 = gpu_b200.make_desc(SCAN["nx"], SCAN["ny"], SCAN["nz"], SCAN["vx"], SCAN["nu"], SCAN["nv"], SCAN["du"],
                                 SCAN["dso"], SCAN["dod"], SCAN["n_views"], entry64=True)
        for key, gm in (("entry_f32", geom), ("entry_f64", gpu_b200.Geometry(d64))):
            gm.set_shapes(tuned["f32"]["fp_shape"], tuned["f32"]["bp_shape"])
            s = gpu_b200.Solver(gm, gpu_b200.F32, beta=BETA, lambda_tv=LAMBDA_TV, fgp_iters=FGP_ITERS, fista=True,
                                objective=False)
            s.set_sinogram(sino32)
            s.set_volume(None)
            s.iterate(n_early, objectives=False)
            entry64[key] = err(s.get_volume_f32(torch.empty(vshape, device=dev)), ref_early)
            s.close()
            vol = torch.zeros(vshape, device=dev)
            gm.sart_views(vol, sino32, BETA, 0, 4, flags=gpu_b200.SART_TILED)
            fp_t = bp_t = 0.0
            for j in range(16):
                f_ms, b_ms = gm.sart_views(vol, sino32, BETA, (j * 97) % SCAN["n_views"], 1,
                                           flags=gpu_b200.SART_TILED, timed=True)
                fp_t += f_ms
                bp_t += b_ms
            entry64[key].update({"fp_ms_per_view": fp_t / 16, "bp_ms_per_view": bp_t / 16})
            del vol
        entry64["iterations"] = n_early
        entry64["relative_to"] = "the phantom's maximum attenuation, against the FP64 reference solver"
        del ref_early
    except Exception as e:  # an accuracy side figure must not hide the timing
        mixed_acc = {"error": str(e)[:300]}

    # end to end through the public API with host buffers: every step copies the
    # measured sinogram in from pinned host memory, runs one iteration and reads
    # the reconstructed volume back; the steps' objectives are read at the end
    # (each is projected inside the next step's SART traversal, the last one
    # by that read, all inside the timed region)
    mode = "mixed"
    geoms[mode].set_shapes(tuned[mode]["fp_shape"], tuned[mode]["bp_shape"])
    solver, sino = runs[mode]["solver"], runs[mode]["sino"]
    h_sino = sino.cpu().pin_memory()
    h_vol = torch.empty(vshape, dtype=mixed_dt).pin_memory()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    k0 = solver.iteration
    for _ in range(args.steps):
        sino.copy_(h_sino, non_blocking=True)
        solver.iterate(1, objectives=False)
        solver.get_volume(h_vol)
    e2e_objs = solver.objectives(k0 + 1, args.steps)
    e1.record(stream)
    barrier()
    e2e_ms = job_ms(e0.elapsed_time(e1) / args.steps)
    h2d = h_sino.numel() * h_sino.element_size()
    d2h = h_vol.numel() * h_vol.element_size() + 3 * 8

    # per-kernel durations of the SART projector kernels, from CUDA events the
    # library records around each launch on this stream (32 views spread over the scan)
    kern = {}
    for mode in ("f32", "mixed"):
        gk = geoms[mode]
        gk.set_shapes(tuned[mode]["fp_shape"], tuned[mode]["bp_shape"])
        sino = runs[mode]["sino"]
        vol = torch.zeros(vshape, device=dev, dtype=torch.float32 if mode == "f32" else mixed_dt)
        tl = gpu_b200.SART_TILED                                      # the solver's layout
        gk.sart_views(vol, sino, BETA, 0, 4, flags=tl)                # warm-up
        fp_t = bp_t = 0.0
        nt = 32
        for j in range(nt):
            f_ms, b_ms = gk.sart_views(vol, sino, BETA, (j * 97) % SCAN["n_views"], 1, flags=tl, timed=True)
            fp_t += f_ms
            bp_t += b_ms
        kern[mode] = {"fp_ms": fp_t / nt, "bp_ms": bp_t / nt}
        del vol

    # the iteration without the objective (the reference's loop evaluates it
    # every iteration, so the headline keeps it)
    # (side figures below: a few timed iterations each)
    side_steps = min(args.steps, 3)
    geoms["mixed"].set_shapes(tuned["mixed"]["fp_shape"], tuned["mixed"]["bp_shape"])
    noobj = gpu_b200.Solver(geoms["mixed"], mixed_code, beta=BETA, lambda_tv=LAMBDA_TV, fgp_iters=FGP_ITERS,
                            fista=True, objective=False, use_graph=True, refine=args.refine)
    noobj.set_sinogram(runs["mixed"]["sino"])
    noobj.set_volume(None)
    noobj.iterate(1)
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    noobj.iterate(side_steps)
    e1.record(stream)
    barrier()
    noobj_ms = job_ms(e0.elapsed_time(e1) / side_steps)
    noobj.close()

    # the reference backprojector's arithmetic (CTR_SART_REFERENCE_BP: the
    # SART pass equals the reference's bit for bit), FP32 as the reference
    geom.set_shapes(tuned["f32"]["fp_shape"], tuned["f32"]["bp_shape"])
    refbp = gpu_b200.Solver(geom, gpu_b200.F32, beta=BETA, lambda_tv=LAMBDA_TV, fgp_iters=FGP_ITERS, fista=True,
                            objective=True, use_graph=True, sart_flags=gpu_b200.SART_REFERENCE_BP)
    refbp.set_sinogram(runs["f32"]["sino"])
    refbp.set_volume(None)
    refbp.iterate(1)
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    refbp.iterate(side_steps)
    e1.record(stream)
    barrier()
    refbp_ms = job_ms(e0.elapsed_time(e1) / side_steps)
    refbp.close()
    vtmp = torch.zeros(vshape, device=dev)
    geom.sart_views(vtmp, runs["f32"]["sino"], BETA, 0, 4, flags=gpu_b200.SART_TILED | gpu_b200.SART_REFERENCE_BP)
    rb_bp = 0.0
    for j in range(32):
        _, b_ms = geom.sart_views(vtmp, runs["f32"]["sino"], BETA, (j * 97) % SCAN["n_views"], 1,
                                     flags=gpu_b200.SART_TILED | gpu_b200.SART_REFERENCE_BP, timed=True)
        rb_bp += b_ms
    # the reference's default build's whole loop (Number_of_Devices 4): the
    # solver with its slab pass and backprojection arithmetic, FP32, every
    # iteration's objective projected on its own (bit-exact with that build)
    dflt = gpu_b200.Solver(geom, gpu_b200.F32, beta=BETA, lambda_tv=LAMBDA_TV, fgp_iters=FGP_ITERS, fista=True,
                           objective=True, use_graph=True, sart_flags=gpu_b200.SART_REFERENCE_BP)
    dflt.set_slabs(4)
    dflt.set_sinogram(runs["f32"]["sino"])
    dflt.set_volume(None)
    dflt.iterate(1)
    barrier()
    e0.record(stream)
    dflt.iterate(2)
    e1.record(stream)
    barrier()
    dflt_ms = job_ms(e0.elapsed_time(e1) / 2)
    dflt.close()
    # the reference's default build (Number_of_Devices 4, its z-slab SART,
    # bit-exact with its multi-GPU kernels) on this one GPU: per view 4 slab
    # partial projections, the ordered combination, 4 slab updates
    slab4 = {}
    for key, fl in (("reference_bp", gpu_b200.SART_TILED | gpu_b200.SART_REFERENCE_BP),
                    ("engine", gpu_b200.SART_TILED)):
        geom.sart_pass_slabs(vtmp, runs["f32"]["sino"], BETA, 4, 0, 4, flags=fl)          # warm-up
        barrier()
        e0.record(stream)
        geom.sart_pass_slabs(vtmp, runs["f32"]["sino"], BETA, 4, 100, 32, flags=fl)
        e1.record(stream)
        barrier()
        slab4[key] = e0.elapsed_time(e1) / 32
    del vtmp

    # ray-voxel intersections of one pass over all views (Siddon segments of
    # every ray, counted once per geometry); an iteration visits each of them
    # three times: SART forward projection, SART backprojection, objective
    nseg = torch.empty(sshape[1:], device=dev, dtype=torch.int32)
    hsh = torch.empty(sshape[1:], device=dev, dtype=torch.int64)
    lng = torch.empty(sshape[1:], device=dev, dtype=torch.float32)
    zero = torch.zeros(vshape, device=dev)
    segs = torch.zeros((), device=dev, dtype=torch.int64)
    for j in range(SCAN["n_views"]):
        geom.forward_trace(zero, j, nseg, hsh, lng)
        segs += nseg.sum(dtype=torch.int64)
    segs_per_pass = int(segs.item())
    del nseg, hsh, lng

    # FDK of the same scan (FP32), reported beside the iterative numbers
    geom.fdk(sino32, zero)
    barrier()
    e0.record(stream)
    geom.fdk(sino32, zero)
    e1.record(stream)
    barrier()
    fdk_ms = job_ms(e0.elapsed_time(e1))
    del zero

    peak, peak_kind = measured_peak_hbm()
    s_v = 2  # mixed storage bytes
    bp_bytes = 2 * V * s_v + 4 * P            # BP with SART update, per view: volume in + out, the FP32 correction
    bp_ms = kern["mixed"]["bp_ms"]
    achieved = bp_bytes / (bp_ms * 1e-3) / 1e9
    traffic = profiled_traffic()

    line = None
    if rank == 0:
        ms_mixed = runs["mixed"]["ms"]
        ms_f32 = runs["f32"]["ms"]
        value = job_rate(ms_mixed, world)
        # every step of the refinement solver: the pass's FISTA factor, FP + BP
        # per view, the sum y_k + d, FGP (2 per inner step), the final prox with
        # the rotation; objective of steps 1..K-1 fused into the next pass (TV +
        # reduce, 2-level reduce of the partials); of step K separate (FP of all
        # views, 2 reduce, TV, reduce)
        launches_per_step = 1 + 2 * SCAN["n_views"] + 1 + 2 * FGP_ITERS + 1
        launches_total = launches_per_step * args.steps + 4 * (args.steps - 1) + 5
        line = {
            "metric": METRIC, "value": value, "unit": "iter/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_mixed, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None,
            "dtype": f"{args.mixed} storage for the projectors (refinement: FP32 FISTA state, {refine_note(args)}, "
                     f"FP16 sinogram), f32 arithmetic" + (", fused ray sums" if args.fast_sums else ""),
            "data": "synthetic",
            "config": scan_config(world),
            "accuracy_vs_fp64": mixed_acc,
            "entry_f64": entry64,
            "voxel_updates_per_s": value * V * SCAN["n_views"],
            "ray_voxel_intersections_per_s": value * 3 * segs_per_pass,
            "ray_voxel_intersections_per_pass": segs_per_pass,
            "ms_per_step_without_objective": noobj_ms,
            "reference_bp_f32": {"iter_per_s": job_rate(refbp_ms, world), "ms_per_step": refbp_ms,
                                 "bp_ms_per_view": rb_bp / 32,
                                 "note": "CTR_SART_REFERENCE_BP: the reference backprojector's arithmetic, "
                                         "SART pass bit-exact with the reference"},
            "reference_default_build_f32": {"iter_per_s": job_rate(dflt_ms, world), "ms_per_step": dflt_ms,
                                            "note": "the reference's default Number_of_Devices=4 build's SART + "
                                                    "FISTA + FGP-TV loop, bit-exact with it, on one B200 "
                                                    "(ctr_solver_set_slabs(4), CTR_SART_REFERENCE_BP, FP32); "
                                                    "2 timed iterations after 1"},
            "slabs4_f32": {"ms_per_view_reference_bp": slab4["reference_bp"], "ms_per_view_engine": slab4["engine"],
                           "one_device_ms_per_view": {"f32_fp": kern["f32"]["fp_ms"], "reference_bp": rb_bp / 32},
                           "note": "the reference's default Number_of_Devices=4 build: z-slab SART views (4 slab "
                                   "partial projections, the ordered combination, 4 slab updates) on one B200, "
                                   "views 100-131, FP32, tiled; bit-exact with its multi-GPU kernels"},
            "fdk_ms": fdk_ms,
            "f32": {"iter_per_s": job_rate(ms_f32, world), "ms_per_step": ms_f32,
                    "voxel_updates_per_s": job_rate(ms_f32, world) * V * SCAN["n_views"]},
            "mixed_over_f32": ms_f32 / ms_mixed,
            "objective_last": {"f32": runs["f32"]["objective_last"], "mixed": runs["mixed"]["objective_last"]},
            "e2e": {"value": job_rate(e2e_ms, world), "unit": "iter/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "roofline": {"bound": "hbm", "kernel": "k_sart_walk (SART update, f16 volume, tiled layout)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_kind": peak_kind,
                         "traffic": (traffic or {}).get("bytes_per_launch"),
                         "algorithmic_bytes_per_launch": bp_bytes,
                         "launch_ms": bp_ms,
                         "issue": issue_roofline(traffic, bp_ms, runs["mixed"]["clocks"]["sm_mhz"], dev)},
            "kernels_ms": kern,
            "launch_shapes": tuned,
            "clocks": runs["mixed"]["clocks"],
            "clocks_f32": runs["f32"]["clocks"],
            "gpu_launches": launches_total,
        }
    for m in runs.values():
        m["solver"].close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        if world == 1 and not args.no_cpu_baseline:
            try:
                cb = cpu_baseline()
                line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
            except Exception as e:  # the CPU leg must not hide the GPU result
                line["cpu_baseline"] = {"value": None, "error": str(e)[:200]}
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
