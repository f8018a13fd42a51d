"""Benchmark of the McSART engine: SART iterations/s on one or more B200s.

Workload (default, --config motion256): the motion-compensated McSART problem of
volume 256x256x160 at 1 mm, flat detector 512x384 at 0.776 mm, SAD/SDD
1000/1500 mm, 660 views over 360 degrees at 15 views/s with a 5DCT breathing
model.  One step is one outer iteration = one image-update pass over all 660
views (warp, project, residual, backproject, normalise, inverse warp, update)
plus one DVF-update pass over 659 views, i.e. host_AUMISART with op_iter =
[1, 0].  --config motion128 selects the 128x128x96 problem (detector 256x192 at
1.2 mm, 360 views), static64 the static 64^3 one (60 views).  Inputs are seeded
synthetic data of that shape (phantom, smooth random DVF, projections of the
warped phantom), generated outside the timed region.

  value   iterations/s through the device-resident driver, inputs in HBM,
          L2 flushed (256 MiB write) before every timed step, device time by
          CUDA events; whole job over N replicas (one per GPU, no data-path
          collective: the path does not shard, see the design notes).
  e2e     iterations/s through the host-pointer entry point mcsart_aumisart
          (host_AUMISART's interface): H2D of the step's inputs from pinned
          memory, the iteration, D2H of image, residuals, norms, alpha_x.
  --impl reference   the reference's path on the host cores: the FP32 OpenMP
          transcription of the reference kernels (the reference has no CPU
          code of its own), each step a bounded sample of views, the
          iterations/s extrapolated linearly in view count; beside it, the
          reference's own CUDA build timed on the GPU over whole steps.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--config", default="motion256")
    ap.add_argument("--cpu-views", type=int, default=0,
                    help="views per pass in the CPU sample (0 = auto)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the 16-bit-storage and split-sum side measurements")
    ap.add_argument("--profile-steps", type=int, default=0,
                    help="only run this many untimed steps inside the NVTX range "
                         "'mcsart_step' (for a profiler's launch list) and exit")
    ap.add_argument("--profile-subset", type=int, default=1,
                    help="with --profile-steps: image passes in ordered subsets of this many "
                         "views (not the drop-in; 1 = the reference's view-by-view loop)")
    ap.add_argument("--no-autotune", action="store_true",
                    help="run the driver with its built-in launch shapes instead of tuning "
                         "them for the workload in the warm-up (mcsart_autotune)")
    ap.add_argument("--kernel-case", default="", choices=["", "fp", "bp", "warp"],
                    help="only time single calls of one kernel at the workload's size "
                         "(projector, backprojector or warp through the C ABI, CUDA events, "
                         "--steps calls after --warmup) and exit")
    return ap.parse_args()


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms in the background."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        under = [s for s in sm if mx and s > 0.5 * mx] or sm
        return {"sm_mhz": float(np.median(under)) if under else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------------- problem
def build_problem(ctx, torch, cfg_name: str, seed: int = 0):
    """Seeded problem; projections made by the engine's own warp + projector."""
    from mcsart_b200 import synthetic as S
    p = S.make_problem(cfg_name, seed)
    g = p.geo
    dev = torch.device("cuda", torch.cuda.current_device())
    truth = torch.as_tensor(p.truth, device=dev)
    fields = [torch.as_tensor(f, device=dev) for f in p.fields] if p.fields else None
    proj = torch.empty((p.cfg.n_views, g["nb"], g["na"]), dtype=torch.float32, device=dev)
    tmp = torch.empty_like(truth)
    for v in range(p.cfg.n_views):
        src = truth
        if fields is not None:
            ctx.host_deform(tmp, truth, g["nx"], g["ny"], g["nz"],
                            np.float32(p.volumes[v] - p.volumes[0]),
                            np.float32(p.flows[v] - p.flows[0]), *fields)
            src = tmp
        ctx.host_projection(proj[v], src, float(p.angles[v]), g["SO"], g["SD"], g["da"], g["na"],
                            g["ai"], g["db"], g["nb"], g["bi"], g["nx"], g["ny"], g["nz"])
    ctx.synchronize()
    return p, proj, fields


def algorithmic_bytes(p) -> dict:
    """Compulsory bytes per launch of the driver's kernels (FP32 storage)."""
    g = p.geo
    V = g["nx"] * g["ny"] * g["nz"]
    P = g["na"] * g["nb"]
    return {
        # read the warped volume, the measured view; write residual + (residual, ones) pairs
        "fp_image": 4 * V + 4 * P + 4 * P + 8 * P,
        # read img, img0, ones; read the measured view; write the pairs
        "fp_motion": 12 * V + 4 * P + 8 * P,
        # read the pairs; write the ratio volume
        "bp_div": 8 * P + 4 * V,
        # the same in the DVF pass when it runs as its own launch
        "bp_div_motion": 8 * P + 4 * V,
        # read volume (+ its update), write volume and its y-fastest copy
        "bp_div_add": 8 * P + 12 * V,
        # read img, 6 fields; write the warped volume in the layout the
        # view's projector reads (x- or y-fastest)
        "warp_fwd": 4 * V + 24 * V + 4 * V,
        # read ratio, 6 fields, img; write img and (texture model, the
        # default) its 3D-array copy
        "warp_back_add": 4 * V + 24 * V + 8 * V + 4 * V,
        # read img, 6 fields; write img0 and ones in the layout the view's
        # projector reads
        "motion_prep": 4 * V + 24 * V + 8 * V,
        # read ratio, img, read+write 6 fields
        "field_update": 8 * V + 48 * V,
        # the two above in one pass: read ratio, img, read+write 6 fields,
        # write img0 and ones in the layout the next view's projector reads
        "field_update_prep": 8 * V + 48 * V + 8 * V,
        # the DVF pass's backprojector and field update in one kernel: read
        # the pairs, img, read+write 6 fields, write img0 and ones (the ratio
        # stays on chip)
        "bp_field_update_prep": 8 * P + 4 * V + 48 * V + 8 * V,
    }


# DRAM bytes per launch of the workload's kernels (dram__bytes.sum.per_second
# x gpu__time_duration.sum), from one ncu capture of each in the benchmark
# step (cold cache, FP32 storage, built-in launch shapes); summaries with the
# commands are kept under profiles/.
NCU_DRAM_BYTES = {
    "motion256": {"fp_motion": 132078080, "fp_image": 42956032, "bp_div": 2872064,
                  "field_update_prep": 613819647, "bp_field_update_prep": 573643608},
}

# Issue-slot utilisation (smsp__issue_active) of the projector and
# backprojector from the same captures: these kernels are bound by issue and
# latency, not by HBM.
NCU_ISSUE_ACTIVE = {"motion256": {"fp_image": 0.570, "fp_motion": 0.602, "bp_div": 0.817,
                                  "bp_field_update_prep": 0.663}}

# Views per pass of the CPU samples: the engine line's cpu_baseline leg
# (about 10 s of CPU work) and each step of the reference arm (a few seconds,
# so that --steps 20 --warmup 5 ends within a few minutes).
CPU_VIEWS = {"static64": 60, "motion128": 160, "motion256": 16, "clinical512": 4}
REF_ARM_VIEWS = {"static64": 30, "motion128": 64, "motion256": 6, "clinical512": 2}


def measured_peaks() -> dict:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    except (OSError, KeyError, ValueError):
        return {"hbm_gbs": 6650.0, "source": "fallback"}


# --------------------------------------------------------------- CPU side
def cpu_sample(p, proj_host, views: int, threads: int):
    """One image pass and one DVF-update pass of the FP32 OpenMP transcription
    over `views` views each; returns (seconds, iterations/s extrapolated)."""
    from oracle import oracle as O
    O.set_num_threads(threads)
    nv = p.cfg.n_views
    views = max(2, min(views, nv))
    op = np.array([1, 0] if p.fields is not None else [1], np.int32)
    it = dict(n_iter=len(op), op_iter=op, n_views=nv, outIter=1,
              volumes=p.volumes, flows=p.flows, angles=p.angles, **{"lambda": p.cfg.lam})
    t0 = time.perf_counter()
    O.aumisart(p.img0, proj_host, p.geo, it, p.fields, prec="cpu", view_lo=0, view_hi=views)
    dt = time.perf_counter() - t0
    # image pass: `views` views; motion pass: views-1 views (starts at view 1)
    # motion: `views` image-pass views and views-1 DVF-pass views (it starts
    # at view 1); static: `views` image-pass views
    motion = p.fields is not None
    per_view = dt / ((2 * views - 1) if motion else views)
    t_iter = per_view * ((nv + (nv - 1)) if motion else nv)
    return dt, 1.0 / t_iter, views


def cpu_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_model() -> str:
    """The host CPU's model name, recorded beside the CPU baseline."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def reference_gpu_step(p, steps: int = 3) -> dict:
    """The reference's own CUDA code (host_AUMISART rebuilt from its unmodified
    sources into oracle/_ref) timed on this GPU over `steps` whole steps of
    the same workload (after one untimed call): its host-pointer call, with
    its per-call allocations, copies and device reset, each call in a fresh
    process as the reference resets the device.  Reported beside the CPU
    arm, not as the arm's value."""
    lib = os.path.join(ROOT, "oracle", "_ref", "libmcsart_ref.so")
    if not os.path.exists(lib):
        return {"unavailable": "the rebuilt reference library is not present"}
    try:
        import torch
        if not torch.cuda.is_available():
            return {"unavailable": "no CUDA device"}
    except ImportError:
        return {"unavailable": "torch is not importable"}
    from oracle import ref_runner
    ref = ref_runner.Ref()
    g = p.geo
    # measured projections made by the reference's own warp and projector
    proj = ref.motion_projections(p.truth, p.fields, p.volumes, p.flows, p.angles, g)
    op = np.array([1, 0], np.int32) if p.fields is not None else np.array([1], np.int32)
    it = {"n_iter": len(op), "op_iter": op, "n_views": p.cfg.n_views,
          "lambda": p.cfg.lam, "outIter": 1, "volumes": p.volumes, "flows": p.flows,
          "angles": p.angles}
    secs = []
    for _ in range(steps + 1):  # the first call is a warm-up
        r = ref_runner.aumisart(np.zeros_like(p.truth), proj, g, it, p.fields)
        secs.append(float(r["seconds"]))
    s = np.array(secs[1:])
    t = float(np.median(s))
    return {"value": 1.0 / t, "unit": "iterations/s", "seconds_per_step": t,
            "seconds_min": float(s.min()), "seconds_max": float(s.max()),
            "kind": "reference CUDA build, host_AUMISART with host pointers",
            "steps_timed": int(len(s))}


def run_reference_arm(args, rank: int):
    """--impl reference: the reference's path on the host cores (FP32 OpenMP port)."""
    if rank != 0:
        return
    from mcsart_b200 import synthetic as S
    p = S.make_problem(args.config, 0)
    # measured projections from the oracle port of the reference projector (CPU)
    from oracle import oracle as O
    threads = cpu_threads()
    O.set_num_threads(threads)
    proj = np.zeros((p.cfg.n_views, p.cfg.nb, p.cfg.na), np.float32)
    views = args.cpu_views or REF_ARM_VIEWS.get(args.config, 8)
    # only the views the sample touches need measured data
    for v in range(views + 1):
        vol = O.deform(p.truth, np.float32(p.volumes[v] - p.volumes[0]),
                       np.float32(p.flows[v] - p.flows[0]), p.fields, prec="cpu")
        proj[v] = O.projection(vol, float(p.angles[v]), p.geo, prec="cpu")
    for _ in range(args.warmup):
        cpu_sample(p, proj, views, threads)
    times, rates = [], []
    for _ in range(args.steps):
        dt, rate, _ = cpu_sample(p, proj, views, threads)
        times.append(dt)
        rates.append(rate)
    value = float(np.median(rates))
    sample = (f"{views} views of the image pass + {views - 1} of the DVF-update pass of "
              f"{args.config} per step, extrapolated linearly to {p.cfg.n_views} + "
              f"{p.cfg.n_views - 1} views")
    # a step of this arm is the bounded sample: ms_per_step is its measured
    # duration, value the iterations/s extrapolated from it
    line = {"impl": "reference", "metric": "McSART iterations/s", "value": value,
            "unit": "iterations/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * float(np.median(times)),
            "ms_per_iteration_extrapolated": 1000.0 / value, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config_dict(p, args),
            "cpu_baseline": {"value": value, "unit": "iterations/s", "cores": threads,
                             "kind": "port", "sample": sample, "cpu_model": cpu_model(),
                             "host_cpus": os.cpu_count()},
            "e2e": {"value": value, "unit": "iterations/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "note": "the reference has no CPU implementation; this is the FP32 OpenMP "
                    "transcription of its kernels and host_AUMISART loop",
            "reference_gpu": reference_gpu_step(p)}
    print(json.dumps(line), flush=True)


def max_over_ranks(x: float, device: str = "cuda") -> float:
    """The maximum of x over all ranks of the default process group (x if none)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def config_dict(p, args) -> dict:
    c = p.cfg
    return {"workload": f"{args.config}: {c.name}; one step = host_AUMISART with op_iter [1, 0]",
            "volume": [c.nx, c.ny, c.nz], "voxel_mm": c.vox_mm, "detector": [c.na, c.nb],
            "pitch_mm": c.pitch_mm, "views": c.n_views, "sad_sdd_mm": [1000, 1500],
            "lambda": c.lam, "l2": "flushed before every timed step (256 MiB write)"}


# -------------------------------------------------------------- GPU side
def run_kernel_case(args, ctx, torch, stream):
    """One kernel of the workload at its full size, on a smooth random volume
    (the projector's and backprojector's memory traffic depends on the
    geometry, not on the values): --steps calls timed with CUDA events on the
    context's stream, after --warmup untimed ones."""
    from mcsart_b200 import synthetic as S
    cfg = S.CONFIGS[args.config]
    g = S.geometry(cfg)
    shape = (g["nz"], g["ny"], g["nx"])
    gen = torch.Generator(device="cuda").manual_seed(5)
    img = torch.rand(shape, device="cuda", generator=gen)
    proj = torch.rand((g["nb"], g["na"]), device="cuda", generator=gen)
    out_v = torch.empty_like(img)
    out_p = torch.empty_like(proj)
    geo = (g["SO"], g["SD"], g["da"], g["na"], g["ai"], g["db"], g["nb"], g["bi"], g["nx"],
           g["ny"], g["nz"])
    fields = ([torch.rand(shape, device="cuda", generator=gen) * 4 - 2 for _ in range(6)]
              if args.kernel_case == "warp" else None)
    angle = 0.3  # rays driven along x: the projector reads the volume's y-fastest copy

    def call():
        if args.kernel_case == "fp":
            ctx.host_projection(out_p, img, angle, *geo)
        elif args.kernel_case == "bp":
            ctx.host_backprojection(out_v, proj, angle, *geo)
        else:
            ctx.host_deform(out_v, img, g["nx"], g["ny"], g["nz"], 0.7, -0.3, *fields)

    for _ in range(max(args.warmup, 0)):
        call()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    for e0, e1 in ev:
        e0.record(stream)
        call()
        e1.record(stream)
    torch.cuda.synchronize()
    ms = [a.elapsed_time(b) for a, b in ev]
    V, P = g["nx"] * g["ny"] * g["nz"], g["na"] * g["nb"]
    abytes = {"fp": 4 * V + 4 * P, "bp": 4 * P + 4 * V, "warp": 4 * V + 24 * V + 4 * V}
    print(json.dumps({"kernel_case": args.kernel_case, "config": args.config,
                      "volume": [g["nx"], g["ny"], g["nz"]], "detector": [g["na"], g["nb"]],
                      "calls": args.steps, "ms_median": float(np.median(ms)),
                      "ms_min": float(np.min(ms)),
                      "algorithmic_bytes": abytes[args.kernel_case],
                      "note": "each call is one C-ABI call (the projector's includes the "
                              "y-fastest copy of the volume for x-driven rays)"}), flush=True)


def run_batch_config(args, ctx, torch, stream, m, rank, world):
    """--config batch8: the 8 seeded uneven problems (96x96x64 .. 256x256x128,
    detectors 192x128 .. 512x384, 120 .. 660 views) reconstructed together by
    mcsart_batch_run, image passes in ordered subsets of 10 views.  One step =
    one outer iteration (image pass + DVF-update pass) of every problem.
    value = problem-iterations per second; beside it the same work as one
    mcsart_aumisart_device call per problem after another, and the voxel-ray
    updates per second of the batch."""
    from mcsart_b200 import synthetic as S
    cfgs = S.batch_configs()
    op = np.array([1, 0], np.int32)
    probs = []
    for i, cfg in enumerate(cfgs):
        p, proj, fields = build_problem(ctx, torch, cfg, seed=200 * (rank + 1) + i)
        g = p.geo
        probs.append(dict(geo=g, n_views=cfg.n_views, lambda_=p.cfg.lam, angles=p.angles,
                          volumes=p.volumes, flows=p.flows, proj=proj,
                          img=torch.zeros((g["nz"], g["ny"], g["nx"]), device="cuda"),
                          fields=torch.stack(fields).contiguous()))
        del fields
    vox_rays = sum(q["geo"]["nx"] * q["geo"]["ny"] * q["geo"]["nz"] * q["n_views"] for q in probs)
    flush = torch.empty(256 * 2**20 // 4, dtype=torch.float32, device="cuda")
    out = {}
    for label, storage in (("f32", m.F32), ("bf16", m.BF16)):
        opt = m.default_options(subset=S.BATCH_SUBSET, storage=storage, autotune=1)
        if storage == m.F32:
            batch = probs
        else:
            batch = [dict(q, proj=q["proj"].to(torch.bfloat16),
                          fields=q["fields"].to(torch.bfloat16)) for q in probs]

        def batch_step():
            ctx.batch_run(batch, n_iter=2, op_iter=op, options=opt)

        def seq_step():
            for q in batch:
                ctx.aumisart_device(n_iter=2, op_iter=op, options=opt, **q)

        res = {}
        for name, fn in (("batch", batch_step), ("sequential", seq_step)):
            for _ in range(args.warmup):
                fn()
            torch.cuda.synchronize()
            ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                  for _ in range(args.steps)]
            for e0, e1 in ev:
                flush.fill_(1.0)
                e0.record(stream)
                fn()
                e1.record(stream)
            torch.cuda.synchronize()
            t = max_over_ranks(sum(a.elapsed_time(b) for a, b in ev) / 1000.0)
            res[name] = len(probs) * args.steps / t * world
        out[label] = res
        del batch
    line = {"metric": "McSART iterations/s (all problems)", "value": out["f32"]["batch"],
            "unit": "problem-iterations/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * len(probs) / out["f32"]["batch"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": "batch8: 8 uneven motion-compensated problems, one outer "
                                   "iteration each per step, ordered subsets of 10 views",
                       "problems": [c.name for c in cfgs],
                       "l2": "flushed before every timed step (256 MiB write)"},
            "voxel_ray_updates_per_s": out["f32"]["batch"] / len(probs) * vox_rays,
            "sequential_f32": out["f32"]["sequential"], "batch_bf16": out["bf16"]["batch"],
            "sequential_bf16": out["bf16"]["sequential"],
            "tuned_shapes": {c.name: ctx.tuning_get(q["geo"]) for c, q in zip(cfgs, probs)}}
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference_arm(args, rank)
        return

    import torch
    import torch.distributed as dist
    import mcsart_b200 as m

    torch.cuda.set_device(local)
    dist_on = world > 1
    if dist_on:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx = m.Context(local, stream=stream)
    if args.kernel_case:
        if rank == 0:
            run_kernel_case(args, ctx, torch, stream)
        ctx.close()
        if dist_on:
            dist.destroy_process_group()
        return
    if args.config == "batch8":
        run_batch_config(args, ctx, torch, stream, m, rank, world)
        ctx.close()
        if dist_on:
            dist.destroy_process_group()
        return
    p, proj, fields = build_problem(ctx, torch, args.config, seed=rank)
    g = p.geo
    nv = p.cfg.n_views
    V = g["nx"] * g["ny"] * g["nz"]
    # motion workloads: an image pass and a DVF-update pass; static: an image pass
    op = np.array([1, 0] if fields is not None else [1], np.int32)
    img = torch.zeros((g["nz"], g["ny"], g["nx"]), dtype=torch.float32, device="cuda")
    F = torch.stack(fields).contiguous() if fields is not None else None
    F0 = F.clone() if F is not None else None
    norm = torch.zeros(len(op) * nv, device="cuda")
    resid = torch.zeros((nv, g["nb"], g["na"]), device="cuda")
    flush = torch.empty(256 * 2**20 // 4, dtype=torch.float32, device="cuda")

    def step(opts, img_t, F_t):
        ctx.aumisart_device(geo=g, n_views=nv, lambda_=p.cfg.lam, angles=p.angles,
                            volumes=p.volumes, flows=p.flows, img=img_t, proj=proj, fields=F_t,
                            resid=resid, norm=norm, n_iter=len(op), op_iter=op, options=opts)

    def timed(opts, steps, warmup, img_t, F_t, count_launches=False):
        for _ in range(warmup):
            step(opts, img_t, F_t)
        torch.cuda.synchronize()
        if dist_on:
            dist.barrier()
        torch.cuda.synchronize()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(steps)]
        l0 = ctx.launches
        for e0, e1 in ev:
            flush.fill_(1.0)  # evict L2 between steps (not timed)
            e0.record(stream)
            step(opts, img_t, F_t)
            e1.record(stream)
        torch.cuda.synchronize()
        launches = ctx.launches - l0
        if dist_on:
            dist.barrier()
        total = max_over_ranks(sum(a.elapsed_time(b) for a, b in ev) / 1000.0)
        return total, launches

    # FP32, texture-model warp, reference summation order; launch shapes tuned
    # for the workload on the first (warm-up) run, which changes no result bit
    drop_in = m.default_options(autotune=0 if args.no_autotune else 1)
    if args.profile_steps:
        prof_opt = (drop_in if args.profile_subset <= 1 else
                    m.default_options(autotune=drop_in.autotune, subset=args.profile_subset))
        for _ in range(args.profile_steps):
            torch.cuda.nvtx.range_push("mcsart_step")
            step(prof_opt, img, F)
            torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        if rank == 0:
            print(json.dumps({"profile_steps": args.profile_steps, "launches": ctx.launches}))
        ctx.close()
        if dist_on:
            dist.destroy_process_group()
        return
    clocks = ClockSampler(local)
    clocks.start()
    total, launches = timed(drop_in, args.steps, args.warmup, img, F)
    clk = clocks.stop()
    per_rank = args.steps / total
    value = per_rank * world
    vox_ray = value * V * nv

    # per-kernel device time of one profiled step (graphs bypassed while profiling)
    ctx.profile_begin()
    step(drop_in, img, F)
    prof = ctx.profile_end()
    kernel_ms = {k: v[1] for k, v in prof.items()}
    tot_ms = sum(kernel_ms.values())
    top = max(prof, key=lambda k: prof[k][1])
    abytes = algorithmic_bytes(p)
    peaks = measured_peaks()
    top_launch_ms = prof[top][1] / prof[top][0]
    achieved = abytes.get(top, 0) / (top_launch_ms / 1000.0) / 1e9
    roofline = {"bound": "hbm", "kernel": top, "achieved": achieved, "peak": peaks["hbm_gbs"],
                "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"],
                "traffic": NCU_DRAM_BYTES.get(args.config, {}).get(top),
                "issue_active_ncu": NCU_ISSUE_ACTIVE.get(args.config) or None,
                "peak_source": peaks["source"], "launch_ms": top_launch_ms,
                "algorithmic_bytes_per_launch": abytes.get(top, 0),
                "share": {k: round(v / tot_ms, 4) for k, v in kernel_ms.items()}}

    # end to end through the host-pointer entry point (host_AUMISART's interface)
    pin = lambda a: torch.as_tensor(np.ascontiguousarray(a)).pin_memory().numpy()
    h_img = pin(np.zeros((g["nz"], g["ny"], g["nx"]), np.float32))
    h_proj = pin(proj.cpu().numpy())
    h_fields = [pin(f.cpu().numpy()) for f in fields] if fields is not None else [None] * 6
    o_img, o_ax = pin(np.zeros_like(h_img)), pin(np.zeros_like(h_img))
    o_proj = pin(np.zeros((nv, g["nb"], g["na"]), np.float32))
    o_norm = pin(np.zeros(len(op) * nv, np.float32))
    errw = np.zeros(nv, np.float32)

    def e2e_step():
        ctx.host_AUMISART(o_img, o_proj, o_norm, o_ax, h_img, h_proj, g["nx"], g["ny"], g["nz"],
                          g["na"], g["nb"], 1, nv, len(op), op, g["da"], g["db"], g["ai"], g["bi"],
                          g["SO"], g["SD"], 1.0, p.cfg.lam, p.volumes, p.flows, errw, p.angles,
                          *h_fields)

    for _ in range(max(1, args.warmup)):
        e2e_step()
    torch.cuda.synchronize()
    if dist_on:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    e2e_total = max_over_ranks(time.perf_counter() - t0)
    e2e = {"value": args.steps / e2e_total * world, "unit": "iterations/s",
           "h2d_bytes_per_step": int(h_img.nbytes + h_proj.nbytes +
                                     (6 * h_img.nbytes if fields is not None else 0)),
           "d2h_bytes_per_step": int(o_img.nbytes + o_proj.nbytes + o_norm.nbytes + o_ax.nbytes),
           "api": "mcsart_aumisart (host pointers, pinned)"}

    extras = {}
    # side measurements: a few steps each, after two untimed ones
    xsteps = max(1, min(args.steps, 5))
    if not args.no_extras:
        # side measurements: the split-sum (Kahan) projector in FP32, 16-bit
        # storage of fields, projections and projector inputs with the
        # reference-order projector and exact trilinear warps, and ordered
        # subsets
        for name, kw in (("split_kahan_f32", dict(fp_sum=2)),
                         ("bf16_storage", dict(storage=m.BF16, interp=m.INTERP_EXACT)),
                         ("bf16_storage_texture_warp", dict(storage=m.BF16)),
                         ("f16_storage", dict(storage=m.F16, interp=m.INTERP_EXACT)),
                         # ordered subsets of 8 views (a different algorithm:
                         # one projector and one backprojector launch per subset)
                         ("subsets_of_8_f32", dict(subset=8)),
                         ("subsets_of_8_bf16", dict(subset=8, storage=m.BF16,
                                                    interp=m.INTERP_EXACT))):
            o = m.default_options(autotune=drop_in.autotune, **kw)
            if o.storage == m.F32:
                pr, Ft = proj, (F0.clone() if F0 is not None else None)
            else:
                dt = torch.bfloat16 if o.storage == m.BF16 else torch.float16
                pr, Ft = proj.to(dt), (F0.to(dt) if F0 is not None else None)
            img2 = torch.zeros_like(img)

            def st(o=o, pr=pr, Ft=Ft, img2=img2):
                ctx.aumisart_device(geo=g, n_views=nv, lambda_=p.cfg.lam, angles=p.angles,
                                    volumes=p.volumes, flows=p.flows, img=img2, proj=pr,
                                    fields=Ft, resid=resid, norm=norm, n_iter=len(op), op_iter=op,
                                    options=o)
            for _ in range(2):
                st()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(xsteps):
                st()
            e1.record(stream)
            torch.cuda.synchronize()
            ext = max_over_ranks(e0.elapsed_time(e1) / 1000.0)
            extras[name] = {"value": xsteps / ext * world,
                            "unit": "iterations/s"}
            if name.startswith("subsets") or name.startswith("bf16"):
                # where the time goes in this mode (one step, graphs bypassed)
                ctx.profile_begin()
                st()
                pr_ = ctx.profile_end()
                extras[name]["kernel_ms_per_step"] = {k: round(v[1], 2) for k, v in pr_.items()
                                                      if v[1] >= 0.05}

        # four independent problems of this workload (different seeds) run
        # concurrently through mcsart_batch_run: problems per second x steps
        nb_ = 4
        batch = []
        for s in range(nb_):
            pb, prb, fb = build_problem(ctx, torch, args.config, seed=100 * (rank + 1) + s)
            batch.append(dict(geo=pb.geo, n_views=nv, lambda_=pb.cfg.lam, angles=pb.angles,
                              volumes=pb.volumes, flows=pb.flows,
                              img=torch.zeros_like(img), proj=prb,
                              fields=torch.stack(fb).contiguous() if fb else None))
        for _ in range(2):
            ctx.batch_run(batch, n_iter=len(op), op_iter=op, options=drop_in)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(xsteps):
            ctx.batch_run(batch, n_iter=len(op), op_iter=op, options=drop_in)
        e1.record(stream)
        torch.cuda.synchronize()
        ext = max_over_ranks(e0.elapsed_time(e1) / 1000.0)
        extras["batch_4_problems"] = {
            "value": nb_ * xsteps / ext * world, "unit": "iterations/s (all problems)",
            "note": "4 independent problems of the workload, one mcsart_batch_run per step"}
        del batch

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = cpu_threads()
        h_proj_np = proj.cpu().numpy()
        views = args.cpu_views or CPU_VIEWS.get(args.config, 8)
        dt, rate, views = cpu_sample(p, h_proj_np, views, threads)
        cpu = {"value": rate, "unit": "iterations/s", "cores": threads, "kind": "port",
               "sample": f"{views} views of the image pass + {views - 1} of the DVF-update "
                         f"pass ({dt:.1f} s), extrapolated to {nv} + {nv - 1} views",
               "cpu_model": cpu_model(), "host_cpus": os.cpu_count()}

    if rank == 0:
        line = {"metric": "McSART iterations/s", "value": value, "unit": "iterations/s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": 1000.0 * total / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": config_dict(p, args), "voxel_ray_updates_per_s": vox_ray,
                "e2e": e2e, "gpu_launches": int(launches), "roofline": roofline,
                "cpu_baseline": cpu, "clocks": clk, "kernel_ms_per_step": kernel_ms,
                "launch_shapes": {"autotuned": bool(drop_in.autotune),
                                  "variants_fp1_fp3_bp_warp_fup": ctx.tuning_get(g)},
                "extras": extras}
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist_on:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
