#!/usr/bin/env python
"""Throughput benchmark of the B200 wavefront path tracer (Mpaths/s).

Workload (default ``volume``): the heterogeneous-volume scene -- a 512^3 FP32 fractal-noise
cloud (about 30% of voxels non-zero, max sigma_t 20 per unit, albedo 0.99, HG g = 0.8),
lit by a directional sun (irradiance 5) and a constant sky (0.3), 1280x720, 256 spp, up to
128 scattering events.  One step renders that whole image.  ``spheres`` and ``mesh`` run
the other two scenes (640x360x64 spp; 1920x1080x256 spp over ~1.3M triangles).

Arms:
* ours (default): ``value`` is device time (CUDA events on the library's stream) with the
  scene resident in HBM; ``e2e`` is wall time through the public C ABI with host buffers:
  each step uploads the scene from pinned host memory (pg_upload_scene), renders and reads
  the film back (mean, variance, count) into pinned host memory.
* ``--impl reference``: pine's own CPU integrator (the reference compiled from its sources
  into oracle/_ref) on the same scene file.  Scenes with the constant sky render with
  oracle/_ref/pine_ref_const, pine plus a `Constant{ color }` environment light
  (oracle/constant_env.py), since pine's own environment set cannot express it; all host
  threads, one bounded sample of the image per step.  This arm loads no part of this
  repository's renderer (the scene inputs come from the separate pine-scenegen tool).

Multi-GPU (``torchrun --nproc-per-node N bench.py --gpus N``): independent replicas, each
rank renders the full workload with its own seed (weak scaling); times are the max over
ranks.
"""

from __future__ import annotations

import argparse
import csv
import io
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "pine_ref")
REF_BIN_CONST = os.path.join(ROOT, "oracle", "_ref", "pine_ref_const")
TRAFFIC_FILE = os.path.join(ROOT, "profiles", "volume_traffic.json")
FALLBACK_HBM_GBS = 6650.0

WORKLOADS = {
    "volume": dict(kind="volume", width=1280, height=720, spp=256, max_depth=128, n=512),
    "spheres": dict(kind="spheres", width=640, height=360, spp=64, max_depth=8),
    "mesh": dict(kind="mesh", width=1920, height=1080, spp=256, max_depth=16, subdiv=8),
}
# ncu cases (--profile-case): each workload's scene and film at a few samples per pixel, so
# that the first wavefront launches are full queues of the default 2^23 path slots, as in
# the benchmark (the 512^3 grid and the 1.31M-triangle mesh are larger than L2 either way;
# a few GB on the device).
PROFILE_CASES = {
    "volume": dict(WORKLOADS["volume"], spp=16),
    "spheres": dict(WORKLOADS["spheres"], spp=32),
    "mesh": dict(WORKLOADS["mesh"], spp=4),
}


def parse_args():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="volume")
    ap.add_argument("--math", choices=["pine", "fast"], default="fast")
    ap.add_argument("--cache", default=os.environ.get("PINE_B200_SCENES",
                                                      os.path.join(tempfile.gettempdir(),
                                                                   "pine_b200_scenes")))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--sampler", choices=["Uniform", "Halton"], default="Uniform",
                    help="the scene file's sampler (both arms render the same file)")
    ap.add_argument("--filter", choices=["Box", "Triangle", "Gaussian", "Mitchell",
                                         "LanczosSinc"], default="Box",
                    help="the scene file's film filter (radius 0.5)")
    ap.add_argument("--bvh", choices=["host", "gpu", "gpu_sah"], default="gpu_sah",
                    help="BVH builder for the scene upload")
    ap.add_argument("--majorant-brick", type=int, choices=[8, 16, 32, 64], default=None,
                    help="majorant brick edge in voxels (default: the library's tuning)")
    ap.add_argument("--queue-capacity", type=int, default=None,
                    help="path slots of the wavefront (default: the library's tuning)")
    ap.add_argument("--sort-queue", type=int, choices=[0, 1, 2], default=None,
                    help="order the active list by medium cell before tracking (default: "
                         "the library's tuning)")
    ap.add_argument("--profile-case", action="store_true",
                    help="render the small ncu case once and print its per-kernel counters")
    ap.add_argument("--guided", action="store_true",
                    help="with --profile-case: render it guided (one pass, then training)")
    ap.add_argument("--batch-eval", action="store_true",
                    help="the 64-request batch: aggregate Mpaths/s and per-request latency "
                         "p50/p99, graph-captured waves vs one request at a time")
    ap.add_argument("--batch-requests", type=int, default=64)
    ap.add_argument("--batch-seed", type=int, default=0)
    ap.add_argument("--guiding-eval", action="store_true",
                    help="time to RMSE <= --rmse-target against a plain reference, guided vs "
                         "plain, on --workload (one GPU; prints its own JSON line)")
    ap.add_argument("--rmse-target", type=float, default=1e-2)
    ap.add_argument("--ref-spp", type=int, default=65536)
    ap.add_argument("--guide-size", type=int, nargs=2, default=None, metavar=("W", "H"),
                    help="film size of the guiding evaluation (default: the workload's)")
    ap.add_argument("--guide-time-limit", type=float, default=90.0,
                    help="seconds of render time per method before extrapolating")
    ap.add_argument("--guide-depth", type=int, default=0,
                    help="--guiding-eval: guide vertices below this bounce depth (0: the library's default)")
    ap.add_argument("--guide-budget", type=int, default=0,
                    help="--guiding-eval: Adam steps per network (0: the library's default)")
    return ap.parse_args()


# ---------------------------------------------------------------- scenes
SCENE_OPTS = {"sampler": "Uniform", "filter": "Box"}


def scene_path(cfg, cache, env, spp=None, size=None):
    from pine_b200 import scenegen
    os.makedirs(cache, exist_ok=True)
    w, h = size or (cfg["width"], cfg["height"])
    spp = cfg["spp"] if spp is None else spp
    kind = cfg["kind"]
    # By default every workload uses the Uniform sampler (the library's independent stream,
    # no Halton draws) and a box filter of radius 0.5; the reference arm renders the same
    # file.
    smp, flt = SCENE_OPTS["sampler"], SCENE_OPTS["filter"]
    name = f"{kind}_{env}_{w}x{h}_{spp}_{smp.lower()}_{flt.lower()}.txt"
    path = os.path.join(cache, name)
    if kind == "volume":
        scenegen.volume_scene(path, n=cfg["n"], width=w, height=h, spp=spp,
                              max_depth=cfg["max_depth"], env=env,
                              env_radiance=0.3 if env == "constant" else 1.0)
    elif kind == "spheres":
        scenegen.spheres_scene(path, width=w, height=h, spp=spp, max_depth=cfg["max_depth"],
                               env=env, env_radiance=0.2 if env == "constant" else 0.5,
                               sampler=smp)
    else:
        scenegen.mesh_scene(path, subdiv=cfg["subdiv"], width=w, height=h, spp=spp,
                            max_depth=cfg["max_depth"], env="none", sampler=smp)
    if flt != "Box":
        with open(path) as f:
            text = f.read()
        assert "filter: Box{" in text
        with open(path, "w") as f:
            f.write(text.replace("filter: Box{", "filter: " + flt + "{"))
    return path


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples every 200 ms while the timed region runs."""

    FIELDS = ["index", "clocks.sm", "clocks.max.sm", "power.draw", "clocks_event_reasons.active",
              "clocks_event_reasons.hw_slowdown", "clocks_event_reasons.hw_thermal_slowdown",
              "clocks_event_reasons.sw_thermal_slowdown", "clocks_event_reasons.sw_power_cap"]

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.out = None

    def start(self):
        try:
            self.out = tempfile.TemporaryFile(mode="w+")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + ",".join(self.FIELDS),
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.out, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.out.seek(0)
        rows = [r for r in csv.reader(io.StringIO(self.out.read())) if len(r) == len(self.FIELDS)]
        sm, smax, reasons, power = [], [], set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                smax.append(float(r[2]))
                power.append(float(r[3]))
            except ValueError:
                continue
            for name, v in zip(names, r[5:]):
                if v.strip().lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "power_w_max": max(power) if power else None,
                "samples": len(sm), "reasons": sorted(reasons)}


# ---------------------------------------------------------------- roofline
def hbm_peak():
    try:
        with open(PEAKS_FILE) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


# Algorithmic bytes (a fixed model):
# * a traced ray (k_trace, and shadow rays through a BVH): B_ray = 32 B ray read + 16 B hit
#   write + 80 B per level of the 8-wide BVH (one compressed node, ceil(log8 N) levels for
#   N primitives) + one leaf primitive (48 B triangle, 16 B sphere);
# * a path iteration of k_shade: 128 B of path state (64 B read, 64 B written);
# * a shadow ray of k_shadow without a BVH (volume-only scenes): 64 B (48 B ray read, 16 B
#   radiance update);
# * a ray walked by k_track (delta tracking of an extension ray): 32 B ray read + 16 B result
#   written; by k_transmit (ratio tracking of a shadow ray): 48 B ray read + 16 B
#   contribution read and written;
# * per volume tracking step 32 B (the 8 voxels of a trilinear lookup), 4 B per majorant
#   brick entered;
# * a camera path started by k_regen: 80 B of new path state.
STATE_BYTES = {"shade": 128, "shadow": 64, "regen": 80, "track": 48, "transmit": 80}


def ray_bytes(prims, triangles):
    """B_ray for a scene of `prims` BVH primitives (0: no BVH)."""
    if prims <= 0:
        return 0
    levels = max(1, math.ceil(math.log(prims, 8) - 1e-12))
    return 32 + 16 + 80 * levels + (48 if triangles else 16)


def algorithmic_bytes(name, k, b_ray):
    if name == "trace":
        per_item = b_ray
    elif name == "shadow" and b_ray:
        per_item = b_ray
    else:
        per_item = STATE_BYTES[name]
    return per_item * k["items"] + 32 * k["volume_steps"] + 4 * k["bricks"]


def read_traffic():
    """DRAM bytes per algorithmic byte of each kernel, measured by ncu on the small case and
    committed beside its summary (profiles/volume_traffic.json)."""
    try:
        with open(TRAFFIC_FILE) as f:
            return {k: float(v) for k, v in json.load(f)["dram_bytes_per_algorithmic_byte"].items()}
    except (OSError, KeyError, ValueError):
        return {}


def roofline(kernels, peak, peak_kind, b_ray, workload):
    timed = {n: k for n, k in kernels.items() if k["seconds"] > 0 and k["launches"] > 0}
    if not timed:
        return None
    name = max(timed, key=lambda n: timed[n]["seconds"])
    k = timed[name]
    per_launch_bytes = algorithmic_bytes(name, k, b_ray) / k["launches"]
    launch_s = k["seconds"] / k["launches"]
    achieved = per_launch_bytes / launch_s / 1e9
    traffic, traffic_note = None, None
    tr = read_traffic() if workload == "volume" else {}
    if name in tr:
        traffic = tr[name] * per_launch_bytes
        traffic_note = ("scaled from the 16-spp ncu case: DRAM bytes per algorithmic byte of the "
                        "kernel (profiles/volume_traffic.json) x this run's algorithmic bytes "
                        "per launch")
    out = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
           "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
           "kernel": "k_" + name, "algorithmic_bytes_per_launch": per_launch_bytes,
           "avg_launch_ms": launch_s * 1e3, "launches": k["launches"],
           "share_of_device_time": k["seconds"] / sum(v["seconds"] for v in timed.values())}
    if b_ray:
        out["bytes_per_traced_ray"] = b_ray
    if traffic_note:
        out["traffic_note"] = traffic_note
    return out


def add_kernels(acc, k):
    for name, v in k.items():
        a = acc.setdefault(name, {key: 0 for key in v})
        for key, val in v.items():
            a[key] += val


# ---------------------------------------------------------------- CPU baseline (pine)
def scene_env(cfg):
    """The environment of a workload's scene: the constant sky, or none for the mesh."""
    return "none" if cfg["kind"] == "mesh" else "constant"


def ref_binary(env):
    """pine built from its sources; scenes with the constant sky need the build that adds
    pine's missing `Constant` environment (oracle/constant_env.py)."""
    return REF_BIN_CONST if env == "constant" else REF_BIN


def run_pine(binary, scene, repeats, spp):
    p = subprocess.run([binary, "time", scene, str(repeats), str(spp)], capture_output=True,
                       text=True, cwd=os.path.dirname(scene))
    lines = [json.loads(l) for l in p.stdout.splitlines() if l.startswith("{")]
    if p.returncode != 0 or not lines:
        raise RuntimeError(f"{os.path.basename(binary)} failed ({p.returncode}): "
                           f"{p.stderr[-500:]}")
    return lines


def cpu_baseline(cfg, cache):
    """pine's Path integrator on the host cores, on the scene file our arm renders: a 1-spp
    calibration run sizes a sample of about 10 s, which is then timed (scene loading and
    BVH build excluded)."""
    env = scene_env(cfg)
    binary = ref_binary(env)
    if not os.path.exists(binary):
        return None
    scene = scene_path(cfg, cache, env)
    runs = run_pine(binary, scene, 2, 1)
    cal = runs[-1]
    spp = int(max(1, min(cfg["spp"], 10.0 / max(cal["seconds"], 1e-3))))
    run = run_pine(binary, scene, 1, spp)[0]
    return {"value": run["mpaths_per_s"], "unit": "Mpaths/s", "cores": run["threads"],
            "kind": "reference",
            "sample": f"{cfg['width']}x{cfg['height']} at {spp} of the file's {cfg['spp']} spp "
                      f"({run['paths']:.0f} paths, {run['seconds']:.2f} s), the same scene file "
                      f"({os.path.basename(binary)})"}


def reference_arm(args, cfg, rank):
    if rank != 0:
        return 0
    env = scene_env(cfg)
    binary = ref_binary(env)
    line = {"metric": "Mpaths/s", "unit": "Mpaths/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"{args.workload}: " + describe(cfg) + "; pine's Path "
                                   "integrator on the host cores, the same scene file",
                       "binary": os.path.relpath(binary, ROOT)}}
    if not os.path.exists(binary):
        line["unavailable"] = (f"{os.path.relpath(binary, ROOT)} is not built (it needs the "
                               "pine sources at build time)")
        print(json.dumps(line))
        return 0
    scene = scene_path(cfg, args.cache, env)
    cal = run_pine(binary, scene, 2, 1)[-1]
    # Steps sized so that warmup + steps finish in about two minutes.
    per_step = 120.0 / max(1, args.steps + args.warmup)
    spp = int(max(1, min(cfg["spp"], per_step / max(cal["seconds"], 1e-3))))
    runs = run_pine(binary, scene, args.warmup + args.steps, spp)[args.warmup:]
    secs = sum(r["seconds"] for r in runs)
    paths = sum(r["paths"] for r in runs)
    value = paths / secs / 1e6
    line.update({"value": value, "ms_per_step": secs / len(runs) * 1e3,
                 "cpu_baseline": {"value": value, "unit": "Mpaths/s", "cores": runs[0]["threads"],
                                  "kind": "reference",
                                  "sample": f"{cfg['width']}x{cfg['height']} at {spp} of the "
                                            f"file's {cfg['spp']} spp per step"},
                 "e2e": {"value": value, "unit": "Mpaths/s", "h2d_bytes_per_step": 0,
                         "d2h_bytes_per_step": 0}})
    line["config"].update({"width": cfg["width"], "height": cfg["height"], "spp": cfg["spp"],
                           "spp_per_step": spp, "max_depth": cfg["max_depth"],
                           "scene_file": os.path.basename(scene)})
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------- our arm
def apply_tuning(ctx, args):
    """The library's tuning with the command line's overrides."""
    tune = ctx.tuning()
    if args.majorant_brick:
        tune["majorant_brick"] = args.majorant_brick
    if args.queue_capacity:
        tune["queue_capacity"] = args.queue_capacity
    if args.sort_queue is not None:
        tune["sort_queue"] = args.sort_queue
    ctx.set_tuning(**tune)
    return tune


def main():
    args = parse_args()
    SCENE_OPTS["sampler"], SCENE_OPTS["filter"] = args.sampler, args.filter
    cfg = WORKLOADS[args.workload]
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return reference_arm(args, cfg, rank)

    import pine_b200 as pb

    dist = None
    if world > 1:
        import torch
        import torch.distributed as tdist
        from datetime import timedelta
        torch.cuda.set_device(local)
        tdist.init_process_group("nccl", timeout=timedelta(seconds=600))
        dist = tdist

    def barrier():
        if dist:
            dist.barrier()

    def max_over_ranks(x):
        return reduce_max(x, dist, f"cuda:{local}")

    env = scene_env(cfg)
    if args.guiding_eval:
        if rank == 0:
            print(json.dumps(guiding_eval(args, cfg, env)))
        return 0
    if args.batch_eval:
        if rank == 0:
            print(json.dumps(batch_eval(args)))
        return 0
    if args.profile_case:
        case = PROFILE_CASES[args.workload]
        path = scene_path(case, args.cache, env)
        ctx = pb.Context(local)
        apply_tuning(ctx, args)
        sid = ctx.load_scene(path)
        if args.guided:
            ctx.guide_reset(seed=0)
        r = ctx.render(sid, seed=1, math_mode=args.math, outputs=False, guiding=args.guided,
                       profile=args.guided)
        print(json.dumps({"profile_case": case, "guided": args.guided,
                          "stats": r["stats"]}))
        ctx.close()
        return 0

    # Scene files are generated once per cache directory (rank 0 first).
    if rank == 0:
        path = scene_path(cfg, args.cache, env)
    barrier()
    if rank != 0:
        path = scene_path(cfg, args.cache, env)

    ctx = pb.Context(local)
    ctx.set_bvh_builder(args.bvh)
    tune = apply_tuning(ctx, args)
    sid = ctx.load_scene(path)
    info = ctx.scene_info(sid)
    bvh = ctx.bvh_info(sid)
    paths_per_step = info["width"] * info["height"] * cfg["spp"]
    seed0 = 1000 * rank

    for w in range(args.warmup):
        ctx.render(sid, seed=seed0 + w, math_mode=args.math, outputs=False)

    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    device_s = 0.0
    launches = 0
    kernels = {}
    stats_acc = {"rays": 0, "volume_steps": 0, "paths": 0, "dropped": 0}
    for s in range(args.steps):
        r = ctx.render(sid, seed=seed0 + 100 + s, math_mode=args.math, outputs=False,
                       profile=True)
        st = r["stats"]
        device_s += st["seconds"]
        launches += st["launches"]
        add_kernels(kernels, st["kernels"])
        for k in stats_acc:
            stats_acc[k] += st[k]
    barrier()
    clk = clocks.stop()
    device_s_max = max_over_ranks(device_s)

    # End-to-end through the public API: upload from pinned host memory, render, read the
    # film back into pinned host memory, release; wall clock, max over ranks.
    import torch
    parsed = pb.ParsedScene(path)
    desc = parsed.desc
    pinned = []
    h2d = 0
    for m in range(desc.num_media):
        med = desc.media[m]
        if med.density:
            n = med.size[0] * med.size[1] * med.size[2]
            src = np.ctypeslib.as_array(med.density, shape=(n,))
            buf = torch.empty(n, dtype=torch.float32, pin_memory=True)
            buf.numpy()[:] = src
            pinned.append(buf)
            med.density = ctypes_float_ptr(buf.data_ptr())
            h2d += n * 4
    h2d += desc.num_vertices * 12 + desc.num_triangles * 12
    w, h = info["width"], info["height"]
    out_mean = torch.empty((h, w, 3), dtype=torch.float32, pin_memory=True).numpy()
    out_var = torch.empty((h, w, 3), dtype=torch.float32, pin_memory=True).numpy()
    out_cnt = torch.empty((h, w), dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
    d2h = out_mean.nbytes + out_var.nbytes + out_cnt.nbytes
    e2e_steps = max(1, min(args.steps, 4))
    sid2 = ctx.upload_scene(desc)
    ctx.render(sid2, spp=1, seed=7, math_mode=args.math, into=(out_mean, out_var, out_cnt))
    ctx.release_scene(sid2)
    barrier()
    phases = {"upload": 0.0, "render_and_readback": 0.0, "release": 0.0}
    t0 = time.perf_counter()
    for s in range(e2e_steps):
        ta = time.perf_counter()
        sid2 = ctx.upload_scene(desc)
        tb = time.perf_counter()
        ctx.render(sid2, seed=seed0 + 500 + s, math_mode=args.math,
                   into=(out_mean, out_var, out_cnt))
        tc = time.perf_counter()
        ctx.release_scene(sid2)
        td = time.perf_counter()
        phases["upload"] += tb - ta
        phases["render_and_readback"] += tc - tb
        phases["release"] += td - tc
    barrier()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    # BVH primitives for the traced-ray bytes: triangles plus the analytic shapes (planes are
    # tested outside the BVH).
    shapes = [desc.shapes[i].type for i in range(desc.num_shapes)]
    prims = int(desc.num_triangles) + sum(t in (pb.SHAPE_SPHERE, pb.SHAPE_RECT,
                                                pb.SHAPE_TRIANGLE) for t in shapes)
    b_ray = ray_bytes(prims, desc.num_triangles > 0) if bvh["nodes"] > 0 else 0
    parsed.close()

    value = aggregate(paths_per_step, args.steps, world, device_s_max)
    e2e = aggregate(paths_per_step, e2e_steps, world, e2e_s)
    peak, peak_kind = hbm_peak()
    line = {
        "metric": "Mpaths/s", "value": value, "unit": "Mpaths/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": device_s_max / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded generators; no dataset)",
        "config": {"workload": f"{args.workload}: " + describe(cfg), "width": info["width"],
                   "height": info["height"], "spp": cfg["spp"], "max_depth": cfg["max_depth"],
                   "math_mode": args.math, "parallelism": f"replicas x{world}",
                   "sampler": args.sampler, "filter": args.filter, "tuning": tune,
                   "bvh": dict(builder=args.bvh, **bvh),
                   "l2": "inputs larger than L2 (512 MiB density grid vs 126 MB L2)"
                         if cfg["kind"] == "volume" else "scene resident; no flush"},
        "e2e": {"value": e2e, "unit": "Mpaths/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "steps": e2e_steps,
                "timing": "wall clock: pg_upload_scene + pg_render + film readback + release",
                "phase_ms_per_step": {k: round(v / e2e_steps * 1e3, 2) for k, v in phases.items()}},
        "gpu_launches": launches,
        "mrays_per_s": stats_acc["rays"] * world / device_s_max / 1e6,
        "gsteps_per_s": stats_acc["volume_steps"] * world / device_s_max / 1e9,
        "dropped_samples": stats_acc["dropped"],
        "roofline": roofline(kernels, peak, peak_kind, b_ray, args.workload),
        "kernels": {n: {"launches": k["launches"], "seconds": k["seconds"],
                        "items": k["items"], "volume_steps": k["volume_steps"]}
                    for n, k in kernels.items()},
        "clocks": clk,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            line["cpu_baseline"] = cpu_baseline(cfg, args.cache)
        except Exception as e:  # the baseline is reported, never required
            line["cpu_baseline"] = {"value": None, "error": str(e)[:200]}
    if rank == 0:
        print(json.dumps(line))
    ctx.close()
    if dist:
        dist.destroy_process_group()
    return 0


def batch_eval(args):
    """The batched-requests workload: requests drawn by seed from the spheres, mesh and
    volume generators, resolution side uniform in 128..1024 with aspect uniform in
    1..16/9, spp log-uniform in 16..256.  The autotuner picks the tuning; then the whole
    set renders as one batch of graph-captured waves (latency = completion time of each
    request from the batch start, device clock) and, for comparison, one request at a time
    (latency = the running sum of the single-request device times), both in the caller's
    order and shortest job first, the order a wave serves its requests in.  The batch is
    timed all three ways the tuning allows: one wave per scene, one per scene kind and one
    for the whole batch.
    `wall_*` adds the host's share (graph capture, launches, synchronisation): the
    render_batch call's wall time, and the sum of the single calls' wall times."""
    import pine_b200 as pb
    ctx = pb.Context(0)
    kinds = ["spheres", "mesh", "volume"]
    sids = {}
    for k in kinds:
        sids[k] = ctx.load_scene(scene_path(WORKLOADS[k], args.cache,
                                            "none" if k == "mesh" else "constant"))
    rng = np.random.default_rng(args.batch_seed)
    reqs, mix = [], {k: 0 for k in kinds}
    for i in range(args.batch_requests):
        k = kinds[int(rng.integers(3))]
        side = int(rng.uniform(128, 1024))
        aspect = float(rng.uniform(1.0, 16.0 / 9.0))
        w, h = side, max(1, int(round(side / aspect)))
        spp = int(round(np.exp(rng.uniform(np.log(16), np.log(256)))))
        reqs.append(dict(scene=sids[k], width=w, height=h, spp=spp,
                         max_depth=WORKLOADS[k]["max_depth"], seed=1000 + i))
        mix[k] += 1
    paths = sum(r["width"] * r["height"] * r["spp"] for r in reqs)
    tuning = ctx.autotune(reqs)
    pct = lambda a, q: float(np.percentile(a, q))
    batches = {}
    for g in (2, 1, 0):  # one wave per scene, per scene kind, one for the whole batch
        ctx.set_tuning(**dict(tuning, group_kinds=g))
        ctx.render_batch(reqs, outputs=False)  # warm-up
        t0 = time.perf_counter()
        b = ctx.render_batch(reqs, outputs=False)
        wall = time.perf_counter() - t0
        lat = np.array(b["request_seconds"])
        batches[g] = {"seconds": b["seconds"], "value": paths / b["seconds"] / 1e6,
                      "latency_p50_s": pct(lat, 50), "latency_p99_s": pct(lat, 99),
                      "wall_seconds": wall, "wall_value": paths / wall / 1e6}
    # The batch at every queue capacity the autotuner chooses from.
    sweep = {}
    for cap in (1 << 20, 1 << 21, 1 << 22, 1 << 23):
        ctx.set_tuning(**dict(tuning, queue_capacity=cap))
        ctx.render_batch(reqs, outputs=False)
        sweep[cap] = paths / ctx.render_batch(reqs, outputs=False)["seconds"] / 1e6
    ctx.set_tuning(**tuning)
    single, single_wall = [], []
    for r in reqs:
        t0 = time.perf_counter()
        single.append(ctx.render_batch([r], outputs=False)["seconds"])
        single_wall.append(time.perf_counter() - t0)

    def sequential(order):
        done = np.cumsum(np.asarray(single)[order])
        t = float(done[-1])
        wall = float(np.sum(single_wall))
        return {"seconds": t, "value": paths / t / 1e6, "latency_p50_s": pct(done, 50),
                "latency_p99_s": pct(done, 99), "wall_seconds": wall, "wall_value": paths / wall / 1e6}

    # Each kind batched alone, against the same requests one at a time (device seconds).
    per_kind = {}
    for k in kinds:
        idx = [i for i, r in enumerate(reqs) if r["scene"] == sids[k]]
        sub = [reqs[i] for i in idx]
        ctx.render_batch(sub, outputs=False)
        per_kind[k] = {"requests": len(sub),
                       "batch_seconds": ctx.render_batch(sub, outputs=False)["seconds"],
                       "one_at_a_time_seconds": float(np.sum(np.asarray(single)[idx]))}
    sjf = sorted(range(len(reqs)), key=lambda i: reqs[i]["width"] * reqs[i]["height"] * reqs[i]["spp"])
    ctx.close()
    return {"metric": "Mpaths/s", "workload": f"{len(reqs)} requests (seed {args.batch_seed}): {mix}",
            "paths": int(paths), "tuning": tuning,
            "batch": batches[tuning["group_kinds"]],
            "batch_wave_per_scene": batches[2],
            "batch_wave_per_kind": batches[1],
            "batch_one_wave": batches[0],
            "batch_mpaths_per_s_by_queue_capacity": sweep,
            "per_kind": per_kind,
            "one_at_a_time": sequential(list(range(len(reqs)))),
            "one_at_a_time_shortest_first": sequential(sjf)}


def guiding_eval(args, cfg, env):
    """Time for the plain and the guided estimator to reach an RMSE target against a
    high-spp plain reference (the reference is rendered once per cache directory).

    Each method renders a progressive sequence (16 spp, then doubling the total) into an
    accumulating film, and its RMSE against the reference is measured after every call.
    Time is the render calls' device time, training included for the guided method.  The
    reference's own noise (mean per-pixel sample variance / its spp) is a floor under the
    measured MSE.  The time at which a method crosses the target is interpolated (or, past
    the time limit, extrapolated) from its last two points with MSE - floor falling as
    1 / time, so that the doubling steps do not quantise it."""
    import pine_b200 as pb
    size = tuple(args.guide_size) if args.guide_size else (cfg["width"], cfg["height"])
    path = scene_path(cfg, args.cache, env, size=size)
    ctx = pb.Context(0)
    sid = ctx.load_scene(path)
    info = ctx.scene_info(sid)
    # Sample ids of one call stay below 2^32 (pg_render); longer renders accumulate calls
    # with independent seeds.
    npix = info["width"] * info["height"]
    max_call = 1 << int(np.log2(max(1, ((1 << 32) - 1) // npix)))
    ref_file = os.path.join(args.cache, f"ref_{os.path.basename(path)}_{args.ref_spp}_{args.math}.npz")
    if os.path.exists(ref_file):
        z = np.load(ref_file)
        ref, ref_var = z["mean"], z["var"]
    else:
        done, k = 0, 0
        while done < args.ref_spp:
            sp = min(max_call, args.ref_spp - done)
            r = ctx.render(sid, spp=sp, seed=7770 + k, accumulate=done > 0, math_mode=args.math)
            done += sp
            k += 1
        ref, ref_var = r["mean"], r["var"]
        np.savez(ref_file, mean=ref, var=ref_var)
    floor = float(ref_var.mean()) / args.ref_spp
    target2 = args.rmse_target ** 2
    out = {"metric": f"time to RMSE <= {args.rmse_target:g} against a {args.ref_spp}-spp plain "
                     "reference (s)",
           "workload": f"{args.workload}: " + describe(cfg) + f" at {size[0]}x{size[1]}",
           "math_mode": args.math,
           "reference": {"spp": args.ref_spp, "rmse_floor": floor ** 0.5},
           "guide_depth": args.guide_depth or "all", "guide_budget": args.guide_budget or 1024}
    ctx.guide_config(args.guide_depth, args.guide_budget)
    for method in ("plain", "guided"):
        guided = method == "guided"
        if guided:
            ctx.guide_reset(seed=0)
        t, done, chunk, curve, k = 0.0, 0, 16, [], 0
        reached = False
        while True:
            left = chunk
            while left > 0:
                sp = min(left, max_call)
                r = ctx.render(sid, spp=sp, seed=(1100 if guided else 1200) + k,
                               accumulate=done > 0, math_mode=args.math, guiding=guided)
                t += r["stats"]["seconds"]
                done += sp
                left -= sp
                k += 1
            mse = float(np.mean((r["mean"] - ref) ** 2))
            curve.append({"spp": done, "seconds": round(t, 4), "rmse": mse ** 0.5,
                          "sample_variance": float(r["var"].mean())})
            if mse <= target2:
                reached = True
                break
            if t >= args.guide_time_limit or done >= args.ref_spp:
                break
            chunk = done
        # MSE - floor falls as 1 / time: the crossing of the target is interpolated from the
        # last two measured points (one point when the first call already reached it).
        tail = [c for c in curve[-2:] if c["rmse"] ** 2 > floor]
        if target2 > floor and tail:
            cst = sum((c["rmse"] ** 2 - floor) * c["seconds"] for c in tail) / len(tail)
            t_target = cst / (target2 - floor)
        else:
            t_target = t if reached else None
        out[method] = {"seconds": t_target, "reached": reached, "curve": curve}
    tp, tg = out["plain"]["seconds"], out["guided"]["seconds"]
    out["guided_over_plain"] = tg / tp if tp and tg else None
    ctx.close()
    return out


def reduce_max(x, dist, device):
    """Max of x over the ranks of the process group (x itself without one)."""
    if not dist:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate(paths_per_step, steps, world, device_seconds_max):
    """Whole-job throughput in Mpaths/s: every rank renders paths_per_step per step."""
    return paths_per_step * steps * world / device_seconds_max / 1e6


def ctypes_float_ptr(addr):
    import ctypes
    return ctypes.cast(ctypes.c_void_p(addr), ctypes.POINTER(ctypes.c_float))


def describe(cfg):
    if cfg["kind"] == "volume":
        return (f"{cfg['n']}^3 FP32 cloud grid, sigma_t 20, albedo 0.99, HG g 0.8, sun 5 + "
                f"constant sky 0.3, {cfg['width']}x{cfg['height']}, {cfg['spp']} spp, "
                f"max {cfg['max_depth']} events")
    if cfg["kind"] == "spheres":
        return (f"64 spheres + plane + rect light + constant env 0.2, {cfg['width']}x"
                f"{cfg['height']}, {cfg['spp']} spp, depth {cfg['max_depth']}")
    return (f"icosphere 20*4^{cfg['subdiv']} triangles in a Cornell box, {cfg['width']}x"
            f"{cfg['height']}, {cfg['spp']} spp, depth {cfg['max_depth']}")


if __name__ == "__main__":
    sys.exit(main())
