"""Benchmark: path-traced frames of the 1M-triangle torus field on B200.

Workload (one "step"): one progressive frame of the 1920x1080 torus-field
scene (4096 instances of a 256-triangle torus = 1,048,576 triangles, 8
emissive sphere lights, ground plane, sun and sky; seed 2) at 64 samples per
pixel and depth 8 -- 132,710,400 path samples. Step k renders the sample
window [64k, 64k+64), so successive steps refine the same image.

value     : whole-job Msamples/s (device time, CUDA events on the launching
            stream, max over ranks), inputs resident in HBM.
e2e       : the same metric through the drop-in entry point
            mt_pathtrace_render (camera from host memory, RGB8 image read back
            to host memory every step).
roofline  : dominant kernel against the measured HBM copy bandwidth, with the
            canonical BVH2 byte accounting per ray (64 B per node pair, 48 B
            per triangle, 16 B per sphere, 48 B of ray + hit record).
time_to_rmse : linear-RGB RMSE 1e-3 reached at N* = mean(sigma^2) / 1e-6
            samples per pixel for this unbiased estimator; sigma^2 is measured
            from the timed frames themselves (variance of the per-frame means).

--impl reference times the reference's own multithreaded CPU path tracer
(oracle/_ref, compiled from the reference sources) on the same scene.
Multi-GPU (torchrun): every rank renders its own replica of the frame (weak
scaling, no data-path collective).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
os.environ.setdefault("RAYTRACER_NO_PROGRESS", "1")

import numpy as np  # noqa: E402

W, H, SPP, DEPTH = 1920, 1080, 64, 8
WORKLOAD = "torus-field 1920x1080, 64 spp, depth 8, 1,048,576 triangles + 8 emissive spheres + plane (seed 2)"
METRIC = "Msamples/s (1080p 64-spp path tracing, 1M-triangle PBR scene; time-to-RMSE 1e-3 beside)"


def _dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = ROOT / "gpurun_out" / f"clocks_{os.getpid()}.csv"

    def __enter__(self):
        try:
            self.path.parent.mkdir(exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if self.proc is None or not self.path.exists():
            return None
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def build_scene():
    from marmel_trace_b200 import scenes

    return scenes.torus_field_scene()


def algorithmic_bytes(stats, samples_counted: int, samples_launch: int) -> float:
    """Canonical BVH2 accounting (64 B per node pair, 48 B per triangle,
    16 B per other primitive, 48 B ray + hit record per ray), scaled from the
    counted launch to one timed launch."""
    rays = stats.extension_rays + stats.shadow_rays
    other = stats.prim_tests - stats.tri_tests
    b = 64.0 * stats.node_visits + 48.0 * stats.tri_tests + 16.0 * other + 48.0 * rays
    return b * samples_launch / samples_counted


def run_ours(args):
    import torch

    rank, world, local = _dist_env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))

    import marmel_trace_b200 as mt
    from marmel_trace_b200 import _capi

    desc = build_scene()
    cam = desc.make_camera(W, H)
    g = mt.GpuScene(desc, precision="fp32", integrator=args.integrator, device=local)
    lib = g.lib
    stream = torch.cuda.current_stream()
    accum = torch.zeros((H, W, 3), dtype=torch.float32, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")  # > 126 MB L2

    def step(k: int, acc: int):
        rc = lib.mt_render_accumulate_device(g.h, cam.ref, W, H, k * SPP, (k + 1) * SPP, DEPTH, 0,
                                             accum.data_ptr(), acc, stream.cuda_stream)
        _capi.check(rc, "mt_render_accumulate_device")

    # counting pass (untimed): rays, node pairs, primitive tests per sample
    g.set_counting(True)
    cnt_spp = 4
    rc = lib.mt_render_accumulate_device(g.h, cam.ref, W, H, 10_000, 10_000 + cnt_spp, DEPTH, 0, accum.data_ptr(), 0,
                                         stream.cuda_stream)
    _capi.check(rc, "count pass")
    torch.cuda.synchronize()
    cnt = g.stats()
    g.set_counting(False)

    for k in range(args.warmup):
        step(1000 + k, 0)
    torch.cuda.synchronize()

    frame_means = []
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        t_wall = time.perf_counter()
        for k in range(args.steps):
            flush.zero_()
            ev[k][0].record(stream)
            step(k, 0)
            ev[k][1].record(stream)
            if k < 8:
                frame_means.append((accum / SPP).cpu())  # untimed readback between steps
        torch.cuda.synchronize()
        t_wall = time.perf_counter() - t_wall
    if dist:
        dist.barrier()
    ms = [a.elapsed_time(b) for a, b in ev]
    dev_s = sum(ms) / 1e3
    if dist:
        t = torch.tensor([dev_s], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dev_s = float(t.item())
    samples = W * H * SPP * args.steps * world
    value = samples / dev_s / 1e6
    st = g.stats()

    # e2e through the drop-in entry point (host camera in, host RGB8 out)
    rgb = np.zeros((H, W, 3), np.uint8)
    e2e_ms = []
    for k in range(0 if args.no_e2e else max(1, min(args.steps, 3))):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _capi.check(lib.mt_pathtrace_render(g.h, cam.ref, W, H, SPP, DEPTH, rgb.ctypes.data), "mt_pathtrace_render")
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
    e2e_val = (W * H * SPP) / (statistics.median(e2e_ms) / 1e3) / 1e6 * world if e2e_ms else None

    # time to RMSE 1e-3 from the measured per-pixel variance of 64-spp frames
    ttr = None
    if len(frame_means) >= 3:
        fm = torch.stack(frame_means).double()
        var64 = fm.var(dim=0, unbiased=True).mean().item()  # variance of a 64-spp mean, per channel
        sigma2 = var64 * SPP
        n_star = sigma2 / 1e-6
        ttr = {"rmse_target": 1e-3, "spp_needed": n_star, "seconds": n_star * W * H / (value * 1e6 / world),
               "sigma2_per_sample": sigma2, "rmse_at_64spp": var64 ** 0.5,
               "method": "N* = mean per-pixel sample variance / 1e-6 (unbiased estimator); variance measured "
                         "across the timed frames"}

    peak, peak_kind = peaks()
    kernel_s = (sum(ms) / 1e3) / args.steps  # this rank's average launch duration
    alg = algorithmic_bytes(cnt, W * H * cnt_spp, W * H * SPP)
    achieved = alg / kernel_s / 1e9
    rays_per_sample = (cnt.extension_rays + cnt.shadow_rays) / (W * H * cnt_spp)
    traffic = None
    tf = ROOT / "profiles" / "traffic_bytes_per_sample.json"
    if tf.exists():
        tv = json.loads(tf.read_text()).get(args.integrator)
        if tv:
            traffic = tv * W * H * SPP

    out = {
        "metric": METRIC,
        "value": round(value, 3),
        "unit": "Msamples/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(1e3 * dev_s / args.steps, 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded generator, no dataset)",
        "config": {"workload": WORKLOAD, "width": W, "height": H, "spp_per_step": SPP, "depth": DEPTH,
                   "integrator": args.integrator, "parallelism": f"replicas x{world}",
                   "l2": "flushed between timed steps (256 MB write); scene 90 MB < L2"},
        "mrays_per_s": round(value * rays_per_sample, 2),
        "rays_per_sample": round(rays_per_sample, 3),
        "time_to_rmse": ttr,
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": traffic,
                     "peak_source": f"{peak_kind} MEASURED_PEAKS.json hbm_gbs" if peak_kind == "measured" else "fallback",
                     "kernel": "k_render<float, PT> (megakernel)" if args.integrator == "megakernel" else "wavefront",
                     "algorithmic_bytes_per_launch": alg},
        "e2e": {"value": round(e2e_val, 3) if e2e_val else None, "unit": "Msamples/s", "h2d_bytes_per_step": 128,
                "d2h_bytes_per_step": W * H * 3, "entry_point": "mt_pathtrace_render"},
        "gpu_launches": int(st.launches) * args.steps,
        "wall_s_timed_loop": round(t_wall, 3),
    }
    if rank == 0:
        clocks = clk.summary()
        if clocks:
            out["clocks"] = clocks
        if not args.no_cpu_baseline:
            out["cpu_baseline"] = cpu_baseline(desc, cam, args.cpu_spp)
        print(json.dumps(out), flush=True)
    g.release()
    if dist:
        dist.destroy_process_group()


def cpu_baseline(desc, cam, spp: int):
    """The reference's own multithreaded path tracer (oracle/_ref) on the same
    scene: a bounded sample of the workload (full frame at `spp`)."""
    from oracle import ref

    cores = os.cpu_count() or 1
    os.environ["RAYTRACER_THREADS"] = str(cores)
    rs = ref.RefScene.from_desc(desc, cam)
    t0 = time.perf_counter()
    rs.pathtrace_render(W, H, spp, DEPTH)
    dt = time.perf_counter() - t0
    rs.free()
    return {"value": round(W * H * spp / dt / 1e6, 4), "unit": "Msamples/s", "cores": cores, "kind": "reference",
            "sample": f"pathtrace_render full frame {W}x{H} at {spp} spp, depth {DEPTH} "
                      f"({dt:.1f} s, RAYTRACER_THREADS={cores})"}


def run_reference(args):
    rank, world, local = _dist_env()
    if rank != 0:
        return
    from oracle import ref

    import marmel_trace_b200 as mt  # noqa: F401  (camera_create through the C ABI's host code)

    desc = build_scene()
    cam = desc.make_camera(W, H)
    cores = os.cpu_count() or 1
    os.environ["RAYTRACER_THREADS"] = str(cores)
    rs = ref.RefScene.from_desc(desc, cam)
    spp = args.cpu_spp
    for _ in range(args.warmup):
        rs.pathtrace_render(W, H, spp, DEPTH)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        rs.pathtrace_render(W, H, spp, DEPTH)
        times.append(time.perf_counter() - t0)
    value = W * H * spp * len(times) / sum(times) / 1e6
    out = {
        "impl": "reference",
        "metric": METRIC,
        "value": round(value, 4),
        "unit": "Msamples/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(1e3 * sum(times) / len(times), 1),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded generator, no dataset)",
        "config": {"workload": WORKLOAD, "width": W, "height": H, "spp_per_step": spp, "depth": DEPTH,
                   "parallelism": f"{cores} CPU threads"},
        "cpu_baseline": {"value": round(value, 4), "unit": "Msamples/s", "cores": cores, "kind": "reference",
                         "sample": f"each step: pathtrace_render full frame at {spp} spp (bounded sample of the "
                                   f"64-spp workload)"},
        "e2e": {"value": round(value, 4), "unit": "Msamples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--integrator", default="megakernel", choices=["megakernel", "wavefront"])
    ap.add_argument("--cpu-spp", type=int, default=1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--spp", type=int, default=SPP, help="samples per pixel per step (profiling cases)")
    ap.add_argument("--no-e2e", action="store_true", help="skip the e2e leg (profiling cases)")
    args = ap.parse_args()
    globals()["SPP"] = args.spp
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
