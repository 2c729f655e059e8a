"""Benchmark: path-traced frames of the 1M-triangle torus field on B200.

Workload (one "step"): one progressive frame of the 1920x1080 torus-field
scene (4096 instances of a 256-triangle torus = 1,048,576 triangles, 8
emissive sphere lights, ground plane, sun and sky; seed 2) at 64 samples per
pixel and depth 8 -- 132,710,400 path samples. Step k renders the sample
window [64k, 64k+64), so successive steps refine the same image.

value        : whole-job Msamples/s of the wavefront integrator (device time,
               CUDA events on the launching stream, max over ranks), inputs
               resident in HBM, L2 flushed between steps.
plain_gpu    : the same frames through the megakernel (one thread per pixel,
               the "plain GPU" form of the same estimator).
e2e          : the same metric through the drop-in entry point
               mt_pathtrace_render (camera from host memory, RGB8 image read
               back to host memory every step).
roofline     : dominant kernel (any-hit traversal: the wavefront's shadow
               stage; the extend stage beside it) against the measured HBM
               copy bandwidth, canonical accounting per ray: one node record
               per visit (64 B binary), 48 B per triangle, 16 B per other
               primitive, 48 B of ray + hit record.
autotune     : mt_autotune's choice for this scene and view (4-spp probe),
               used by the timed frames.
batch        : the batched uneven workload (64 scenes) in one graph launch.
time_to_rmse : both integrators evaluate the same unbiased estimator with the
               same random streams, so linear-RGB RMSE after N samples per
               pixel is sqrt(mean sigma^2 / N); N* = mean(sigma^2) / 1e-6 and
               the time to reach it follows from each integrator's
               throughput. sigma^2 is measured from the timed frames.

--impl reference times the reference's own multithreaded CPU path tracer
(oracle/_ref, compiled from the reference sources) on the same scene.
Multi-GPU (torchrun): every rank renders its own replica of the frame (weak
scaling, no data-path collective).
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
os.environ.setdefault("RAYTRACER_NO_PROGRESS", "1")

import numpy as np  # noqa: E402

W, H, DEPTH = 1920, 1080, 8
WORKLOAD = "torus-field 1920x1080, 64 spp per step, depth 8, 1,048,576 triangles + 8 emissive spheres + plane (seed 2)"
METRIC = "Msamples/s (1080p 64-spp path tracing, 1M-triangle PBR scene; wavefront vs plain GPU; time-to-RMSE 1e-3 beside)"


def _dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def max_over_ranks(x: float, dist=None, device="cpu") -> float:
    """The largest per-rank value over the process group (the slowest rank's
    time). Every rank must call it, in the same order; without a process group
    it returns `x`."""
    if dist is None:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: float, world: int, seconds: float) -> float:
    """Whole-job throughput in millions of units per second: every replica
    processes `units_per_rank`, and the job ends with the slowest rank."""
    return units_per_rank * world / seconds / 1e6


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int, tag: str = ""):
        self.device = device
        self.proc = None
        # the raw samples (MT_CLOCKS_DIR, else the system temp folder); the
        # JSON line carries their summary
        out = Path(os.environ.get("MT_CLOCKS_DIR") or tempfile.gettempdir())
        self.path = out / f"clocks_{os.getpid()}{tag}.csv"

    def __enter__(self):
        try:
            self.path.parent.mkdir(parents=True, exist_ok=True)
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
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def build_scene():
    from marmel_trace_b200 import scenes

    return scenes.torus_field_scene()


# DRAM bytes (read + write) per path sample of the stage kernels, from an ncu
# launch list of this workload (4-spp frames, 2M-slot queue; summarised under
# profiles/): the shadow stage (cache pass 29.44 + 4.20 GB, walk 18.29 + 3.39
# GB) and the extend kernel (5.73 + 0.43 GB) over 7 frames of 4 x 2,073,600
# samples.
TRAFFIC_BYTES_PER_SAMPLE = {"shadow": 55.32e9 / (7 * 4 * 2073600), "extend": 6.16e9 / (7 * 4 * 2073600)}


def traversal_bytes(st, kind: str, width: int = 2) -> float:
    """Canonical bytes of the counted launch (nearest-hit or any-hit): one
    node record per visit (64 B binary, 128 / 256 B for 4 / 8 children)."""
    if kind == "nearest":
        nodes, prims, tris, rays = st.node_visits, st.prim_tests, st.tri_tests, st.extension_rays
    else:
        nodes, prims, tris, rays = st.any_node_visits, st.any_prim_tests, st.any_tri_tests, st.shadow_rays
    node_bytes = {2: 64.0, 4: 128.0, 8: 256.0}[width]
    return node_bytes * nodes + 48.0 * tris + 16.0 * (prims - tris) + 48.0 * rays


class Frames:
    """Timed progressive frames through mt_render_accumulate_device."""

    def __init__(self, g, cam, spp, torch):
        self.g, self.cam, self.spp, self.torch = g, cam, spp, torch
        self.stream = torch.cuda.current_stream()
        self.accum = torch.zeros((H, W, 3), dtype=torch.float32, device="cuda")

    def render(self, k: int, spp: int | None = None, base: int = 0):
        from marmel_trace_b200 import _capi

        n = spp or self.spp
        s0 = base + k * n
        rc = self.g.lib.mt_render_accumulate_device(self.g.h, self.cam.ref, W, H, s0, s0 + n, DEPTH, 0,
                                                    self.accum.data_ptr(), 0, self.stream.cuda_stream)
        _capi.check(rc, "mt_render_accumulate_device")

    def timed(self, steps: int, warmup: int, flush, keep_means: bool = False, base: int = 0):
        torch = self.torch
        for k in range(warmup):
            self.render(k, base=10_000 + base)
        torch.cuda.synchronize()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        means = []
        for k in range(steps):
            flush.zero_()
            ev[k][0].record(self.stream)
            self.render(k, base=base)
            ev[k][1].record(self.stream)
            if keep_means:
                means.append((self.accum / self.spp).cpu())  # outside the events
        torch.cuda.synchronize()
        return [a.elapsed_time(b) for a, b in ev], means


def run_ours(args):
    import torch

    rank, world, local = _dist_env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    import marmel_trace_b200 as mt
    from marmel_trace_b200 import _capi

    SPP = args.spp
    desc = build_scene()
    cam = desc.make_camera(W, H)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")  # 256 MB > 126 MB L2
    qopt = {"queue_capacity": args.queue_capacity} if args.queue_capacity else {}
    g = mt.GpuScene(desc, precision="fp32", integrator=args.integrator, device=local, **qopt)
    fr = Frames(g, cam, SPP, torch)

    # autotuner (untimed): the wavefront configuration for this scene and view,
    # chosen on a 4-spp probe window and kept on the scene for the timed frames
    tune = None
    if args.integrator == "wavefront" and not args.no_autotune:
        tune = g.autotune(cam, W, H, 4, DEPTH)
        ch = tune["chosen"]
        qopt = {"queue_capacity": ch["queue_capacity"], "traversal": 2 if ch["traversal"] == "dynamic" else 1,
                "block_size": ch["block"], "bvh_width": ch["bvh_width"], "sort_threshold": ch["sort_threshold"]}

    # counting pass (untimed): rays, node pairs and primitive tests per sample
    g.set_counting(True)
    fr.render(0, spp=4, base=20_000)
    cnt = g.stats()
    g.set_counting(False)
    n_counted = W * H * 4

    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        t_wall = time.perf_counter()
        ms, means = fr.timed(args.steps, args.warmup, flush, keep_means=True)
        t_wall = time.perf_counter() - t_wall
    if dist:
        dist.barrier()
    dev_s = max_over_ranks(sum(ms) / 1e3, dist, "cuda")
    samples_per_rank = W * H * SPP * args.steps
    value = whole_job_rate(samples_per_rank, world, dev_s)
    launches = int(g.stats().launches)

    # e2e through the drop-in entry point (host camera in, host RGB8 out)
    rgb = np.zeros((H, W, 3), np.uint8)
    e2e_ms, e2e_dev_ms = [], []
    n_e2e = 0 if args.no_e2e else max(3, min(args.steps, 5))
    with ClockSampler(local, "_e2e") as clk_e2e:
        # call 0 is an untimed warm-up: the first call through this entry point
        # captures its CUDA graph (RGB8 output) and pins its staging buffers
        for i in range(n_e2e + 1 if n_e2e else 0):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            _capi.check(g.lib.mt_pathtrace_render(g.h, cam.ref, W, H, SPP, DEPTH, rgb.ctypes.data),
                        "mt_pathtrace_render")
            if i == 0:
                continue
            e2e_ms.append((time.perf_counter() - t0) * 1e3)
            e2e_dev_ms.append(g.stats().kernel_ms)  # the render's own CUDA events
    e2e_val = whole_job_rate(W * H * SPP, world, max_over_ranks(statistics.median(e2e_ms) / 1e3, dist, "cuda")) \
        if e2e_ms else None

    # dominant-kernel duration: one frame with every stage bracketed by events
    stage = None
    if args.integrator == "wavefront":
        gp = mt.GpuScene(desc, precision="fp32", integrator="wavefront", use_graph=-1, device=local, **qopt)
        fp = Frames(gp, cam, SPP, torch)
        fp.render(0, base=30_000)
        gp.set_counting(False)  # resets the stage timers
        flush.zero_()
        fp.render(0, base=40_000)
        torch.cuda.synchronize()
        st = gp.stats()
        stage = {"extend_ms": st.stage_ms[0], "shade_ms": st.stage_ms[1], "shadow_ms": st.stage_ms[2],
                 "other_ms": st.stage_ms[3], "extend_launches": int(st.stage_launches[0]),
                 "shadow_launches": int(st.stage_launches[2])}
        gp.release()
        del fp

    # plain-GPU comparison (megakernel) on the same kind of frames
    plain = None
    if args.integrator == "wavefront" and not args.no_plain:
        gm = mt.GpuScene(desc, precision="fp32", integrator="megakernel", device=local)
        fm = Frames(gm, cam, SPP, torch)
        pms, _ = fm.timed(args.plain_steps, 1, flush, base=50_000)
        plain = W * H * SPP * len(pms) / (sum(pms) / 1e3) / 1e6
        gm.release()
        del fm

    # adjoint (inverse-rendering configuration: 512x512, 32 spp, depth 6,
    # 128 spheres + plane sharing 32 PBR materials, 259 parameters)
    adjoint = None
    if not args.no_adjoint:
        adjoint = adjoint_bench(torch, local, flush)

    # batched uneven workload: 64 scenes in one graph launch
    batch = None
    if not args.no_batch:
        batch = batch_bench(torch, local)

    large = large_bench(torch, local) if args.large else None

    # time to RMSE 1e-3
    ttr = None
    if len(means) >= 3:
        fm_ = torch.stack(means).double()
        var_frame = fm_.var(dim=0, unbiased=True).mean().item()  # variance of a SPP-sample mean, per channel
        sigma2 = var_frame * SPP
        n_star = sigma2 / 1e-6
        ttr = {"rmse_target": 1e-3, "sigma2_per_sample": sigma2, "rmse_per_frame": var_frame ** 0.5,
               "spp_needed": n_star,
               "seconds_wavefront" if args.integrator == "wavefront" else "seconds": n_star * W * H / (value / world * 1e6)}
        if plain:
            ttr["seconds_plain_gpu"] = n_star * W * H / (plain * 1e6)
            ttr["speedup_vs_plain"] = (value / world) / plain

    peak, peak_kind = peaks()
    rays_per_sample = (cnt.extension_rays + cnt.shadow_rays) / n_counted
    secondary = None
    traffic = None
    bw = qopt.get("bvh_width", 2) or 2
    if stage:
        # dominant stage kernel: the shadow (any-hit) stage on this workload
        dom = "shadow" if stage["shadow_ms"] >= stage["extend_ms"] else "extend"
        other = "extend" if dom == "shadow" else "shadow"
        kinds = {"shadow": ("any", "shadow stage: k_wf_shadow_cache<float> (cached occluders) + k_wf_shadow<float> "
                                   "(any-hit walk of the rest), per NEE connection"),
                 "extend": ("nearest", "k_wf_extend<float> (nearest-hit traversal)")}
        alg = traversal_bytes(cnt, kinds[dom][0], bw) * (W * H * SPP) / n_counted
        achieved = alg / (stage[f"{dom}_ms"] / 1e3) / 1e9
        kernel = kinds[dom][1] + "; per-stage CUDA events over one frame"
        per_launch = alg / stage[f"{dom}_launches"]
        traffic = TRAFFIC_BYTES_PER_SAMPLE[dom] * W * H * SPP / stage[f"{dom}_launches"]
        alg2 = traversal_bytes(cnt, kinds[other][0], bw) * (W * H * SPP) / n_counted
        secondary = {"kernel": kinds[other][1], "achieved": round(alg2 / (stage[f"{other}_ms"] / 1e3) / 1e9, 1),
                     "frac": round(alg2 / (stage[f"{other}_ms"] / 1e3) / 1e9 / peak, 4),
                     "traffic": round(TRAFFIC_BYTES_PER_SAMPLE[other] * W * H * SPP / stage[f"{other}_launches"])}
    else:
        alg = (traversal_bytes(cnt, "nearest") + traversal_bytes(cnt, "any")) * (W * H * SPP) / n_counted
        achieved = alg / (sum(ms) / 1e3 / args.steps) / 1e9
        kernel = "k_render<float, PT> (megakernel)"
        per_launch = alg

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
                   "queue_capacity": qopt.get("queue_capacity") or 1 << 25,
                   "tuned": tune["chosen"] if tune else None,
                   "l2": "flushed between timed steps (256 MB write); the 90 MB scene fits in L2"},
        "plain_gpu_msamples_s": round(plain, 3) if plain else None,
        "mrays_per_s": round(value * rays_per_sample, 2),
        "rays_per_sample": round(rays_per_sample, 3),
        "time_to_rmse": ttr,
        "adjoint": adjoint,
        "autotune": tune,
        "batch": batch,
        "large": large,
        "stage_ms": stage,
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": traffic,
                     "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback",
                     "kernel": kernel, "algorithmic_bytes_per_launch": per_launch,
                     "traffic_source": "ncu launch list of the stage kernels (profiles/): DRAM read + "
                                       "write per sample x samples per launch",
                     "second_kernel": secondary},
        "e2e": {"value": round(e2e_val, 3) if e2e_val else None, "unit": "Msamples/s", "h2d_bytes_per_step": 128,
                "d2h_bytes_per_step": W * H * 3, "entry_point": "mt_pathtrace_render",
                "calls_ms": [round(x, 1) for x in e2e_ms], "calls_device_ms": [round(x, 1) for x in e2e_dev_ms],
                "clocks": clk_e2e.summary() if rank == 0 else None},
        "gpu_launches": launches * args.steps,
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


def adjoint_bench(torch, device: int, flush, steps: int = 3):
    """Forward + path-replay backward of the inverse-rendering configuration;
    a gradient is the full 259-parameter vector of an L2 image loss."""
    from marmel_trace_b200 import scenes
    from marmel_trace_b200.adjoint import DiffRenderer

    aw, ah, aspp, adepth = 512, 512, 32, 6
    d = scenes.adjoint_scene()
    r = DiffRenderer(d, aw, ah, aspp, adepth, precision="fp32", integrator="wavefront", device=device)
    target = r.render(s0=1_000_000)
    img = r.render()
    dl = 2.0 * (img - target)
    r.backward(dl)  # warm-up
    torch.cuda.synchronize()
    fw, bw = [], []
    stream = torch.cuda.current_stream()
    for k in range(steps):
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        flush.zero_()
        e[0].record(stream)
        img = r.render(s0=aspp * (k + 1))
        e[1].record(stream)
        r.backward(2.0 * (img - target), s0=aspp * (k + 1))
        e[2].record(stream)
        torch.cuda.synchronize()
        fw.append(e[0].elapsed_time(e[1]))
        bw.append(e[1].elapsed_time(e[2]))
    r.release()
    b = statistics.median(bw) / 1e3
    f = statistics.median(fw) / 1e3
    return {"workload": "inverse rendering 512x512, 32 spp, depth 6, 128 spheres + plane, 32 PBR materials (seed 4)",
            "params": r.n_params, "grads_per_s": round(1.0 / b, 3), "backward_ms": round(1e3 * b, 2),
            "forward_ms": round(1e3 * f, 2), "backward_msamples_s": round(aw * ah * aspp / b / 1e6, 2),
            "forward_msamples_s": round(aw * ah * aspp / f / 1e6, 2),
            "method": "path replay, wavefront form: per batch a primal pass records each sample's radiance, "
                      "then a replay pass re-traces the same paths from their random streams with the stage "
                      "kernels and accumulates the gradient"}


def batch_bench(torch, device: int, lanes: int = 16):
    """The batched uneven workload (64 scenes, seed 3): every image rendered
    by ONE graph launch, with `lanes` concurrent queue sets and with a single
    lane (the images one after another, same launch shape)."""
    from marmel_trace_b200 import scenes
    from marmel_trace_b200.api import GpuScene
    from marmel_trace_b200.batch import BatchRenderer

    wl = scenes.batch_workload(seed=3, n=64)
    gs = [GpuScene(it["desc"], precision="fp32", integrator="wavefront", device=device) for it in wl]
    cams = [it["desc"].make_camera(it["width"], it["height"]) for it in wl]
    items = [(g, c, it["width"], it["height"], it["spp"], it["depth"]) for g, c, it in zip(gs, cams, wl)]
    samples = sum(it["width"] * it["height"] * it["spp"] for it in wl)
    out = {"workload": "64 scenes (seed 3): 500-200k triangles (log-uniform) + 8-40 spheres, resolution from "
                       "256^2/512^2/768x432/1024^2, spp from 16/64/256, depth 4-10, Lambert/GGX/glass/emissive",
           "samples": samples}
    imgs = None
    for nl in (1, lanes):
        br = BatchRenderer(lanes=nl, device=device)
        imgs, _, _ = br.render(items, out=imgs)  # capture + warm-up
        _, item_ms, total = br.render(items, out=imgs)
        br.release()
        item_ms = sorted(item_ms)
        out[f"lanes_{nl}"] = {"ms": round(total, 1), "msamples_s": round(samples / total / 1e3, 2),
                              "item_ms_median": round(statistics.median(item_ms), 1),
                              "item_ms_p90": round(item_ms[int(0.9 * (len(item_ms) - 1))], 1),
                              "item_ms_max": round(item_ms[-1], 1)}
        torch.cuda.empty_cache()
    out["speedup_lanes"] = round(out["lanes_1"]["ms"] / out[f"lanes_{lanes}"]["ms"], 3)
    for g in gs:
        g.release()
    return out


def large_bench(torch, device: int, spp: int = 8, adj_spp: int = 4):
    """Config 5: the 10M-triangle scene (2048^2 water heightfield + 2M-triangle
    trees + 200 spheres + 8 emitters, soft sun; seed 5) at 3840x2160, depth
    12: BVH built on the device, autotuned, one window of `spp` samples timed;
    then the path-replay adjoint (albedos, absorption, ...) over `adj_spp`."""
    from marmel_trace_b200 import _capi, scenes
    from marmel_trace_b200.adjoint import DiffRenderer
    from marmel_trace_b200.api import GpuScene

    LW, LH, LD = 3840, 2160, 12
    t0 = time.perf_counter()
    d = scenes.large_scene()
    gen_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    g = GpuScene(d, precision="fp32", integrator="wavefront", bvh_builder=1, device=device)
    create_s = time.perf_counter() - t0
    tune = g.autotune(d.make_camera(960, 540), 960, 540, 2, LD)
    cam = d.make_camera(LW, LH)
    acc = torch.zeros((LH, LW, 3), device="cuda")
    stream = torch.cuda.current_stream()

    def window(s0, n):
        _capi.check(g.lib.mt_render_accumulate_device(g.h, cam.ref, LW, LH, s0, s0 + n, LD, 0, acc.data_ptr(), 0,
                                                      stream.cuda_stream), "mt_render_accumulate_device")

    window(0, 2)
    torch.cuda.synchronize()
    e = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    e[0].record(stream)
    window(1000, spp)
    e[1].record(stream)
    torch.cuda.synchronize()
    ms = e[0].elapsed_time(e[1])
    g.set_counting(True)
    window(2000, 1)
    st = g.stats()
    g.release()
    ch = tune["chosen"]
    opts = {"traversal": 2 if ch["traversal"] == "dynamic" else 1, "block_size": ch["block"],
            "bvh_width": ch["bvh_width"], "sort_threshold": 0, "queue_capacity": ch["queue_capacity"]}
    r = DiffRenderer(d, LW, LH, adj_spp, LD, precision="fp32", integrator="wavefront", bvh_builder=1, device=device,
                     **opts)
    img = r.render(s0=3000)
    torch.cuda.synchronize()
    e[0].record(stream)
    r.backward(torch.ones_like(img), s0=3000)
    e[1].record(stream)
    torch.cuda.synchronize()
    adj_ms = e[0].elapsed_time(e[1])
    n_params = r.n_params
    r.release()
    samples = LW * LH * spp
    return {"workload": "3840x2160, depth 12, 10,374,259 prims: 2048^2 water heightfield (8.38M triangles) + "
                        "57 trees (1.99M triangles) + 200 glass/metal spheres + 8 emitters + plane, soft sun (seed 5)",
            "scene_gen_s": round(gen_s, 2), "scene_create_s": round(create_s, 2), "bvh": "device build",
            "tuned": ch, "spp_timed": spp, "ms": round(ms, 1), "msamples_s": round(samples / ms / 1e3, 2),
            "mrays_s": round(samples * (st.extension_rays + st.shadow_rays) / (LW * LH) / ms / 1e3, 2),
            "adjoint": {"spp": adj_spp, "params": n_params, "backward_ms": round(adj_ms, 1),
                        "backward_msamples_s": round(LW * LH * adj_spp / adj_ms / 1e3, 2)}}


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
    rank, world, _ = _dist_env()
    if rank != 0:
        return
    from oracle import ref

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
    print(json.dumps({
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
    }), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--integrator", default="wavefront", choices=["megakernel", "wavefront"])
    ap.add_argument("--spp", type=int, default=64, help="samples per pixel per step")
    ap.add_argument("--cpu-spp", type=int, default=1)
    ap.add_argument("--plain-steps", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--large", action="store_true",
                    help="also run the 10M-triangle water / tree scene at 3840x2160 (tens of seconds)")
    ap.add_argument("--queue-capacity", type=int, default=0,
                    help="path slots per wavefront batch (0: the library default, 32M)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
