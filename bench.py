"""Benchmark: path-traced frames of the 1M-triangle torus field on B200.

Workload (one "step"): one progressive frame of the 1920x1080 torus-field
scene (4096 instances of a 256-triangle torus = 1,048,576 triangles, 8
emissive sphere lights, ground plane, sun and sky; seed 2) at 64 samples per
pixel and depth 8 -- 132,710,400 path samples. Step k renders the sample
window [64k, 64k+64), so successive steps refine the same image.

value        : whole-job Msamples/s of the autotuned wavefront integrator
               (device time, CUDA events on the launching stream, max over
               ranks), inputs resident in HBM, L2 flushed between steps.
e2e          : the same metric through the drop-in entry point
               mt_pathtrace_render (camera from host memory, RGB8 image read
               back to host memory every step).
roofline     : the dominant stage (shadow: the occluder-cache pass plus the
               any-hit walk; the extend stage beside it). Algorithmic bytes per
               query: 64 B per inner node whose two child boxes are tested, 48 B
               per triangle test, 16 B per other primitive test, 48 B of ray +
               hit record. `achieved` counts the work the kernels do (their own
               counters); `canonical` beside it counts the reference's cache-less
               walk on its own tree (instrumented, oracle/_ref, in the
               CPU-baseline leg) over the queries the GPU logs on a 480x270
               window, per path sample. `traffic` / `dram_gbs` / `l2_gbs` come
               from the committed ncu capture of the current kernels;
               `l2_frac` puts `l2_gbs` against the L2 read bandwidth
               measured in the same run (`l2_peak_gbs`).
plain_gpu    : the same frames through the megakernel (one thread per pixel,
               the "plain GPU" form of the same estimator).
time_to_rmse : 480x270 frames of the same scene and view: a 16,384-spp
               converged image, then both integrators render samples 0, 1, 2,
               ... of every pixel in 64-spp windows, with the RMSE (linear
               RGB) against the converged image at 64, 128, ..., 1024 spp;
               device time to each RMSE. RMSE 1e-3 itself needs
               mean(sigma^2) / 1e-6 samples per pixel (sigma^2 measured),
               stated beside.
c1           : the 64-sphere configuration (320x240, 8 spp, depth 5): path
               tracer (wavefront and megakernel) and fixed-spp Whitted.
adjoint      : forward + path-replay backward of the inverse-rendering
               configuration (512x512, 32 spp, depth 6, 355 parameters).
inverse      : 200 Adam steps of inverse rendering on that configuration;
               beside them the loss floor (true parameters against the
               target) and the image error of the start and final parameters
               against the true ones on shared samples.
batch        : the batched uneven workload (64 scenes) in one graph launch.
large        : the 10M-triangle water / tree scene at 3840x2160, depth 12
               (cpu_reference_msamples_s: the reference on the same scene and
               view at 960x540, where the host has the ~36 GB it needs).
cpu_baseline : the reference's own multithreaded CPU renderer (oracle/_ref)
               on bounded samples of the same workloads.

--impl reference times the reference's own multithreaded CPU path tracer
(oracle/_ref, compiled from the reference sources) on the same scene.
Multi-GPU (torchrun): every rank renders its own replica of the frame (weak
scaling, no data-path collective); the single-GPU legs run at N = 1 only.
The full detail of each leg (autotune candidates, RMSE curves, inverse-
rendering history) goes to the JSON file named by MT_BENCH_DETAIL (default:
the system temp folder); the printed line carries the summary, with the
headline legs last.
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
CONFIG = {"workload": WORKLOAD, "width": W, "height": H, "spp_per_step": 64, "depth": DEPTH, "scene_seed": 2}


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


def l2_peak_gbs(device: int) -> float:
    """L2 read bandwidth measured on the GPU the bench runs on
    (mt_measure_l2_read_gbs: one launch reads a 32 MB buffer 64 times with
    L2-only 16-byte loads; best of three launches). The denominator of the
    stages' L2 fractions."""
    import ctypes as C

    from marmel_trace_b200 import _capi

    lib = _capi.load()
    out = C.c_double(0.0)
    _capi.check(lib.mt_measure_l2_read_gbs(device, 32 << 20, 64, C.byref(out)), "mt_measure_l2_read_gbs")
    return out.value


def cpu_model() -> str:
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def build_scene():
    from marmel_trace_b200 import scenes

    return scenes.torus_field_scene()


# DRAM and L2 bytes per path sample of the stage kernels, from the ncu capture
# of the stage kernels on the 480x270, 16-spp profiling case (bounces 0-4
# measured, scaled to all bounces by the launch-list time; summarised in
# profiles/wavefront_stages_torus480x270.md). The stage traffic is the queue
# records plus the tree, so it follows the samples.
TRAFFIC = {"shadow": {"dram_bytes_per_sample": 482.0 + 331.0, "l2_bytes_per_sample": 1777.0 + 2865.0},
           "extend": {"dram_bytes_per_sample": 122.0, "l2_bytes_per_sample": 1727.0},
           "source": "ncu capture of the stage kernels, 480x270 x 16 spp (profiles/wavefront_stages_torus480x270.md)"}


def traversal_bytes(st, kind: str, width: int = 2) -> float:
    """Bytes of the counted launch from the GPU's own counters (nearest-hit or
    any-hit): one node record per visit (64 B binary, 128 / 256 B for 4 / 8
    children), 48 B per triangle, 16 B per other primitive, 48 B per ray."""
    if kind == "nearest":
        nodes, prims, tris, rays = st.node_visits, st.prim_tests, st.tri_tests, st.extension_rays
    else:
        nodes, prims, tris, rays = st.any_node_visits, st.any_prim_tests, st.any_tri_tests, st.shadow_rays
    node_bytes = {2: 64.0, 4: 128.0, 8: 256.0}[width]
    return node_bytes * nodes + 48.0 * tris + 16.0 * (prims - tris) + 48.0 * rays


def canonical_bytes(work, n_queries: int, kind: str) -> float:
    """Canonical BVH2 bytes of `n_queries` queries from the reference
    traversal's work (node pairs, triangle tests, other primitive tests)."""
    pairs, tris, other = work
    record = 48.0 if kind == "nearest" else 36.0
    return 64.0 * pairs + 48.0 * tris + 16.0 * other + record * n_queries


class Frames:
    """Timed progressive frames through mt_render_accumulate_device."""

    def __init__(self, g, cam, spp, torch, w=W, h=H, depth=DEPTH):
        self.g, self.cam, self.spp, self.torch = g, cam, spp, torch
        self.w, self.h, self.depth = w, h, depth
        self.stream = torch.cuda.current_stream()
        self.accum = torch.zeros((h, w, 3), dtype=torch.float32, device="cuda")

    def render(self, k: int, spp: int | None = None, base: int = 0, accumulate: int = 0):
        from marmel_trace_b200 import _capi

        n = spp or self.spp
        s0 = base + k * n
        rc = self.g.lib.mt_render_accumulate_device(self.g.h, self.cam.ref, self.w, self.h, s0, s0 + n, self.depth, 0,
                                                    self.accum.data_ptr(), accumulate, self.stream.cuda_stream)
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


def tuned_options(tune) -> dict:
    ch = tune["chosen"]
    return {"queue_capacity": ch["queue_capacity"], "traversal": 2 if ch["traversal"] == "dynamic" else 1,
            "block_size": ch["block"], "bvh_width": ch["bvh_width"], "sort_threshold": ch["sort_threshold"]}


def logged_queries(mt, desc, device, opts, w=480, h=270, spp=1):
    """The traversal queries one window of the wavefront answers (the query
    log), for the canonical accounting: (records, samples, queries seen)."""
    import torch

    from marmel_trace_b200 import _capi

    cam = desc.make_camera(w, h)
    with mt.GpuScene(desc, precision="fp32", integrator="wavefront", device=device, **opts) as g:
        cap = 8_000_000
        g.trace_log_enable(cap)
        acc = torch.zeros((h, w, 3), dtype=torch.float32, device="cuda")
        _capi.check(g.lib.mt_render_accumulate_device(g.h, cam.ref, w, h, 70_000, 70_000 + spp, DEPTH, 0,
                                                      acc.data_ptr(), 0, None), "mt_render_accumulate_device")
        torch.cuda.synchronize()
        rec, seen = g.trace_log_read(cap)
        g.trace_log_enable(0)
    return rec, w * h * spp, seen


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

    detail = {}
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
        qopt = tuned_options(tune)
        detail["autotune"] = tune

    # counting pass (untimed): rays, node visits and primitive tests per sample
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
        ms, means = fr.timed(args.steps, args.warmup, flush, keep_means=False)
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
    g.release()
    single = world == 1

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
        stage = {"extend_ms": round(st.stage_ms[0], 2), "shade_ms": round(st.stage_ms[1], 2),
                 "shadow_ms": round(st.stage_ms[2], 2), "other_ms": round(st.stage_ms[3], 2),
                 "extend_launches": int(st.stage_launches[0]), "shadow_launches": int(st.stage_launches[2])}
        gp.release()
        del fp

    # the queries of a 480x270 window (query log) for the canonical accounting
    queries = None
    if single and args.integrator == "wavefront" and not args.no_cpu_baseline and rank == 0:
        queries = logged_queries(mt, desc, local, qopt)

    plain = None
    if single and args.integrator == "wavefront" and not args.no_plain:
        gm = mt.GpuScene(desc, precision="fp32", integrator="megakernel", device=local)
        fm = Frames(gm, cam, SPP, torch)
        pms, _ = fm.timed(args.plain_steps, 1, flush, base=50_000)
        plain = W * H * SPP * len(pms) / (sum(pms) / 1e3) / 1e6
        gm.release()
        del fm

    ttr = None
    if single and not args.no_rmse and args.integrator == "wavefront":
        ttr, detail["time_to_rmse"] = rmse_bench(torch, mt, desc, local, qopt)
    c1 = None
    if single and not args.no_c1:
        c1 = c1_bench(torch, mt, local)
    adjoint = None
    if single and not args.no_adjoint:
        adjoint = adjoint_bench(torch, local, flush)
    inverse = None
    if single and not args.no_inverse:
        from marmel_trace_b200 import inverse as inv

        res = inv.run(steps=args.inverse_steps, device=local)
        detail["inverse"] = res
        h0, h1 = res["history"][0], res["history"][-1]
        inverse = {"steps": res["steps"], "steps_per_s": round(res["steps_per_s"], 2), "params": res["params"],
                   "loss_first": round(h0["loss"], 6), "loss_last": round(h1["loss"], 6),
                   "loss_at_truth": round(res["loss_at_truth"], 6),
                   "image_rmse_crn": {k: round(v, 5) for k, v in res["image_rmse_crn"].items()},
                   "param_rmse_start": round(res["start_param_rmse"], 4), "param_rmse_last": round(h1["param_rmse"], 4),
                   "group_rmse_start": {k: round(v, 4) for k, v in res["start_groups"].items()},
                   "group_rmse_last": {k: round(v, 4) for k, v in h1["groups"].items()},
                   "materials_seen": res["materials_seen"]}
    batch = None
    if single and not args.no_batch:
        batch, detail["batch"] = batch_bench(torch, local)
    large = None
    if single and not args.no_large:
        large = large_bench(torch, local)

    # roofline of the dominant stage
    peak, peak_kind = peaks()
    l2_peak = l2_peak_gbs(local)
    rays_per_sample = (cnt.extension_rays + cnt.shadow_rays) / n_counted
    bw = qopt.get("bvh_width", 2) or 2
    cpu = None
    if rank == 0 and single and not args.no_cpu_baseline:
        cpu = cpu_baseline(desc, args.cpu_spp, queries)
    kinds = {"shadow": ("any", "shadow stage: k_wf_shadow_cache<float> (cached occluders) + k_wf_shadow<float> "
                               "(any-hit walk of the rest)"),
             "extend": ("nearest", "k_wf_extend<float> (nearest-hit traversal)")}
    roofline = None
    if stage:
        dom = "shadow" if stage["shadow_ms"] >= stage["extend_ms"] else "extend"
        other = "extend" if dom == "shadow" else "shadow"

        def stage_roof(k):
            # achieved: the traversal work the stage's kernels do (GPU
            # counters of a 4-spp pass: node visits, primitive tests, query
            # records); beside it the canonical bytes of the reference's
            # cache-less walk over the same kind of queries (per sample, from
            # the logged queries), whose rate can exceed the HBM peak because
            # the occluder cache answers most connections without a walk and
            # the tree stays in L2
            alg = traversal_bytes(cnt, kinds[k][0], bw) / n_counted * W * H * SPP
            t = stage[f"{k}_ms"] / 1e3
            launches_k = stage[f"{k}_launches"]
            ach = alg / t / 1e9
            tr = TRAFFIC[k]["dram_bytes_per_sample"]
            l2 = TRAFFIC[k]["l2_bytes_per_sample"]
            r = {"kernel": kinds[k][1], "achieved": round(ach, 1), "frac": round(ach / peak, 4),
                 "algorithmic_bytes_per_launch": round(alg / launches_k),
                 "bytes_source": "GPU counters of a 4-spp pass (the walks' node visits and primitive tests)",
                 "traffic": round(tr * W * H * SPP / launches_k) if tr else None,
                 "dram_gbs": round(tr * W * H * SPP / t / 1e9, 1) if tr else None,
                 "l2_gbs": round(l2 * W * H * SPP / t / 1e9, 1) if l2 else None,
                 "l2_frac": round(l2 * W * H * SPP / t / 1e9 / l2_peak, 4) if l2 else None}
            if cpu and cpu.get("canonical"):
                can = cpu["canonical"][f"{k}_bytes_per_sample"] * W * H * SPP
                r["canonical"] = {"bytes_per_launch": round(can / launches_k), "gbs": round(can / t / 1e9, 1),
                                  "frac": round(can / t / 1e9 / peak, 4),
                                  "source": "reference traversal (instrumented, oracle/_ref) over the logged "
                                            "queries of a 480x270 window, per sample"}
            return r

        r_dom, r_oth = stage_roof(dom), stage_roof(other)
        roofline = {"bound": "hbm", "achieved": r_dom["achieved"], "peak": peak, "unit": "GB/s",
                    "frac": r_dom["frac"], "traffic": r_dom["traffic"],
                    "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)" if peak_kind == "measured"
                    else "fallback (6650 GB/s)",
                    "kernel": r_dom["kernel"] + "; per-stage CUDA events over one frame",
                    "algorithmic_bytes_per_launch": r_dom["algorithmic_bytes_per_launch"],
                    "bytes_source": r_dom["bytes_source"], "canonical": r_dom.get("canonical"),
                    "dram_gbs": r_dom["dram_gbs"], "l2_gbs": r_dom["l2_gbs"], "l2_frac": r_dom["l2_frac"],
                    "l2_peak_gbs": round(l2_peak, 1),
                    "l2_peak_source": "mt_measure_l2_read_gbs: 32 MB held in L2 read 64 times in one launch, "
                                      "L2-only loads (measured in this run)",
                    "traffic_source": TRAFFIC["source"], "second_kernel": r_oth}

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
        "config": dict(CONFIG),
        "parallelism": f"replicas x{world}",
        "run": {"integrator": args.integrator, "queue_capacity": qopt.get("queue_capacity") or 1 << 25,
                "tuned": tune["chosen"] if tune else None,
                "l2": "flushed between timed steps (256 MB write); the 90 MB scene fits in L2"},
        "e2e": {"value": round(e2e_val, 3) if e2e_val else None, "unit": "Msamples/s", "h2d_bytes_per_step": 128,
                "d2h_bytes_per_step": W * H * 3, "entry_point": "mt_pathtrace_render",
                "calls_ms": [round(x, 1) for x in e2e_ms], "calls_device_ms": [round(x, 1) for x in e2e_dev_ms],
                "clocks": clk_e2e.summary() if rank == 0 else None},
        "gpu_launches": launches * args.steps,
        "wall_s_timed_loop": round(t_wall, 3),
        "stage_ms": stage,
        "roofline": roofline,
        "rays_per_sample": round(rays_per_sample, 3),
        "mrays_per_s": round(value * rays_per_sample, 2),
    }
    if rank == 0:
        clocks = clk.summary()
        if clocks:
            out["clocks"] = clocks
        if cpu:
            out["cpu_baseline"] = cpu["baseline"]
            out["cpu_more"] = cpu["more"]
        if large and cpu:
            large["cpu_reference_msamples_s"] = cpu["more"].get("c5_msamples_s")
        out["large"] = large
        out["batch"] = batch
        out["c1"] = c1
        out["adjoint"] = adjoint
        out["inverse"] = inverse
        out["time_to_rmse"] = ttr
        out["plain_gpu_msamples_s"] = round(plain, 3) if plain else None
        out["speedup_vs_plain"] = round(value / world / plain, 3) if plain else None
        path = Path(os.environ.get("MT_BENCH_DETAIL") or Path(tempfile.gettempdir()) / f"bench_detail_{os.getpid()}.json")
        try:
            path.parent.mkdir(parents=True, exist_ok=True)
            path.write_text(json.dumps(detail, default=float))
            out["detail_file"] = str(path)
        except OSError:
            pass
        print(json.dumps(out), flush=True)
    if dist:
        dist.destroy_process_group()


def rmse_bench(torch, mt, desc, device: int, opts: dict, w: int = 480, h: int = 270, n_conv: int = 16384,
               n_max: int = 1024, chunk: int = 64, target: float | None = None):
    """Time to RMSE on 480x270 frames of the benchmark scene and view.

    A converged image of `n_conv` samples per pixel (FP32 wavefront, 16
    windows, from which the per-pixel sample variance sigma^2 is also taken)
    is the reference. Each integrator then renders samples 0, 1, 2, ... of
    every pixel in windows of `chunk` samples, accumulating, with device time
    per window; at 64, 128, ..., n_max samples the RMSE (linear RGB) against
    the converged image is taken. The measured RMSE includes the converged
    image's own noise, sigma^2 / n_conv; `rmse_vs_exact` subtracts it.
    `target`: each integrator stops at the first checkpoint where
    rmse_vs_exact <= target, and the summary gives the time to it."""
    from marmel_trace_b200 import _capi

    cam = desc.make_camera(w, h)
    stream = torch.cuda.current_stream()
    acc = torch.zeros((h, w, 3), dtype=torch.float32, device="cuda")

    def window(g, s0, s1, accumulate):
        _capi.check(g.lib.mt_render_accumulate_device(g.h, cam.ref, w, h, s0, s1, DEPTH, 0, acc.data_ptr(),
                                                      accumulate, stream.cuda_stream), "mt_render_accumulate_device")

    gw = mt.GpuScene(desc, precision="fp32", integrator="wavefront", device=device, **opts)
    k_win = 16
    per = n_conv // k_win
    # the converged image in windows of at most 1024 samples, summed per part
    part = torch.zeros((h, w, 3), dtype=torch.float64, device="cuda")
    wins = []
    t0 = time.perf_counter()
    step = min(per, 1024)
    for k in range(k_win):
        part.zero_()
        for s0 in range(5_000_000 + k * per, 5_000_000 + (k + 1) * per, step):
            window(gw, s0, s0 + step, 0)
            part += acc.double()
        wins.append((part / per).cpu().numpy())
    conv_s = time.perf_counter() - t0
    wins = np.stack(wins)
    conv = wins.mean(0)
    sigma2 = float((wins.var(0, ddof=1) * per).mean())  # per-sample variance, mean over pixels and channels
    conv_noise = float(np.sqrt(sigma2 / n_conv))
    checkpoints = []
    n = chunk
    while n <= n_max:
        checkpoints.append(n)
        n *= 2
    curves = {}
    gm = mt.GpuScene(desc, precision="fp32", integrator="megakernel", device=device)
    for name, g in (("wavefront", gw), ("plain_gpu", gm)):
        window(g, 9_000_000, 9_000_000 + chunk, 0)  # warm-up (graph capture) on other samples
        torch.cuda.synchronize()
        t_cum, rows = 0.0, []
        for c in range(n_max // chunk):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            window(g, c * chunk, (c + 1) * chunk, 1 if c else 0)
            e1.record(stream)
            torch.cuda.synchronize()
            t_cum += e0.elapsed_time(e1) / 1e3
            n = (c + 1) * chunk
            if n in checkpoints:
                img = (acc.double() / n).cpu().numpy()
                rmse = float(np.sqrt(np.mean((img - conv) ** 2)))
                exact = float(np.sqrt(max(rmse ** 2 - conv_noise ** 2, 0.0)))
                rows.append({"spp": n, "seconds": round(t_cum, 4), "rmse": round(rmse, 6),
                             "rmse_vs_exact": round(exact, 6)})
                if target is not None and exact <= target:
                    break
        curves[name] = rows
    gw.release()
    gm.release()
    last_w, last_p = curves["wavefront"][-1], curves["plain_gpu"][-1]
    key = "rmse" if target is None else "rmse_vs_exact"
    if target is None:
        target = max(last_w["rmse"], last_p["rmse"])

    def time_to(rows, tau):
        for r in rows:
            if r[key] <= tau:
                return r["seconds"], r["spp"]
        return None, None

    tw, nw = time_to(curves["wavefront"], target)
    tp, np_ = time_to(curves["plain_gpu"], target)
    n_star = sigma2 / 1e-6
    rate_w = last_w["spp"] * w * h / last_w["seconds"]
    rate_p = last_p["spp"] * w * h / last_p["seconds"]
    summary = {"frame": f"{w}x{h}, depth {DEPTH}, same scene and view", "converged_spp": n_conv,
               "converged_noise_rmse": round(conv_noise, 6), "sigma2_per_sample": round(sigma2, 5),
               "target_rmse": round(target, 6), "target_against": key,
               "wavefront_s": tw, "plain_gpu_s": tp, "spp_at_target": [nw, np_],
               "ratio": round(tp / tw, 3) if tw and tp else None,
               "rmse_1e-3": {"spp_needed": round(n_star), "wavefront_s_est": round(n_star * w * h / rate_w, 1),
                             "plain_gpu_s_est": round(n_star * w * h / rate_p, 1)},
               "converged_render_s": round(conv_s, 2)}
    return summary, {"summary": summary, "curves": curves}


def c1_bench(torch, mt, device: int, reps: int = 10):
    """Config 1: the 64-sphere scene at 320x240, 8 spp, depth 5: path tracer
    (wavefront and megakernel; device time per frame) and fixed-spp Whitted
    (--no-pathtrace --no-adaptive; host call with the image read back)."""
    from marmel_trace_b200 import _capi, scenes

    d = scenes.spheres_scene()
    w, h, spp, depth = 320, 240, 8, 5
    cam = d.make_camera(w, h)
    out = {"workload": "320x240, 8 spp, depth 5; plane + 64 spheres (seed 1)"}
    flush = torch.empty(1, device="cuda")
    for name in ("wavefront", "megakernel"):
        with mt.GpuScene(d, precision="fp32", integrator=name, device=device) as g:
            f = Frames(g, cam, spp, torch, w=w, h=h, depth=depth)
            ms, _ = f.timed(reps, 3, flush)
            out[f"pt_{name}_msamples_s"] = round(w * h * spp / (statistics.median(ms) / 1e3) / 1e6, 2)
            out[f"pt_{name}_ms"] = round(statistics.median(ms), 3)
    with mt.GpuScene(d, precision="fp32", device=device) as g:
        rgb = np.zeros((h, w, 3), np.uint8)
        times = []
        for i in range(reps + 2):
            t0 = time.perf_counter()
            _capi.check(g.lib.mt_render_image(g.h, cam.ref, w, h, spp, depth, rgb.ctypes.data), "mt_render_image")
            if i >= 2:
                times.append(time.perf_counter() - t0)
        out["whitted_ms_e2e"] = round(1e3 * statistics.median(times), 3)
        out["whitted_msamples_s_e2e"] = round(w * h * spp / statistics.median(times) / 1e6, 2)
    return out


def adjoint_bench(torch, device: int, flush, steps: int = 3):
    """Forward + path-replay backward of the inverse-rendering configuration;
    a gradient is the full parameter vector of an L2 image loss."""
    from marmel_trace_b200 import scenes
    from marmel_trace_b200.adjoint import DiffRenderer

    aw, ah, aspp, adepth = 512, 512, 32, 6
    d = scenes.adjoint_scene()
    r = DiffRenderer(d, aw, ah, aspp, adepth, precision="fp32", integrator="wavefront", device=device)
    target = r.render(s0=1_000_000)
    img = r.render()
    r.backward(2.0 * (img - target))  # warm-up
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
    n_params = r.n_params
    r.release()
    b = statistics.median(bw) / 1e3
    f = statistics.median(fw) / 1e3
    return {"workload": "512x512, 32 spp, depth 6, 128 spheres + plane, 32 PBR materials (seed 4)",
            "params": n_params, "grads_per_s": round(1.0 / (b + f), 3), "backward_ms": round(1e3 * b, 2),
            "forward_ms": round(1e3 * f, 2), "backward_msamples_s": round(aw * ah * aspp / b / 1e6, 2)}


def batch_bench(torch, device: int, lanes: int = 16):
    """The batched uneven workload (64 scenes, seed 3): every image rendered
    by ONE graph launch, with `lanes` concurrent queue sets, and with a single
    lane (the images one after another, same launch shape)."""
    from marmel_trace_b200 import scenes
    from marmel_trace_b200.api import GpuScene
    from marmel_trace_b200.batch import BatchRenderer

    wl = scenes.batch_workload(seed=3, n=64)
    gs = [GpuScene(it["desc"], precision="fp32", integrator="wavefront", device=device) for it in wl]
    cams = [it["desc"].make_camera(it["width"], it["height"]) for it in wl]
    items = [(g, c, it["width"], it["height"], it["spp"], it["depth"]) for g, c, it in zip(gs, cams, wl)]
    samples = sum(it["width"] * it["height"] * it["spp"] for it in wl)
    out = {"samples": samples}
    detail = {}
    imgs = None
    for nl in (lanes, 1):
        br = BatchRenderer(lanes=nl, device=device)
        if nl == lanes:
            imgs, _, _ = br.render(items, out=imgs)  # capture + warm-up
        imgs, item_ms, total = br.render(items, out=imgs)
        br.release()
        detail[f"lanes_{nl}_item_ms"] = item_ms
        item_ms = sorted(item_ms)
        out[f"lanes_{nl}"] = {"ms": round(total, 1), "msamples_s": round(samples / total / 1e3, 2),
                              "p50_ms": round(statistics.median(item_ms), 1),
                              "p90_ms": round(item_ms[int(0.9 * (len(item_ms) - 1))], 1)}
        torch.cuda.empty_cache()
    out["speedup_lanes"] = round(out["lanes_1"]["ms"] / out[f"lanes_{lanes}"]["ms"], 3)
    for g in gs:
        g.release()
    return out, detail


def large_bench(torch, device: int, spp: int = 2, adj_spp: int = 1):
    """Config 5: the 10M-triangle scene (2048^2 water heightfield + 2M-triangle
    trees + 200 spheres + 8 emitters, soft sun; seed 5) at 3840x2160, depth
    12: BVH built on the device, autotuned on a 1-spp 960x540 probe, one
    window of `spp` samples timed after a 1-spp warm-up; then the path-replay
    adjoint (albedos, absorption, ...) over `adj_spp`."""
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
    tune = g.autotune(d.make_camera(960, 540), 960, 540, 1, LD)
    cam = d.make_camera(LW, LH)
    acc = torch.zeros((LH, LW, 3), device="cuda")
    stream = torch.cuda.current_stream()

    def window(s0, n):
        _capi.check(g.lib.mt_render_accumulate_device(g.h, cam.ref, LW, LH, s0, s0 + n, LD, 0, acc.data_ptr(), 0,
                                                      stream.cuda_stream), "mt_render_accumulate_device")

    e = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    with ClockSampler(device, "_large") as clk:
        window(0, 1)
        torch.cuda.synchronize()
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
    return {"workload": "3840x2160, depth 12, 10.37M prims: 2048^2 water heightfield + 57 trees + 200 spheres "
                        "+ 8 emitters, soft sun (seed 5)",
            "scene_gen_s": round(gen_s, 2), "scene_create_s": round(create_s, 2), "tuned": ch, "spp_timed": spp,
            "ms": round(ms, 1), "msamples_s": round(samples / ms / 1e3, 2),
            "mrays_s": round(samples * (st.extension_rays + st.shadow_rays) / (LW * LH) / ms / 1e3, 2),
            "clocks": clk.summary(),
            "adjoint": {"spp": adj_spp, "params": n_params, "backward_ms": round(adj_ms, 1),
                        "backward_msamples_s": round(LW * LH * adj_spp / adj_ms / 1e3, 2)}}


def cpu_baseline(desc, spp: int, queries=None):
    """The reference's own multithreaded CPU renderer (oracle/_ref) on bounded
    samples of the same workloads, outside every timed GPU region:
    * the benchmark frame: pathtrace_render of the full 1080p frame at `spp`;
    * its traversal work per query on the reference's tree, for the logged
      queries of a 480x270 window (the roofline's canonical bytes), and its
      CPU Mrays/s on those queries;
    * config 1 (path tracer and Whitted), the adjoint configuration's central
      finite-difference gradient cost, and config 3's scenes one after
      another (a sample of 8 of the 64), and config 5 at a quarter of its
      resolution where the host has the memory for it."""
    from marmel_trace_b200 import scenes
    from oracle import ref

    cores = os.cpu_count() or 1
    os.environ["RAYTRACER_THREADS"] = str(cores)
    rs = ref.RefScene.from_desc(desc, ref.scene_camera(desc, W, H))
    t0 = time.perf_counter()
    rs.pathtrace_render(W, H, spp, DEPTH)
    dt = time.perf_counter() - t0
    baseline = {"value": round(W * H * spp / dt / 1e6, 4), "unit": "Msamples/s", "cores": cores, "kind": "reference",
                "cpu": cpu_model(),
                "sample": f"pathtrace_render full frame {W}x{H} at {spp} spp, depth {DEPTH} "
                          f"({dt:.1f} s, RAYTRACER_THREADS={cores})"}
    more = {}
    canonical = None
    if queries is not None:
        rec, n_samples, seen = queries
        o = rec["o"].astype(np.float64)
        d = rec["d"].astype(np.float64)
        ext = rec["kind"] == 0
        shd = rec["kind"] == 1
        t0 = time.perf_counter()
        we = rs.bvh_work("nearest", o[ext], d[ext], 1e-4, 1e30)
        ws = rs.bvh_work("any", o[shd], d[shd], 1e-3, rec["t"][shd].astype(np.float64))
        count_s = time.perf_counter() - t0
        n_ext, n_shd = int(ext.sum()), int(shd.sum())
        canonical = {"extend_bytes_per_sample": canonical_bytes(we, n_ext, "nearest") / n_samples,
                     "shadow_bytes_per_sample": canonical_bytes(ws, n_shd, "any") / n_samples}
        more["canonical"] = {"queries": [n_ext, n_shd], "samples": n_samples, "logged": seen,
                             "node_pairs_per_ray": [round(we[0] / max(n_ext, 1), 2), round(ws[0] / max(n_shd, 1), 2)],
                             "tri_tests_per_ray": [round(we[1] / max(n_ext, 1), 2), round(ws[1] / max(n_shd, 1), 2)],
                             "bytes_per_sample": [round(canonical["extend_bytes_per_sample"]),
                                                  round(canonical["shadow_bytes_per_sample"])],
                             "count_s": round(count_s, 2)}
        # the reference's own query rate on these rays (all host threads)
        t0 = time.perf_counter()
        rs.queries("nearest", o[ext], d[ext], 1e-4, 1e30)
        rs.queries("shadow", o[shd], d[shd], 1e-3, rec["t"][shd].astype(np.float64))
        q_s = time.perf_counter() - t0
        more["mrays_s"] = round((n_ext + n_shd) / q_s / 1e6, 3)
    rs.free()
    # config 1
    c1 = scenes.spheres_scene()
    r1 = ref.RefScene.from_desc(c1, ref.scene_camera(c1, 320, 240))
    t0 = time.perf_counter()
    r1.pathtrace_render(320, 240, 8, 5)
    t_pt = time.perf_counter() - t0
    t0 = time.perf_counter()
    r1.whitted_render(320, 240, 8, 5)
    t_wh = time.perf_counter() - t0
    r1.free()
    more["c1_pt_msamples_s"] = round(320 * 240 * 8 / t_pt / 1e6, 3)
    more["c1_whitted_msamples_s"] = round(320 * 240 * 8 / t_wh / 1e6, 3)
    # config 4: one central-difference gradient = 2 renders per parameter of
    # the 512x512, 32-spp image; one render timed at 1 spp and scaled
    c4 = scenes.adjoint_scene()
    r4 = ref.RefScene.from_desc(c4, ref.scene_camera(c4, 512, 512))
    t0 = time.perf_counter()
    r4.pathtrace_render(512, 512, 1, 6)
    t1 = time.perf_counter() - t0
    r4.free()
    n_params = 11 * len(c4.materials) + 3
    more["c4_fd_grads_per_s"] = round(1.0 / (2 * n_params * 32 * t1), 6)
    more["c4_fd_note"] = f"2 x {n_params} renders of 512x512 x 32 spp; one 1-spp render took {t1:.3f} s"
    # config 3: a sample of the 64 scenes, one after another, at 1 spp
    wl = scenes.batch_workload(seed=3, n=64)[::8]
    n3, t3 = 0, 0.0
    for it in wl:
        r3 = ref.RefScene.from_desc(it["desc"], ref.scene_camera(it["desc"], it["width"], it["height"]))
        t0 = time.perf_counter()
        r3.pathtrace_render(it["width"], it["height"], 1, it["depth"])
        t3 += time.perf_counter() - t0
        n3 += it["width"] * it["height"]
        r3.free()
    more["c3_sequential_msamples_s"] = round(n3 / t3 / 1e6, 3)
    # config 5: the large scene and view at 960x540, 1 spp, depth 12. The
    # reference keeps two 1632-byte copies of every primitive (about 36 GB
    # here), so this runs only with room for it on the host.
    avail = _host_available_bytes()
    if avail >= C5_HOST_BYTES:
        d5 = scenes.large_scene()
        t0 = time.perf_counter()
        r5 = ref.RefScene.from_desc(d5, ref.scene_camera(d5, 960, 540))
        build_s = time.perf_counter() - t0
        t0 = time.perf_counter()
        r5.pathtrace_render(960, 540, 1, 12)
        t5 = time.perf_counter() - t0
        r5.free()
        del d5
        more["c5_msamples_s"] = round(960 * 540 / t5 / 1e6, 4)
        more["c5_note"] = (f"pathtrace_render of the large scene and view at 960x540, 1 spp, depth 12: {t5:.1f} s "
                           f"(scene and tree build {build_s:.0f} s)")
    else:
        more["c5_msamples_s"] = None
        more["c5_note"] = f"skipped: {avail / 1e9:.0f} GB of host memory available, {C5_HOST_BYTES / 1e9:.0f} GB wanted"
    return {"baseline": baseline, "more": more, "canonical": canonical}


# host memory the reference's copy of the large scene wants, with headroom
C5_HOST_BYTES = 80e9


def _host_available_bytes() -> float:
    try:
        import psutil

        return float(psutil.virtual_memory().available)
    except Exception:
        return 0.0


def run_reference(args):
    rank, world, _ = _dist_env()
    if rank != 0:
        return
    from oracle import ref

    desc = build_scene()
    cam = ref.scene_camera(desc, W, H)
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
        "config": dict(CONFIG),
        "parallelism": f"{cores} CPU threads",
        "cpu_baseline": {"value": round(value, 4), "unit": "Msamples/s", "cores": cores, "kind": "reference",
                         "cpu": cpu_model(),
                         "sample": f"each step: pathtrace_render of the full frame at {spp} spp (a bounded sample of "
                                   f"the 64-spp step; the metric is a per-sample rate)"},
        "e2e": {"value": round(value, 4), "unit": "Msamples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def profile_case(w: int = 480, h: int = 270, spp: int = 16):
    """The capture case of the stage kernels: the benchmark scene and view at
    480x270, 16 spp (2.07M paths, about 2 GB of queues), the benchmark's
    stage options (block 128, sort >= 256K, binary tree, grid-stride), plain
    launches so every stage kernel is its own launch. Two frames: the first
    warms the occluder cache, so captures skip its launches."""
    import torch

    import marmel_trace_b200 as mt

    desc = build_scene()
    cam = desc.make_camera(w, h)
    with mt.GpuScene(desc, precision="fp32", integrator="wavefront", use_graph=0, sort_threshold=1 << 18) as g:
        f = Frames(g, cam, spp, torch, w=w, h=h)
        for k in range(2):
            f.render(k)
        torch.cuda.synchronize()


def profile_case_glass(w: int = 512, h: int = 512, spp: int = 4):
    """The capture case of the pass-through shadow chains: item 41 of the
    batched workload (43k triangles, a third of the materials glass, seed 3)
    at 512x512, 4 spp, library defaults, plain launches, two frames."""
    import torch

    import marmel_trace_b200 as mt
    from marmel_trace_b200 import _capi, scenes

    it = scenes.batch_workload(seed=3, n=64)[41]
    cam = it["desc"].make_camera(w, h)
    with mt.GpuScene(it["desc"], precision="fp32", integrator="wavefront", use_graph=0) as g:
        acc = torch.zeros((h, w, 3), dtype=torch.float32, device="cuda")
        for r in range(2):
            _capi.check(g.lib.mt_render_accumulate_device(g.h, cam.ref, w, h, spp * r, spp * (r + 1), it["depth"], 0,
                                                          acc.data_ptr(), 0, None), "mt_render_accumulate_device")
        torch.cuda.synchronize()


def profile_case_adjoint(w: int = 512, h: int = 512, spp: int = 8):
    """The capture case of the adjoint: the inverse-rendering scene (128
    spheres, 32 PBR materials, seed 4) at 512x512, 8 spp, depth 6 (2.1M
    paths), plain launches. Two forward + backward pairs: the first allocates
    the replay buffers, so captures skip its launches."""
    import torch

    from marmel_trace_b200 import scenes
    from marmel_trace_b200.adjoint import DiffRenderer

    r = DiffRenderer(scenes.adjoint_scene(), w, h, spp, 6, use_graph=0)
    target = r.render(s0=1_000_000)
    for k in range(2):
        img = r.render(s0=spp * k)
        r.backward(2.0 * (img - target), s0=spp * k)
    torch.cuda.synchronize()
    r.release()


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
    ap.add_argument("--inverse-steps", type=int, default=200)
    for leg in ("cpu-baseline", "plain", "e2e", "adjoint", "inverse", "autotune", "batch", "large", "rmse", "c1"):
        ap.add_argument(f"--no-{leg}", action="store_true")
    ap.add_argument("--queue-capacity", type=int, default=0,
                    help="path slots per wavefront batch (0: the library default, 32M)")
    ap.add_argument("--rmse-target", type=float, default=0.0,
                    help="only measure the time of both integrators to this RMSE against the exact image "
                         "(480x270, 262,144-spp converged reference, 1024-spp windows); prints its own JSON line")
    ap.add_argument("--profile-case", nargs="?", const="torus", default=None, choices=["torus", "glass", "adjoint"],
                    help="only render a small profiling case twice, plain launches, for ncu captures; prints "
                         "nothing. torus: the benchmark scene at 480x270, 16 spp; glass: item 41 of the batched "
                         "workload at 512x512, 4 spp (the pass-through shadow chains); adjoint: forward + backward "
                         "of the inverse-rendering scene at 512x512, 8 spp")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.profile_case:
        {"torus": profile_case, "glass": profile_case_glass, "adjoint": profile_case_adjoint}[args.profile_case]()
        return
    if args.rmse_target > 0:
        import torch

        import marmel_trace_b200 as mt

        torch.cuda.set_device(0)
        desc = build_scene()
        with ClockSampler(0, "_rmse") as clk:
            summary, detail = rmse_bench(torch, mt, desc, 0, {}, n_conv=262144, n_max=131072, chunk=1024,
                                         target=args.rmse_target)
        summary["clocks"] = clk.summary()
        print(json.dumps({"time_to_rmse": summary, "curves": detail["curves"]}), flush=True)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
