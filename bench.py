"""Throughput benchmark of the ray-casting path (one JSON line on rank 0).

Workload (default): the triangle-mesh scene -- a level-8 displaced
icosphere (1,310,720 triangles) plus 16 displaced 50k-triangle tori, 4 point
lights with shadow rays, mirror bounce (reflect 0.2) and refraction through
the 4 glass tori (ior 1.5), 1920x1080 at 4 samples per pixel.  A step is
one frame of that scene with the scene resident in HBM.

metric: Mrays/s -- every scene query counts (primary, each glass pass of a
shadow ray, each reflection/refraction segment); the per-frame ray count
comes from the renderer's own device counters (a counting frame before the
timed region; the path is deterministic, every frame issues the same rays).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--form wavefront|plain]
                  [--impl ours|reference]

Beside the timed value the line carries the metric's other parts:
  plain     the plain FP32 form (the drop-in) on the same scene, same
            process, same timing (vs_plain = value / plain value);
  serving   p50/p99 latency and Mrays/s of a 64-request prefix of the
            seeded serving stream through the request loop (N = 1 only);
  e2e       the same frame through the host-array drop-in call (upload,
            BVH build, render and read-back inside the timed region);
  cpu_baseline.ray_count_check
            the device's ray count on an 8x8 region against the oracle's
            count of the same scene queries.

--gpus N > 1 runs under torchrun: every rank renders its own replica of the
frame on its own GPU (the path has no data exchange: "replicas only",
weak scaling), timing is the max over ranks.

--impl reference times the reference's own per-pixel code compiled for the
host cores (oracle/_ref/libsheen_ref_host.so) on a bounded band of rows of
the same frame, all host threads; its ray count is that band's count from
this renderer's counters (same queries by construction).
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
sys.path.insert(0, os.path.join(ROOT, "tests"))

W, H, SPP = 1920, 1080, 4
CPU_BAND = (480, 512)
# DRAM bytes (read + write) per shadow ray of the shadow stage, from the
# one-pass ncu capture of the full-size mesh frame (profiles/
# wave_shadow_refill_mesh_1920x1080_4spp_dram.md); the roofline's traffic
# per launch is this times the launch's shadow rays.
SHADOW_DRAM_BYTES_PER_RAY = 5061321984 / 38552584


class quiet_stdout:
    """Sends file descriptor 1 to /dev/null for the duration: the reference's
    shading code prints one debug line per caustic gather (render_kernel.cu:
    291-294), millions per frame on the caustics workload, on the host path
    and through the device printf buffer alike."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        self.null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self.null, 1)
        return self

    def __exit__(self, *exc):
        sys.stdout.flush()
        os.dup2(self.saved, 1)
        os.close(self.saved)
        os.close(self.null)


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return {"hbm_gbs": d["hbm_gbs"], "src": "measured", "sm_max_mhz": d.get("sm_max_mhz", 1965.0)}
    return {"hbm_gbs": 6650.0, "src": "fallback", "sm_max_mhz": 1965.0}


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 7:
                self.samples.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[3 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def dist_setup(n):
    import torch
    import torch.distributed as dist
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    return rank, world, local


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


WORKLOADS = {
    0: "spheres: 64 seeded spheres + ground plane + 1 point light, reflect 0.3, 640x480, 1 spp",
    1: "mesh: displaced icosphere L8 (1,310,720 tris) + 16 displaced 50k-tri tori, 1920x1080, 4 spp, "
       "4 point lights, reflect 0.2, 4 glass tori ior 1.5",
    2: "analytic: 258 superellipsoids, 64 Bezier lathes, 64 Bezier prisms, 32 Catmull-Rom sweeps, "
       "fBm heightfield, depth-3 CSG tree; 1920x1080, 4 spp",
    3: "caustics: glass sphere + glass lathe over a diffuse plane, 1 spot light, 4M photons (hash grid, "
       "cell 0.2), 1920x1080, 16 spp",
}


EXT_WORKLOADS = {
    1: "16 tori as instances of one 50,000-triangle mesh (two-level BVH), reflect + refract recursion to 4 "
       "bounces (BVH4 megakernel)",
    2: "exact cubic-Bezier lathes and prisms (FP64 root isolation), two-exponent superellipsoids, "
       "1024x1024 FP32 height grid, 128 more CSG trees over spheres, boxes and cones",
}


def scene_ext(scene, args):
    """The extension handed to sheen_scene_create_ext: False without
    --extended, the generator's own (True), or a copy with --max-depth."""
    import ctypes

    from sheen_b200 import contract as C
    if not args.extended:
        return False
    if args.max_depth < 0:
        return True
    x = C.SheenSceneExt.from_buffer_copy(ctypes.string_at(scene.ext_ptr, ctypes.sizeof(C.SheenSceneExt)))
    x.max_depth = args.max_depth
    return x


def make_scene(args):
    """The workload's scene; sets the frame size and spp from the generator."""
    import sheen_b200 as sb
    global W, H, SPP
    photons = args.photons if args.photons > 0 else (4000000 if args.config == 3 else 0)
    scene = sb.generate_scene(args.config, args.seed, args.detail if args.config == 1 else 0, photons,
                              extended=args.extended)
    st = scene.settings
    W, H, SPP = st["width"], st["height"], st["aa"]
    # smaller frames of the same scene (profiling captures)
    W = args.width or W
    H = args.height or H
    SPP = args.spp or SPP
    global CPU_BAND
    y0 = (H // 2) // 16 * 16
    # a band of two 16-row blocks; one for the printf-bound caustics workload
    rows = 16 if (scene.view.photons > 0 and scene.view.caustics > 0) else 32
    CPU_BAND = (y0, min(H, y0 + rows))
    return scene


def run_ours(args):
    import torch

    import sheen_b200 as sb
    rank, world, local = dist_setup(args.gpus)
    sb.init(local, 100)
    form = sb.FORM_WAVEFRONT if args.form == "wavefront" else sb.FORM_PLAIN
    scene = make_scene(args)

    # End to end through the drop-in call: host scene arrays in, host RGBA
    # out, per step: BVH build + scene upload + render + read back.  Run
    # before the resident scene below exists: a one-call render next to a
    # resident scene and its frame queues was measured 5-20 ms slower a call
    # (the library's memory pool then serves two working sets), which is not
    # the drop-in caller's situation.
    # (scenes with extensions: sheen_scene_create_ext + render to a host
    # buffer + destroy, the extension's public path)
    ext_arg = scene_ext(scene, args)
    img = np.empty((H, W, 4), np.float32)
    e2e_steps = max(1, min(args.steps, 3))

    def one_call():
        if not args.extended:
            return sb.render_rgba(scene, W, H, SPP, form)
        d = sb.DeviceScene(scene, form, ext=ext_arg)
        out_img, out_st = d.render_host(W, H, SPP)
        d.close()
        return out_img, out_st

    # warm-up calls: the library's memory pool grows to its working set over
    # the first one or two calls (measured: 80 ms builds, then 13.5 ms)
    for _ in range(max(1, args.warmup)):
        one_call()
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        img, st2 = one_call()
    e2e_s = max_over_ranks(time.perf_counter() - t0, world)

    t0 = time.perf_counter()
    ds = sb.DeviceScene(scene, form, ext=ext_arg)
    create_s = time.perf_counter() - t0
    out = torch.empty((H, W, 4), dtype=torch.float32, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")   # > 126 MB L2
    stream = torch.cuda.current_stream().cuda_stream

    # counting frame: rays per frame and the traversal counters
    st = ds.render_device(W, H, SPP, out.data_ptr(), stream, count_rays=True)
    rays = st["total_rays"]
    # box/primitive test counts: one instrumented frame of the same traversal
    stn = ds.render_device(W, H, SPP, out.data_ptr(), stream, count_nodes=True)
    nodes, prims = stn["node_visits"], stn["prim_tests"]
    assert stn["total_rays"] == rays or form == sb.FORM_WAVEFRONT

    # --tiles N: each frame as N uneven screen tiles in one batch (one pass
    # of the queue kernels over all tiles) instead of the captured frame graph
    tiles = uneven_tiles(W, H, args.tiles, 7) if args.tiles > 0 else None

    def frame():
        if tiles is None:
            ds.render_device(W, H, SPP, out.data_ptr(), stream)
        else:
            sb.render_batch([(ds, W, H, SPP, t, out.data_ptr()) for t in tiles], stream)

    for _ in range(args.warmup):
        frame()
    torch.cuda.synchronize()

    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for i in range(args.steps):
            flush.fill_(float(i))                      # evict L2 between frames (outside the events)
            starts[i].record()
            frame()
            ends[i].record()
        torch.cuda.synchronize()
    barrier(world)
    ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
    ms = max_over_ranks(ms, world)
    frame_ms = ms / args.steps
    value = rays * args.steps * world / (ms / 1e3) / 1e6
    e2e = rays * e2e_steps * world / e2e_s / 1e6

    # The metric's denominator: the plain FP32 form (the drop-in) on the same
    # scene in the same process, timed the same way (CUDA events, L2 flushed
    # before each frame).
    plain = None
    if form == sb.FORM_WAVEFRONT and not args.no_plain:
        pds = sb.DeviceScene(scene, sb.FORM_PLAIN)
        prays = pds.render_device(W, H, SPP, out.data_ptr(), stream, count_rays=True)["total_rays"]
        pds.render_device(W, H, SPP, out.data_ptr(), stream)
        torch.cuda.synchronize()
        pk_frames = 3
        p_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(pk_frames)]
        barrier(world)
        for i, (a, b) in enumerate(p_ev):
            flush.fill_(float(i))
            a.record()
            pds.render_device(W, H, SPP, out.data_ptr(), stream)
            b.record()
        torch.cuda.synchronize()
        p_ms = max_over_ranks(sum(a.elapsed_time(b) for a, b in p_ev) / pk_frames, world)
        pds.close()
        plain = {"value": round(prays * world / (p_ms / 1e3) / 1e6, 2), "unit": "Mrays/s",
                 "ms_per_step": round(p_ms, 3), "rays_per_frame": prays, "frames": pk_frames,
                 "form": "plain FP32 (drop-in megakernel, reference traversal order)"}

    # A short serving run: a prefix of the seeded Poisson request stream
    # (20 requests/s, every workload generator, mixed sizes and spp) through
    # the request loop, for the metric's p50/p99 latency.
    serving = None
    if world == 1 and args.serve_requests > 0:
        res = serve_stream(args.serve_requests, args.rate, args.inflight, args.seed, 1, 0, local)
        serving = {"value": round(res["value"], 2), "unit": "Mrays/s", "requests": len(res["stream"]),
                   "rate_per_s": args.rate, "max_inflight": args.inflight,
                   "latency_ms": latency_summary(res), "clocks": res["clocks"],
                   "workload": "first %d requests of the serving stream (%s)" % (len(res["stream"]), SERVE_WORKLOAD)}

    pk = peaks()
    fp32_peak = 148 * 128 * 2 * pk["sm_max_mhz"] * 1e6
    # Algorithmic bytes and FP32 work: 32 B ray in +
    # 16 B hit out per ray, the node record per node visited, 48 B per
    # triangle tested; 14 FP32 ops per box test (a BVH4 node visit tests 4
    # boxes; the plain form counts single boxes), 35 per triangle test.
    # the wavefront form's node counter counts 4-wide BVH4 node visits on
    # triangle scenes and single boxes of the per-class binary trees on the
    # others (the workloads do not mix triangles with those classes)
    wide = form == sb.FORM_WAVEFRONT and scene.view.num_triangles > 0
    b_node, boxes_per_visit = (64, 4) if wide else (32, 1)
    bytes_alg = rays * 48 + nodes * b_node + prims * 48
    fp32_flops = nodes * boxes_per_visit * 14 + prims * 35
    frame_roof = {"achieved_gbs": round(bytes_alg / (frame_ms / 1e3) / 1e9, 1),
                  "frac": round(bytes_alg / (frame_ms / 1e3) / 1e9 / pk["hbm_gbs"], 4),
                  "algorithmic_bytes": int(bytes_alg), "fp32_flops": int(fp32_flops),
                  "fp32_tflops": round(fp32_flops / (frame_ms / 1e3) / 1e12, 2)}

    # Dominant kernel.  Wavefront: the shadow stage (3 launches a frame),
    # timed with CUDA events at the stage boundaries of directly launched
    # frames (L2 flushed before each); its node / triangle tests are the
    # counting megakernel's shadow-query counters (same walks).  Plain: the
    # single megakernel launch, timed above.
    stages = None
    mega = form == sb.FORM_WAVEFRONT and uses_megakernel(ds, W, H, SPP)
    if form == sb.FORM_WAVEFRONT and not mega:
        profs = []
        for i in range(max(3, args.steps // 2)):
            flush.fill_(float(i))
            profs.append(ds.profile_stages(W, H, SPP, out.data_ptr(), stream))
        med = lambda key: float(np.median([p[key] if not isinstance(p[key], list) else sum(p[key]) for p in profs]))
        stages = {k: round(med(k), 3) for k in ("primary_ms", "shadow_ms", "reflect_ms", "refract_ms", "resolve_ms",
                                                 "total_ms")}
        stages["shadow_launch_ms"] = [round(float(np.median([p["shadow_ms"][j] for p in profs])), 3) for j in range(3)]
        stages["shadow_rays"] = list(profs[0]["shadow_rays"])
        stages["share_shadow"] = round(stages["shadow_ms"] / stages["total_ms"], 3)
        k_name, k_launches = "wave_shadow_refill (shadow stage)", 3
        k_ms = stages["shadow_ms"]
        k_rays, k_nodes, k_prims = stn["shadow_rays"], stn["shadow_node_visits"], stn["shadow_prim_tests"]
    else:
        k_name, k_launches, k_ms = ("mega_bvh4_kernel (small frame)" if mega else "plain_kernel"), 1, frame_ms
        k_rays, k_nodes, k_prims = rays, nodes, prims
    k_bytes = k_rays * 48 + k_nodes * b_node + k_prims * 48
    k_flops = k_nodes * boxes_per_visit * 14 + k_prims * 35
    k_gbs = k_bytes / (k_ms / 1e3) / 1e9
    k_tflops = k_flops / (k_ms / 1e3) / 1e12
    hbm_bound = k_bytes / (pk["hbm_gbs"] * 1e9) >= k_flops / fp32_peak
    traffic = None
    if form == sb.FORM_WAVEFRONT and (W, H, SPP) == (1920, 1080, 4) and args.config == 1:
        traffic = int(SHADOW_DRAM_BYTES_PER_RAY * k_rays / k_launches) if SHADOW_DRAM_BYTES_PER_RAY else None
    clocks = clk.summary()
    line = {
        "metric": "Mrays/s", "value": round(value, 2), "unit": "Mrays/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(frame_ms, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded generator)",
        "config": {"workload": WORKLOADS.get(args.config, f"config {args.config}")
                   + (" + extension column: " + EXT_WORKLOADS[args.config] if args.extended else "")
                   + (" (max_depth %d)" % args.max_depth if args.extended and args.max_depth >= 0 else ""),
                   "triangles": scene.view.num_triangles, "width": W, "height": H, "spp": SPP,
                   "form": args.form, "parallelism": f"replicas{world}",
                   "frame": (f"{args.tiles} uneven tiles in one batched pass" if args.tiles > 0
                             else "whole frame, one BVH4 megakernel launch (%s)" % (
                                 "reflect + refract recursion runs outside the queue stages"
                                 if args.extended and args.config == 1 and args.max_depth != 0 and
                                 args.max_depth != 1 else "small frame") if mega
                             else "whole frame, captured CUDA graph"),
                   "l2": "256 MB buffer written between timed frames; scene arrays exceed L2",
                   "rays_per_frame": rays, "box_tests_per_frame": nodes, "prim_tests_per_frame": prims,
                   "scene_create_s": round(create_s, 3), "device_bytes": ds.device_bytes,
                   "tuning": {k: sb.tune_get(k) for k in sb.TUNE_KEYS}},
        "e2e": {"value": round(e2e, 2), "unit": "Mrays/s",
                "h2d_bytes_per_step": int(st2["upload_bytes"]),
                "d2h_bytes_per_step": W * H * 16,
                "call": ("sheen_scene_create_ext + sheen_scene_render_host + destroy (upload + BVH build + render "
                         "+ readback)" if args.extended else
                         "sheen_render_scene_rgba (upload + BVH build + render + readback)"),
                "scene_build_ms": round(st2["build_ms"], 1), "scene_upload_ms": round(st2["upload_ms"], 1)},
        "roofline": {"bound": "hbm" if hbm_bound else "fp32", "achieved": round(k_gbs, 1), "peak": pk["hbm_gbs"],
                     "unit": "GB/s", "frac": round(k_gbs / pk["hbm_gbs"], 4), "traffic": traffic,
                     "peak_source": pk["src"], "kernel": k_name, "launches_per_frame": k_launches,
                     "avg_launch_ms": round(k_ms / k_launches, 3),
                     "algorithmic_bytes_per_launch": int(k_bytes / k_launches),
                     "fp32": {"achieved_tflops": round(k_tflops, 2), "peak_tflops_nominal": round(fp32_peak / 1e12, 1),
                              "frac": round(k_tflops * 1e12 / fp32_peak, 4)},
                     "frame": frame_roof},
        "stages": stages,
        "gpu_launches": args.steps * (1 if mega else launches_per_frame(form)),
        "clocks": clocks,
    }
    if plain is not None:
        line["plain"] = plain
        line["vs_plain"] = round(value / plain["value"], 3)
    if serving is not None:
        line["serving"] = serving
    if rank == 0 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(ds, scene, stream, out)
    if rank == 0 and not args.no_ref_gpu:
        if scene.view.photons > 0 and scene.view.caustics > 0 and W * H * SPP > 4_000_000:
            # render_kernel.cu:291-294 printf()s one line per caustic gather:
            # ~33M lines for this frame, far past the bench's time bound
            line["reference_gpu"] = {"value": None, "unavailable": "printf-bound: the reference kernel prints one "
                                     "debug line per caustic gather (render_kernel.cu:291-294); not timed at this size"}
        else:
            line["reference_gpu"] = reference_gpu(scene, rays)
    if rank == 0:
        print(json.dumps(line), flush=True)
    ds.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def uneven_tiles(W, H, n, seed):
    """n rectangles of uneven size covering a W x H frame: rows of uneven
    height, each cut into tiles of uneven width."""
    rng = np.random.default_rng(seed)
    rows = max(1, int(np.sqrt(n)))
    cols = [n // rows + (1 if r < n % rows else 0) for r in range(rows)]
    ys = [0] + np.sort(rng.choice(np.arange(1, H), rows - 1, replace=False)).tolist() + [H]
    tiles = []
    for r in range(rows):
        xs = [0] + np.sort(rng.choice(np.arange(1, W), cols[r] - 1, replace=False)).tolist() + [W]
        tiles += [(xs[c], ys[r], xs[c + 1], ys[r + 1]) for c in range(cols[r])]
    return tiles


def uses_megakernel(ds, W, H, spp):
    """True when the library renders this frame of a wavefront-form scene on
    the BVH4 megakernel (sheen_scene_frame_path): small frames (the
    wave.mega_samples rule) and scenes outside the queue pipeline."""
    import sheen_b200 as sb
    return ds.frame_path(W, H, spp) == sb.PATH_MEGAKERNEL


def launches_per_frame(form):
    import sheen_b200 as sb
    # plain: one megakernel; wavefront: primary, 3 x shadow, mirror,
    # refraction, resolve, tally (one CUDA graph launch)
    return 1 if form == sb.FORM_PLAIN else 8


def band_rays(ds, stream, out):
    st = ds.render_region(W, H, SPP, 0, CPU_BAND[0], W, CPU_BAND[1], out.data_ptr(), stream, count_rays=True)
    return st["total_rays"]


def cpu_baseline(ds, scene, stream, out, steps=1):
    """The reference's own code on the host cores over a band of rows."""
    from oracle_bindings import RefHost
    if not RefHost.available():
        return {"value": None, "unit": "Mrays/s", "cores": 0, "kind": "reference",
                "sample": "unavailable: oracle/_ref not built"}
    ref = RefHost()
    threads = ref.lib.sheen_ref_max_threads()
    with quiet_stdout():
        h = ref.scene(scene.view_ptr, threads)
    rays = band_rays(ds, stream, out)
    with quiet_stdout():
        t0 = time.perf_counter()
        for _ in range(steps):
            ref.render(h, W, H, SPP, threads, CPU_BAND[0] // 16, CPU_BAND[1] // 16)
        dt = time.perf_counter() - t0
    return {"value": round(rays * steps / dt / 1e6, 3), "unit": "Mrays/s", "cores": threads, "kind": "reference",
            "sample": f"rows {CPU_BAND[0]}-{CPU_BAND[1]} of the {W}x{H} {SPP} spp frame ({rays} rays), "
                      f"{steps} pass(es), {dt:.1f} s",
            "ray_count_check": ray_count_check(ds, scene, stream, out)}


def ray_count_check(ds, scene, stream, out):
    """The ray count cross-check: the renderer's device counters against the
    oracle's count of the same scene queries (its brute-force C restatement
    of the path) on an 8x8-pixel region at the centre of the frame."""
    from oracle_bindings import Oracle
    x0, y0 = (W // 2) & ~7, (H // 2) & ~7
    reg = (x0, y0, x0 + 8, y0 + 8)
    dev = ds.render_region(W, H, SPP, *reg, out.data_ptr(), stream, count_rays=True)["total_rays"]
    o = Oracle()
    with quiet_stdout():
        h = o.scene(scene.view_ptr)
        t0 = time.perf_counter()
        _, q = o.render_region(h, W, H, SPP, *reg)
        dt = time.perf_counter() - t0
    h.close()
    return {"region": list(reg), "device_rays": dev, "oracle_rays": q, "equal": dev == q,
            "oracle_s": round(dt, 2)}


def reference_gpu(scene, rays, steps=3):
    """The reference's own CUDA kernel (render_kernel.cu compiled unchanged for
    sm_100a, oracle/_ref/libsheen_ref_gpu.so) on the same frame, same GPU."""
    import ctypes
    path = os.path.join(ROOT, "oracle", "_ref", "libsheen_ref_gpu.so")
    if not os.path.exists(path):
        return {"value": None, "unavailable": "oracle/_ref/libsheen_ref_gpu.so not built"}
    L = ctypes.CDLL(path)
    L.sheen_refgpu_scene_create.argtypes = [ctypes.c_void_p]
    L.sheen_refgpu_scene_create.restype = ctypes.c_void_p
    L.sheen_refgpu_render.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                      ctypes.c_int, ctypes.POINTER(ctypes.c_float)]
    L.sheen_refgpu_render.restype = ctypes.c_int
    L.sheen_refgpu_scene_destroy.argtypes = [ctypes.c_void_p]
    with quiet_stdout():
        h = L.sheen_refgpu_scene_create(scene.view_ptr)
        if not h:
            return {"value": None, "unavailable": "reference scene upload failed"}
        ms = ctypes.c_float(0.0)
        L.sheen_refgpu_render(h, W, H, SPP, None, 1, ctypes.byref(ms))          # warm-up
        rc = L.sheen_refgpu_render(h, W, H, SPP, None, steps, ctypes.byref(ms))
        L.sheen_refgpu_scene_destroy(h)
    if rc != 0:
        return {"value": None, "unavailable": "reference kernel launch failed"}
    frame_ms = ms.value / steps
    line = {"value": round(rays / (frame_ms / 1e3) / 1e6, 2), "unit": "Mrays/s", "ms_per_frame": round(frame_ms, 2),
            "kernel": "reference render_kernel (render_kernel.cu:438-814) built for sm_100a, 16x16 blocks, "
                      "16 KB stack limit", "rays": "this renderer's count for the frame (same queries)"}
    v = scene.view
    if v.photons > 0 and v.caustics > 0:
        line["note"] = ("the reference kernel printf()s one debug line per caustic gather "
                        "(render_kernel.cu:291-294); timed as shipped")
    return line


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import torch

    import sheen_b200 as sb
    from oracle_bindings import RefHost
    if not RefHost.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libsheen_ref_host.so not built"}))
        return
    if args.config == 4:
        print(json.dumps({"impl": "reference", "unavailable": "the reference has no request loop (one frame per "
                          "sheen_render_scene call, api/sheen_c_api.cu:187-361); its per-frame rate is the mesh "
                          "workload's reference line"}))
        return
    sb.init(int(os.environ.get("LOCAL_RANK", "0")), 100)
    scene = make_scene(args)
    ref = RefHost()
    threads = ref.lib.sheen_ref_max_threads()
    with quiet_stdout():
        h = ref.scene(scene.view_ptr, threads)
    # ray count of the band: this renderer's counters (bookkeeping only; the
    # timed work below is the reference's code alone)
    ds = sb.DeviceScene(scene, sb.FORM_PLAIN)
    out = torch.empty((H, W, 4), dtype=torch.float32, device="cuda")
    rays = band_rays(ds, torch.cuda.current_stream().cuda_stream, out)
    count_check = ray_count_check(ds, scene, torch.cuda.current_stream().cuda_stream, out)
    ds.close()
    by0, by1 = CPU_BAND[0] // 16, CPU_BAND[1] // 16
    with quiet_stdout():
        for _ in range(args.warmup):
            ref.render(h, W, H, SPP, threads, by0, by0 + 1)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            ref.render(h, W, H, SPP, threads, by0, by1)
        dt = time.perf_counter() - t0
    value = rays * args.steps / dt / 1e6
    sample = (f"rows {CPU_BAND[0]}-{CPU_BAND[1]} of the {W}x{H} {SPP} spp frame per step ({rays} rays), "
              f"host-compiled reference render_kernel, {threads} threads")
    print(json.dumps({
        "impl": "reference", "metric": "Mrays/s", "value": round(value, 3), "unit": "Mrays/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(dt / args.steps * 1e3, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded generator)",
        "config": {"workload": WORKLOADS.get(args.config, "") + " (row band sample)",
                   "rays_per_step": rays, "ray_count_check": count_check},
        "cpu_baseline": {"value": round(value, 3), "unit": "Mrays/s", "cores": threads, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": round(value, 3), "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


SERVE_WORKLOAD = ("serving: Poisson request stream at 20/s, each request a scene of the spheres / mesh / "
                  "analytic / caustics generators (4 seeds each, resident on the device), resolution from "
                  "{256^2, 512^2, 1280x720, 1920x1080, 2048^2}, spp from {1, 4, 16, 64}")


def _serving_scene(config, seed):
    import sheen_b200 as sb
    photons = 4000000 if config == 3 else 0
    return sb.generate_scene(config, seed, 8 if config == 1 else 0, photons)


def serve_stream(n_requests, rate, inflight, seed, warmup, serial_k=0, local=0):
    """The request loop under a seeded Poisson stream: requests are submitted
    at their arrival times and the server admits, overlaps and completes
    them; every request's image lands in a host buffer.  Returns value = all
    rays of all requests / (last completion - first arrival) and the
    per-request latencies (arrival -> image in host memory).  With serial_k,
    also the first serial_k requests one at a time through a plain-form
    server and through the wavefront server (what overlap adds)."""
    import sheen_b200 as sb
    from sheen_b200 import serve
    stream = serve.request_stream(n_requests, rate, seed=seed)
    keys = sorted({(r["config"], r["seed"]) for r in stream})
    t0 = time.perf_counter()
    host_scenes = {k: _serving_scene(*k) for k in keys}
    gen_s = time.perf_counter() - t0
    srv = serve.Server(sb.FORM_WAVEFRONT, max_inflight=inflight)
    t0 = time.perf_counter()
    sid = {k: srv.add_scene(host_scenes[k]) for k in keys}
    add_s = time.perf_counter() - t0
    # warm-up: one small request per scene (kernels loaded), then one
    # 1080p 4-spp request per generator (the pool primed to a full row band)
    for k in keys:
        srv.submit(sid[k], 256, 256, 1).wait()
    for cfg in sorted({k[0] for k in keys}):
        srv.submit(sid[next(k for k in keys if k[0] == cfg)], 1920, 1080, 4).wait()
    for _ in range(max(0, warmup - 1)):
        srv.submit(sid[keys[0]], 512, 512, 4).wait()

    reqs = [None] * len(stream)
    infos = [None] * len(stream)

    def collect():
        for i in range(len(stream)):
            while reqs[i] is None:
                time.sleep(0.0005)
            _, infos[i] = reqs[i].wait()
            reqs[i].image = None          # the image was delivered; drop it

    th = threading.Thread(target=collect)
    th.start()
    with ClockSampler(local) as clk:
        t_start = time.perf_counter()
        for i, r in enumerate(stream):
            delay = t_start + r["t"] - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            reqs[i] = srv.submit(sid[(r["config"], r["seed"])], r["width"], r["height"], r["spp"])
        th.join()
        wall_s = time.perf_counter() - t_start
    st = srv.stats()
    rays = sum(i["rays"] for i in infos)
    lat = np.array([i["latency_ms"] for i in infos])
    res = {"stream": stream, "infos": infos, "keys": keys, "wall_s": wall_s, "rays": rays,
           "value": rays / wall_s / 1e6, "lat": lat, "stats": st, "clocks": clk.summary(),
           "gen_s": gen_s, "add_s": add_s}
    if serial_k:
        # serial plain-form baseline on a prefix of the stream
        k = min(serial_k, len(stream))
        psrv = serve.Server(sb.FORM_PLAIN, max_inflight=1)
        pkeys = sorted({(r["config"], r["seed"]) for r in stream[:k]})
        psid = {kk: psrv.add_scene(host_scenes[kk]) for kk in pkeys}
        psrv.submit(psid[pkeys[0]], 256, 256, 1).wait()
        t0 = time.perf_counter()
        prays = 0
        for r in stream[:k]:
            _, info = psrv.submit(psid[(r["config"], r["seed"])], r["width"], r["height"], r["spp"]).wait()
            prays += info["rays"]
        plain_s = time.perf_counter() - t0
        psrv.close()
        # the chosen form serially on the same prefix (what overlap adds)
        t0 = time.perf_counter()
        wrays = 0
        for r in stream[:k]:
            _, info = srv.submit(sid[(r["config"], r["seed"])], r["width"], r["height"], r["spp"]).wait()
            wrays += info["rays"]
        wave_serial_s = time.perf_counter() - t0
        res.update(serial_k=k, prays=prays, plain_s=plain_s, wrays=wrays, wave_serial_s=wave_serial_s)
    srv.close()
    return res


def latency_summary(res):
    lat, infos = res["lat"], res["infos"]
    return {"p50": round(float(np.percentile(lat, 50, method="inverted_cdf")), 2),
            "p99": round(float(np.percentile(lat, 99, method="inverted_cdf")), 2),
            "mean": round(float(lat.mean()), 2), "max": round(float(lat.max()), 2),
            "queue_mean": round(float(np.mean([i["queue_ms"] for i in infos])), 2),
            "run_mean": round(float(np.mean([i["run_ms"] for i in infos])), 2)}


def run_serving(args):
    """The serving workload: the whole seeded stream through the request
    loop, with the serial plain-form and serial wavefront baselines on a
    prefix of it."""
    rank = int(os.environ.get("RANK", "0"))
    import torch

    import sheen_b200 as sb
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    sb.init(local, 100)
    res = serve_stream(args.requests, args.rate, args.inflight, args.seed, args.warmup, args.serial_sample, local)
    if rank != 0:
        return
    st, stream, infos, n = res["stats"], res["stream"], res["infos"], len(res["stream"])
    k = res["serial_k"]
    line = {
        "metric": "Mrays/s (serving)", "value": round(res["value"], 2), "unit": "Mrays/s", "n_gpus": 1,
        "steps": n, "warmup": args.warmup, "ms_per_step": round(res["wall_s"] * 1e3 / n, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded generators, seeded request stream)",
        "config": {"workload": SERVE_WORKLOAD, "requests": n, "rate_per_s": args.rate, "scenes": len(res["keys"]),
                   "max_inflight": args.inflight, "form": "wavefront",
                   "l2": "inputs (2.1M-triangle scenes, 4M-photon maps) exceed L2; no flush between requests",
                   "scene_generate_s": round(res["gen_s"], 2), "scene_add_s": round(res["add_s"], 2),
                   "scene_bytes": st["scene_bytes"], "hbm_budget": st["hbm_budget"],
                   "hbm_peak": st["hbm_peak"], "inflight_peak": st["inflight_peak"]},
        "latency_ms": latency_summary(res),
        "serial_plain": {"value": round(res["prays"] / res["plain_s"] / 1e6, 2), "unit": "Mrays/s",
                         "sample": f"first {k} requests of the stream, one at a time, plain form, "
                                   f"scenes resident ({res['prays']} rays, {res['plain_s']:.1f} s)"},
        "serial_wavefront": {"value": round(res["wrays"] / res["wave_serial_s"] / 1e6, 2), "unit": "Mrays/s",
                             "sample": f"same {k} requests one at a time through the wavefront server"},
        "e2e": {"value": round(res["value"], 2), "unit": "Mrays/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": int(sum(r["width"] * r["height"] * 16 for r in stream) / n),
                "call": "sheen_server_submit / sheen_server_wait, images into host buffers"},
        "gpu_launches": int(sum(i["tiles"] for i in infos) * 8),
        "clocks": res["clocks"],
        "server_stats": {kk: st[kk] for kk in ("completed", "failed", "p50_ms", "p99_ms", "busy_ms")},
    }
    print(json.dumps(line), flush=True)


CAPTURE_CASES = {
    # name: (generator config, detail, photons, width, height, spp, form, small-frame switch on,
    #        extension max_depth or None for no extension)
    "wave": (1, 8, 0, 640, 360, 4, "wavefront", False, None),
    "plain": (1, 8, 0, 640, 360, 4, "plain", False, None),
    "mega": (0, 0, 0, 640, 480, 1, "wavefront", True, None),
    "photon": (3, 0, 1000000, 320, 180, 1, "wavefront", True, None),
    "wave_inst": (1, 8, 0, 640, 360, 4, "wavefront", False, 0),
    "analytic": (2, 0, 0, 640, 360, 4, "wavefront", False, None),
    "mega_deep": (1, 8, 0, 640, 360, 4, "wavefront", True, 4),
}


def run_capture(name):
    """One small frame of a named case, for profiler captures (ncu -k ...):
    wave / plain: the mesh workload at 640x360 4 spp through the queue stages
    or the plain form; mega: the spheres workload at 640x480 1 spp (the
    small-frame megakernel); photon: the caustics workload with 1M photons
    per light (its scene build runs the photon emission); wave_inst: the mesh
    workload with instanced tori at 640x360 4 spp through the queue stages;
    analytic: the analytic + CSG workload at 640x360 4 spp through the queue
    stages;
    mega_deep: the same with reflect + refract recursion to 4 bounces (BVH4
    megakernel)."""
    import torch

    import sheen_b200 as sb
    cfg, detail, photons, w, h, spp, form, mega, depth = CAPTURE_CASES[name]
    sb.init(0, 100)
    if not mega:
        sb.tune_set("wave.mega_samples", 0)
    scene = sb.generate_scene(cfg, 1, detail, photons, extended=depth is not None)
    ext = False
    if depth is not None:
        ext = scene_ext(scene, argparse.Namespace(extended=True, max_depth=depth))
    ds = sb.DeviceScene(scene, sb.FORM_WAVEFRONT if form == "wavefront" else sb.FORM_PLAIN, ext=ext)
    out = torch.empty((h, w, 4), dtype=torch.float32, device="cuda")
    ds.render_device(w, h, spp, out.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    print(json.dumps({"capture": name, "mean": float(out[..., :3].mean())}))
    ds.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--form", default="wavefront", choices=["wavefront", "plain"])
    ap.add_argument("--config", type=int, default=1)
    ap.add_argument("--detail", type=int, default=8)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--photons", type=int, default=0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-ref-gpu", action="store_true")
    ap.add_argument("--width", type=int, default=0, help="override the workload's frame width")
    ap.add_argument("--height", type=int, default=0, help="override the workload's frame height")
    ap.add_argument("--spp", type=int, default=0, help="override the workload's samples per pixel")
    ap.add_argument("--tiles", type=int, default=0,
                    help="render each frame as this many uneven screen tiles in one batched pass (wavefront form)")
    ap.add_argument("--tune", action="append", default=[], metavar="KEY=VALUE",
                    help="launch parameter of the wavefront form (sheen_tune_set), repeatable")
    ap.add_argument("--requests", type=int, default=512, help="serving config: requests in the stream")
    ap.add_argument("--rate", type=float, default=20.0, help="serving config: arrivals per second")
    ap.add_argument("--inflight", type=int, default=4, help="serving config: requests on the GPU at once")
    ap.add_argument("--serial-sample", type=int, default=24, help="serving config: serial baseline prefix")
    ap.add_argument("--serve-requests", type=int, default=64,
                    help="requests of the short serving run in the default bench line (0: skip)")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain-form denominator")
    ap.add_argument("--extended", action="store_true",
                    help="the workload's extension column -- config 1: reflect + refract recursion to 4 "
                         "bounces; config 2: exact Bezier lathes and prisms, two-exponent superellipsoids, "
                         "FP32 height grid, 128 CSG trees; the reference has none of these, so the line "
                         "carries no reference or host-array legs")
    ap.add_argument("--max-depth", type=int, default=-1,
                    help="with --extended: the extension's reflect + refract depth instead of the generator's "
                         "(0: the reference's depth-1 rules)")
    ap.add_argument("--capture", choices=sorted(CAPTURE_CASES),
                    help="render one small frame of a named case and exit (for profiler captures)")
    args = ap.parse_args()
    if args.capture:
        run_capture(args.capture)
        return
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if args.extended:
        if args.config not in (1, 2):
            ap.error("--extended applies to --config 1 and 2")
        args.no_cpu = args.no_ref_gpu = args.no_plain = True
        args.serve_requests = 0
    if args.tune:
        import sheen_b200 as sb
        for kv in args.tune:
            k, v = kv.split("=", 1)
            sb.tune_set(k, int(v))
    if args.impl == "reference":
        run_reference(args)
    elif args.config == 4:
        run_serving(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
