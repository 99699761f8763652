"""Benchmark of the wavefront path tracer on the 262,144-triangle scene (1920x1080, 16 spp, max depth 12).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step renders one full frame (1920 x 1080 x 16 = 33,177,600 paths) through pt_render on a scene
already resident in device memory; the metric is Msamples/s (a sample is one whole path). Steps are
timed on the device with CUDA events recorded on the renderer's own stream, one event pair per
step, with a 256 MiB write between steps to flush the 126 MB L2; the JSON line reports the whole
job (all ranks) and max-over-ranks time. Under torchrun each rank renders its own frames (weak
scaling, replicas: no collective on the data path).

Also reported: `e2e` (pt_render + pt_download_image into a host buffer, wall clock per step), the
roofline of the dominant kernel from the library's per-kernel event timing and traversal counters,
clocks sampled with nvidia-smi during the timed region, Photon's megakernel on the same GPU, scene and
frame (`megakernel`), and the reference CPU renderer timed on the host cores on a bounded sample.

`--impl reference` times only Photon's own CPU renderer, through Photon's code alone: the scene is the
generator's raw meshes built by Photon's Scene::build (oracle/_ref, which carries its own copy of the
generator), so that arm loads nothing of this library and walks Photon's tree, while this arm walks
the tree of the library's own builder (the same meshes; different trees, same workload).
"""
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

METRIC = "Msamples/s at 262K tris; p50/p99 request latency, served vs plain, 1 B200"
UNIT = "Msamples/s"
WIDTH, HEIGHT, SPP, DEPTH, TRIS, SEED = 1920, 1080, 16, 12, 262144, 1
WORKLOAD = "262,144-triangle terrain scene (value-noise height field + 200 instanced shapes, 64 materials, " \
           "64 emitters, 4 punctual lights, 1024x512 HDR sky), 1920x1080, 16 spp, max depth 12, seed 1"
# Algorithmic bytes of the traversal kernels: one 64-byte node per visit, one 48-byte triangle per test.
NODE_BYTES, TRI_BYTES = 64, 48
# Modelled bytes of one shaded vertex in k_shade (path state in and out, hit, shadow entry, triangle,
# indices, vertex attributes, material).
SHADE_BYTES_PER_VERTEX = 450
# DRAM bytes (read + write) per traced ray of the closest-hit walk: its first launch in the 960x540x4
# profile case of the same scene (photon_b200/profile_case.py; 2,073,600 camera rays, 75.03 MB read +
# 11.30 MB written in one ncu capture), scaled by the rays of a launch here: mostly the path state
# streaming in and the hits out; the nodes and triangles stay in L2.
TRACE_DRAM_BYTES_PER_RAY = (75.03e6 + 11.30e6) / 2073600
# Active threads per warp instruction (smsp__thread_inst_executed_per_inst_executed) of the pair walks
# in the same capture (ncu --set full on python -m photon_b200.profile_case): the camera rays' launch,
# then the first two bounces. The per-lane walks it replaced ran at 11.9 / 8.1 / 7.0 (closest hit) and
# 7.7 / 6.1 / 5.8 (any hit) on the same case.
NCU_THREADS_PER_INSTRUCTION = {"trace": [18.2, 15.4, 14.1], "shadow": [15.0, 13.0, 12.5], "of": 32,
                               "per_lane_walks": {"trace": [11.9, 8.1, 7.0], "shadow": [7.7, 6.1, 5.8]}}
# Workload description shared by both arms (the reference arm renders a bounded sample of it).
CONFIG = {"workload": WORKLOAD, "scene_triangles": TRIS, "width": WIDTH, "height": HEIGHT, "spp": SPP, "max_depth": DEPTH,
          "samples_per_step": WIDTH * HEIGHT * SPP,
          "l2": "GPU arm: 256 MiB device write between steps, outside the event pair (the CPU arm has no device L2)"}


def dist_info():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def init_dist(world, local, backend="nccl"):
    """One process per GPU (torchrun's env). NCCL carries only the barrier and the max-over-ranks
    time; the data path has no collective. `backend="gloo"` runs the same host logic on CPU."""
    if world <= 1:
        return None
    import datetime
    import torch
    import torch.distributed as dist
    if backend == "nccl":
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))
    else:
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=60))
    return dist


def reduce_max(dist, value, local):
    if dist is None:
        return value
    import torch
    device = f"cuda:{local}" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world, steps, units_per_step, max_seconds):
    """Millions of units per second for the whole job: every rank processes `steps` x
    `units_per_step` (weak scaling), and the job takes the slowest rank's time."""
    return world * steps * units_per_step / max_seconds / 1e6


def barrier(dist):
    if dist is not None:
        dist.barrier()


class ClockSampler:
    """nvidia-smi samples (every 100 ms) of SM clock and throttle reasons during the timed region; start()
    returns once the first sample is in (nvidia-smi takes a moment to come up), so the samples cover the
    region from its start."""

    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
            return
        deadline = time.time() + 5.0
        while not self.lines and self.proc.poll() is None and time.time() < deadline:
            time.sleep(0.01)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(mx), "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            j = json.load(f)
        return float(j["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def cpu_baseline(desc, cam, seconds_hint=20.0):
    """Photon's own CpuRenderer (oracle/_ref, built from its sources) on all host cores, on a bounded
    sample: 1 spp of the full 1920x1080 frame after a 1 spp warm-up at 480x270."""
    from oracle import oracle as O
    from photon_b200 import abi
    if not O.reference_available():
        return None
    ref = O.RefScene.from_desc(desc)
    cores = os.cpu_count() or 1
    warm = abi.render_settings(480, 270, max_depth=DEPTH, seed=SEED)
    ref.render(cam, warm, 1, threads=cores)
    rs = abi.render_settings(WIDTH, HEIGHT, max_depth=DEPTH, seed=SEED)
    _, secs = ref.render(cam, rs, 1, threads=cores)
    return {"value": WIDTH * HEIGHT / secs / 1e6, "unit": UNIT, "cores": cores, "kind": "reference",
            "sample": f"1 spp of the 1920x1080 frame ({WIDTH * HEIGHT} paths, {secs:.2f} s) after a 1 spp 480x270 warm-up"}


def run_reference(args, world, rank):
    """The reference arm: Photon's own CPU renderer (CpuRenderer::render, cpu_renderer.cpp:20-39) on all
    host cores, rank 0 only, through Photon's code alone. The scene is the generator's raw meshes built
    by Photon's Scene::build (scene.cpp:212-255, bvh.cpp:152-258) and the camera Photon's Camera::view of
    the generator's camera; each step renders 1 spp of the full 1920x1080 frame, reported as a rate as
    `photon bench` does (render_cli.cpp:319-327)."""
    if rank != 0:
        return 0
    from oracle import oracle as O
    from photon_b200 import abi  # ctypes structures only: loads no library
    if not O.reference_available():
        print(json.dumps({"impl": "reference", "unavailable": "Photon's CPU build (oracle/_ref/libphoton_ref.so) is missing"}))
        return 0
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    ref = O.RefScene.generated(abi.PT_GEN_TERRAIN, TRIS, SEED, threads=cores)
    build_s = time.perf_counter() - t0
    cam = ref.camera(WIDTH / HEIGHT)
    rs = abi.render_settings(WIDTH, HEIGHT, max_depth=DEPTH, seed=SEED)
    for _ in range(args.warmup):
        ref.render(cam, rs, 1, threads=cores)
    t = []
    for _ in range(args.steps):
        _, secs = ref.render(cam, rs, 1, threads=cores)
        t.append(secs)
    total = sum(t)
    value = args.steps * WIDTH * HEIGHT / total / 1e6
    sample = f"1 spp of the 1920x1080 frame per step ({WIDTH * HEIGHT} paths), all {cores} host threads"
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000 * total / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (procedural scene, seeded)", "config": dict(CONFIG),
            "parallelism": f"{cores} host threads",
            "scene_build": {"builder": "Photon's Scene::build of the generator's raw meshes", "seconds": build_s,
                            "nodes": ref.desc.num_nodes, "triangles": ref.desc.num_tris},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def megakernel(desc, cam, steps):
    """Photon's megakernel (gpu_renderer.cu's render_kernel, built for sm_100a with Photon's flags into
    oracle/_ref/libphoton_ref_gpu.so) on the same GPU, scene and frame, the way `photon bench` runs it
    (render_cli.cpp:329-341): a 4-spp warm-up, then the frame's 16 spp as 8-spp launches. Device time
    is GpuRenderer::last_frame_ms (CUDA events around each launch); wall time is also given."""
    import ctypes as C
    from oracle import oracle as O
    from photon_b200 import abi
    if not os.path.exists(O.REF_GPU_SO):
        return {"unavailable": "Photon's CUDA build (oracle/_ref/libphoton_ref_gpu.so) is missing"}
    L = O.reference_gpu()
    if not L.refgpu_available():
        return {"unavailable": "Photon's cuda_available() is false"}
    ref_scene = O.RefScene.from_desc(desc, lib=L)
    rs = abi.render_settings(WIDTH, HEIGHT, max_depth=DEPTH, seed=SEED)
    g = L.refgpu_create()
    try:
        if not L.refgpu_upload(g, ref_scene.h):
            return {"unavailable": "GpuRenderer::upload failed"}
        L.refgpu_resize(g, WIDTH, HEIGHT)
        L.refgpu_render(g, C.byref(cam), C.byref(rs), 4)
        dev_ms, wall = 0.0, 0.0
        for _ in range(steps):
            L.refgpu_reset(g)
            t0 = time.perf_counter()
            for done in range(0, SPP, 8):
                dev_ms += L.refgpu_render(g, C.byref(cam), C.byref(rs), min(8, SPP - done))
            wall += time.perf_counter() - t0
    finally:
        L.refgpu_destroy(g)
    samples = steps * WIDTH * HEIGHT * SPP
    return {"msamples_per_s": samples / (dev_ms / 1000.0) / 1e6, "wall_msamples_per_s": samples / wall / 1e6,
            "ms_per_frame": dev_ms / steps, "frames": steps,
            "method": "GpuRenderer on the same resident scene: 4-spp warm-up, then 8-spp launches (photon bench)"}


SERVED_RATE, SERVED_REQUESTS = 500.0, 1000


def systems_sections(r, g, desc, rank):
    """The batched and served forms on the same 262K scene (extra keys of the JSON line):
    - batched: 64 seeded views (320x180..1920x1080, spp {1,4,16,64}, cameras on a sphere of radius
      1.5x the scene extent) in one pt_render_views call (median of three), against the same views
      rendered one pt_render call at a time;
    - served: the serving configuration's Poisson stream (seed 7) over four resident scenes of 36,
      262,144, 1,048,576 and 4,194,304 triangles under a 150 GB budget, resolution / spp / depth drawn
      as the configuration says, at a saturating 500 req/s (1,000 requests: the offered work exceeds
      what the GPU renders, so the throughput is the server's, not the offered load), through the
      server against the same stream rendered one request at a time in arrival order; p50/p99 latency
      from submission to result;
    - sessions: eight real-time SVGF sessions (1600x900, 1 spp per frame, 120-frame orbits) on host
      threads; p50/p99 frame time."""
    from photon_b200 import abi, native, serving, workloads
    out = {}
    views = workloads.batch_views(desc, 64, seed=2)
    total = sum(v.width * v.height * v.spp for v in views)

    def time_batch():  # median of three pt_render_views calls after a warm-up call
        r.render_views(views)
        ts = []
        for _ in range(3):
            t0 = time.perf_counter()
            r.render_views(views)
            ts.append(time.perf_counter() - t0)
        return sorted(ts)[1]

    tb = time_batch()
    t0 = time.perf_counter()
    for v in views:
        r.resize(v.width, v.height)
        r.reset()
        r.render(v.camera, abi.RenderSettings(v.width, v.height, v.path, 1.0, abi.PT_TONEMAP_ACES, v.seed), v.spp)
    tp = time.perf_counter() - t0
    # The autotuner on the view set (a copy scaled to 2^25 paths), then the same batch with its choice.
    default_tuning = r.tuning()
    t0 = time.perf_counter()
    chosen, probe_default, probe_tuned = r.autotune_views(views, probe_samples=1 << 25)
    tune_s = time.perf_counter() - t0
    tt = time_batch()
    r.set_tuning(**default_tuning)
    out["batched"] = {"workload": "64 views of the 262K scene (seed 2)", "samples": total, "msamples_per_s": total / tb / 1e6,
                      "plain_msamples_per_s": total / tp / 1e6, "batched_over_plain": tp / tb, "api": "pt_render_views",
                      "tuned": {"msamples_per_s": total / tt / 1e6, "tuned_over_default": tb / tt, "autotune_seconds": tune_s,
                                "probe_msamples_per_s": {"default": probe_default / 1e6, "tuned": probe_tuned / 1e6},
                                "chosen": chosen, "api": "pt_autotune_views"}}
    # The four resident scenes of the serving configuration (the larger two built on the device).
    scenes = [(native.box_scene(), None), (g, None), (native.terrain_scene(1 << 20, SEED), None), (native.terrain_scene(1 << 22, SEED), None)]
    built = []
    for k, (gs, _) in enumerate(scenes):
        built.append(gs.build(gpu=k >= 2) if k != 1 else None)
    descs = [built[0].desc, desc, built[2].desc, built[3].desc]
    budget = 150 << 30
    server = native.Server(budget_bytes=budget, device=r_device(r))
    sids = [server.add_scene(d) for d in descs]
    pairs = list(zip(sids, descs))
    stream = workloads.request_stream(pairs, SERVED_REQUESTS, SERVED_RATE, seed=7)
    # Warm-up for both forms: a burst of 64 requests of another stream (first-time memory pinning
    # and pool growth stay out of the measurement).
    warm = [dict(x, t=0.0) for x in workloads.request_stream(pairs, 64, SERVED_RATE, seed=8)]
    serving.run_served(server, warm)
    served = serving.run_served(server, stream)
    server.close()
    plain_r = {}
    for sid, d in pairs:
        if d is desc:
            plain_r[sid] = r
        else:
            rr = native.Renderer(r_device(r))
            rr.upload(d)
            plain_r[sid] = rr
    serving.run_plain(plain_r, warm)
    plain = serving.run_plain(plain_r, stream)
    for rr in plain_r.values():
        if rr is not r:
            rr.close()
    out["served"] = {"workload": f"Poisson, {SERVED_REQUESTS} requests at {SERVED_RATE:g} req/s (saturating), seed 7, "
                                 "scenes of 36 / 262,144 / 1,048,576 / 4,194,304 triangles, 150 GB budget",
                     "served": served, "plain": plain, "budget_bytes": budget,
                     "served_over_plain": served["msamples_per_s"] / plain["msamples_per_s"]}
    # Eight real-time SVGF sessions served by the same server alongside the same stream (the server's
    # session lane), and the same sessions on renderers of their own.
    server = native.Server(budget_bytes=budget, device=r_device(r))
    sids = [server.add_scene(d) for d in descs]
    serving.run_served(server, warm)
    both = serving.run_sessions_served(server, sids[1], desc, 8, 120, 1600, 900,
                                       stream=workloads.request_stream(list(zip(sids, descs)), SERVED_REQUESTS, SERVED_RATE, seed=7))
    server.close()
    from photon_b200 import sessions
    out["sessions"] = dict(both, workload="8 real-time SVGF sessions (120-frame orbits, 0.5 deg/frame, of the 262K scene, 1600x900, "
                                          "1 spp) served by the request server alongside the served stream above",
                           api="pt_server_open_session / pt_server_submit_frame",
                           standalone=dict(sessions.run_sessions(desc, 8, 120, 1600, 900, device=r_device(r)), api="pt_render_denoised, one renderer per session"))
    return out


def r_device(r):
    import torch
    return torch.cuda.current_device()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-systems", action="store_true", help="skip the batched-views and served-stream sections")
    ap.add_argument("--no-megakernel", action="store_true", help="skip the megakernel comparison")
    args = ap.parse_args()
    world, rank, local = dist_info()
    if args.impl == "reference":
        return run_reference(args, world, rank)
    if args.warmup < 3:
        args.warmup = 3

    import torch
    from photon_b200 import abi, native

    dist = init_dist(world, local)
    torch.cuda.set_device(local)
    g = native.terrain_scene(TRIS, SEED)
    b = g.build()
    desc = b.desc
    cam = g.camera(WIDTH / HEIGHT)
    rs = abi.render_settings(WIDTH, HEIGHT, max_depth=DEPTH, seed=SEED + rank)
    r = native.Renderer(local)
    r.upload(desc)
    r.resize(WIDTH, HEIGHT)
    stream = torch.cuda.ExternalStream(r.stream(), device=f"cuda:{local}")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")

    # Warm-up, then one untimed render with traversal counters (the roofline's algorithmic bytes).
    for _ in range(args.warmup):
        r.render(cam, rs, SPP)
        r.reset()
    r.set_profiling(abi.PT_PROFILE_TRAVERSAL_COUNTS)
    r.render(cam, rs, SPP)
    r.reset()
    counts = r.profile()

    # Timed steps.
    r.set_profiling(abi.PT_PROFILE_KERNEL_TIMES)
    clocks = ClockSampler(local)
    barrier(dist)
    torch.cuda.synchronize()
    clocks.start()
    step_ms = []
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(1)
            start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            start.record(stream)
        r.render(cam, rs, SPP)
        end.record(stream)
        end.synchronize()
        step_ms.append(start.elapsed_time(end))
        r.reset()
    torch.cuda.synchronize()
    clock_info = clocks.stop()
    barrier(dist)
    prof = r.profile()
    total_ms = reduce_max(dist, float(sum(step_ms)), local)
    samples_per_step = WIDTH * HEIGHT * SPP
    value = whole_job_rate(world, args.steps, samples_per_step, total_ms / 1000.0)

    # End to end through the C ABI: render + download into a page-locked host buffer (the download
    # copies straight into it), wall clock (no profiling). One untimed step first: switching profiling
    # off re-captures the iteration graphs.
    r.set_profiling(0)
    e2e_t = []
    host = torch.empty((HEIGHT, WIDTH, 3), dtype=torch.float32, pin_memory=True).numpy()
    r.reset()
    r.render(cam, rs, SPP)
    r.download_image(out=host)
    for _ in range(args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r.reset()
        r.render(cam, rs, SPP)
        r.download_image(out=host)
        e2e_t.append(time.perf_counter() - t0)
    e2e_total = reduce_max(dist, float(sum(e2e_t)), local)
    e2e_value = whole_job_rate(world, args.steps, samples_per_step, e2e_total)

    # Roofline of the dominant kernel.
    kernels = {"setup": prof.setup.ms, "generate": prof.generate.ms, "trace": prof.trace.ms, "shade": prof.shade.ms,
               "shadow": prof.shadow.ms, "accumulate": prof.accumulate.ms}
    ktotal = sum(kernels.values()) or 1.0
    trace_bytes_per_frame = counts.closest_node_visits * NODE_BYTES + counts.closest_tri_tests * TRI_BYTES
    shadow_bytes_per_frame = counts.shadow_node_visits * NODE_BYTES + counts.shadow_tri_tests * TRI_BYTES
    peak, peak_kind = measured_peak()
    trace_launches = max(1, prof.trace.launches)
    achieved = (trace_bytes_per_frame * args.steps) / (prof.trace.ms / 1000.0) / 1e9 if prof.trace.ms > 0 else 0.0
    shadow_achieved = (shadow_bytes_per_frame * args.steps) / (prof.shadow.ms / 1000.0) / 1e9 if prof.shadow.ms > 0 else 0.0
    # Every traced closest-hit ray of a queued iteration is one shaded vertex (the tail's are counted in
    # closest_rays too, so this slightly overstates the shade kernel's share of them).
    shaded_vertices = counts.closest_rays
    shade_achieved = (shaded_vertices * SHADE_BYTES_PER_VERTEX * args.steps) / (prof.shade.ms / 1000.0) / 1e9 if prof.shade.ms > 0 else 0.0
    # The scene (nodes, triangles) stays in the 126 MB L2 during a frame, so the walk's bytes are L2
    # (and L1) traffic: the live L2 read probe is the bandwidth they are bounded by. The HBM fraction
    # is kept beside it because the copy bandwidth is the measured peak of the schema.
    l2_peak = native.l2_read_bandwidth(local)
    closest_rays_frame = counts.closest_rays  # the counted render is one frame
    pairs = r.tuning()["pair_walk"] > 0
    roofline = {"bound": "hbm", "limiter": "L2/L1 latency and issue: the scene is L2-resident (see l2, simt)",
                "kernel": "k_trace_pairs (closest-hit BVH traversal, pair walk)" if pairs else "k_trace (closest-hit BVH traversal)",
                "l2": {"achieved": achieved, "peak": l2_peak, "unit": "GB/s", "frac": achieved / l2_peak if l2_peak > 0 else None,
                       "peak_source": "live pt_measure_l2_bandwidth: 32 MiB L2-resident buffer read 64 times per launch "
                                      "(ld.global.cg), best of 5"},
                "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_source": f"{peak_kind} hbm_gbs (MEASURED_PEAKS.json)",
                "traffic": TRACE_DRAM_BYTES_PER_RAY * closest_rays_frame * args.steps / trace_launches,
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per traced ray of k_trace on the "
                                  "960x540x4 profile case, times this frame's rays per launch",
                "algorithmic_bytes_per_launch": trace_bytes_per_frame * args.steps / trace_launches,
                "avg_launch_ms": prof.trace.ms / trace_launches,
                "model": "64 B per node visit + 48 B per triangle test (closest-hit rays)",
                "node_visits_per_ray": counts.closest_node_visits / max(1, counts.closest_rays),
                "tri_tests_per_ray": counts.closest_tri_tests / max(1, counts.closest_rays),
                # SIMT use of the two walks: from the counted render, the lanes that visit a node per
                # node-visit round of a pair walk (per walk step of a per-lane walk), of 32; from the
                # profile capture, the active threads per warp instruction.
                "simt": {"trace_lanes_per_round" if pairs else "trace_lanes_per_step": counts.closest_lane_steps / max(1, counts.closest_warp_steps),
                         "shadow_lanes_per_round" if pairs else "shadow_lanes_per_step": counts.shadow_lane_steps / max(1, counts.shadow_warp_steps),
                         "of": 32, "ncu_threads_per_instruction": NCU_THREADS_PER_INSTRUCTION},
                "shadow": {"kernel": "k_shadow_pairs (any-hit BVH traversal, pair walk)" if pairs else "k_shadow (any-hit BVH traversal)",
                           "bytes_per_frame": shadow_bytes_per_frame,
                           "ms_per_frame": prof.shadow.ms / args.steps, "achieved": shadow_achieved,
                           "l2_frac": shadow_achieved / l2_peak if l2_peak > 0 else None, "hbm_frac": shadow_achieved / peak},
                "shade": {"kernel": "k_shade (material-sorted shading of the traced paths)",
                          "model": f"{SHADE_BYTES_PER_VERTEX} B per shaded vertex: path state 80 B in and out, hit 16 B, "
                                   "shadow entry 48 B, triangle record, vertex indices, three vertices' attributes and "
                                   "the material (a model, not a count)",
                          "vertices_per_frame": shaded_vertices,
                          "ms_per_frame": prof.shade.ms / args.steps, "achieved": shade_achieved,
                          "hbm_frac": shade_achieved / peak,
                          "limiter": "latency: attribute, material and texture gathers at 16 warps per SM (114 registers)"}}
    rays_per_sample = (counts.closest_rays + counts.shadow_rays) / samples_per_step

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (procedural scene, seeded; no dataset)",
            "config": dict(CONFIG), "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 64 + 36 + 256,
                    "d2h_bytes_per_step": WIDTH * HEIGHT * 12, "api": "pt_reset + pt_render + pt_download_image",
                    "host_buffer": "page-locked (torch pin_memory), reused"},
            "gpu_launches": prof.kernel_launches,
            "rays_per_sample": rays_per_sample,
            "mrays_per_s": value * rays_per_sample,
            "kernel_ms_per_step": {k: v / args.steps for k, v in kernels.items()},
            "kernel_share": {k: v / ktotal for k, v in kernels.items()},
            "roofline": roofline,
            "clocks": clock_info}
    if rank == 0 and world == 1 and not args.no_megakernel:
        mk = megakernel(desc, cam, 3)
        if "msamples_per_s" in mk:
            mk["wavefront_over_megakernel"] = value / mk["msamples_per_s"]
            mk["wavefront_e2e_over_megakernel"] = e2e_value / mk["msamples_per_s"]
        line["megakernel"] = mk
    if world == 1 and not args.no_systems:
        # The batched, served and session forms are single-GPU forms; a replica run reports the frame.
        line.update(systems_sections(r, g, desc, rank))
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(desc, cam)
    if rank == 0:
        print(json.dumps(line))
    del stream
    r.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
