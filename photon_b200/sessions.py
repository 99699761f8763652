"""Real-time SVGF sessions: each session renders an orbit of one resident scene, one path per pixel
per frame, denoised by SVGF (pt_render_denoised), on its own renderer and stream; several sessions
run concurrently from host threads. Reports per-frame latency percentiles and the aggregate rate.

    python -m photon_b200.sessions [--sessions 8] [--frames 120] [--width 1600] [--height 900]
"""
import argparse
import json
import sys
import threading
import time

import numpy as np

from . import abi, native, workloads


def run_sessions(desc, n_sessions=8, frames=120, width=1600, height=900, max_depth=12, device=0, warmup=3, tuning=None):
    """Returns {"sessions", "frames", "p50_ms", "p99_ms", "mean_ms", "frames_per_s", ...}; frame time is
    the wall clock of one pt_render_denoised call (render, G-buffer, SVGF, synchronised). `tuning`:
    pt_set_tuning fields applied to every session's renderer."""
    renderers, cams = [], []
    for k in range(n_sessions):
        r = native.Renderer(device)
        r.upload(desc)
        r.resize(width, height)
        if tuning:
            r.set_tuning(**tuning)
        renderers.append(r)
        cams.append(workloads.orbit_cameras(desc, frames + warmup, width / height, start_deg=45.0 * k))
    rs = abi.render_settings(width, height, max_depth=max_depth, seed=11)
    sv = abi.svgf_settings()
    times = [[] for _ in range(n_sessions)]
    barrier = threading.Barrier(n_sessions + 1)

    def session(k):
        r, cs = renderers[k], cams[k]
        for f in range(warmup):
            r.render_denoised(cs[f], cs[max(f - 1, 0)], rs, sv)
        barrier.wait()
        for f in range(warmup, warmup + frames):
            t0 = time.perf_counter()
            r.render_denoised(cs[f], cs[f - 1], rs, sv)
            times[k].append(time.perf_counter() - t0)

    threads = [threading.Thread(target=session, args=(k,)) for k in range(n_sessions)]
    for t in threads:
        t.start()
    barrier.wait()
    t0 = time.perf_counter()
    for t in threads:
        t.join()
    wall = time.perf_counter() - t0
    for r in renderers:
        r.close()
    ms = np.asarray([t for ts in times for t in ts]) * 1e3
    return {"sessions": n_sessions, "frames": int(ms.size), "width": width, "height": height, "spp": 1,
            "p50_ms": float(np.percentile(ms, 50)), "p99_ms": float(np.percentile(ms, 99)), "mean_ms": float(ms.mean()),
            "frames_per_s": ms.size / wall, "msamples_per_s": ms.size * width * height / wall / 1e6}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--sessions", type=int, default=8)
    ap.add_argument("--frames", type=int, default=120)
    ap.add_argument("--width", type=int, default=1600)
    ap.add_argument("--height", type=int, default=900)
    ap.add_argument("--triangles", type=int, default=262144)
    a = ap.parse_args(argv)
    g = native.terrain_scene(a.triangles, 1)
    b = g.build()
    print(json.dumps(run_sessions(b.desc, a.sessions, a.frames, a.width, a.height)))
    return 0


if __name__ == "__main__":
    sys.exit(main())
