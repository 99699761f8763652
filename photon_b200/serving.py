"""Drives a request stream through the server (continuous batching) or through plain renderers
(one request at a time, in arrival order) and reports latency percentiles and throughput."""
import threading
import time

import numpy as np

from . import abi, native


def _summary(lat, samples, makespan):
    lat = np.asarray(lat, np.float64)
    return {"requests": int(lat.size), "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "max_s": float(lat.max()), "msamples_per_s": samples / makespan / 1e6,
            "makespan_s": makespan, "samples": int(samples)}


def run_served(server, stream, timeout_s=600.0):
    """Submits each request at its arrival time; latency = server-side done time - submit time. Also
    reports the device time of the server's bounce-iteration batches over the run (busy fraction of its
    stream) and the batches and iterations it launched."""
    st0 = server.stats()
    ids = [None] * len(stream)
    t0 = time.perf_counter()

    def submitter():
        for k, r in enumerate(stream):
            delay = r["t"] - (time.perf_counter() - t0)
            if delay > 0:
                time.sleep(delay)
            ids[k] = server.submit(r["scene"], r["cam"], r["w"], r["h"], r["spp"], r["seed"], r["path"])

    th = threading.Thread(target=submitter)
    th.start()
    lat, samples, first, last = [], 0, None, None
    for k, r in enumerate(stream):
        while ids[k] is None:
            time.sleep(0.0005)
        server.wait(ids[k], timeout_s)
        _, st = server.fetch(ids[k], r["w"], r["h"])
        lat.append(st.done_s - st.submit_s)
        samples += st.samples
        first = st.submit_s if first is None else min(first, st.submit_s)
        last = st.done_s if last is None else max(last, st.done_s)
    th.join()
    st1 = server.stats()
    out = _summary(lat, samples, last - first)
    out.update(device_busy=(st1.device_seconds - st0.device_seconds) / max(last - first, 1e-9), batches=st1.batches - st0.batches,
               iterations=st1.bounce_iterations - st0.bounce_iterations)
    return out


def run_sessions_served(server, scene_id, desc, n_sessions=8, frames=120, width=1600, height=900, max_depth=12, warmup=3,
                        stream=None):
    """Real-time SVGF sessions served by `server`'s session lane (pt_server_open_session): each session,
    on its own host thread, submits the frames of an orbit of the scene one after the other (frame
    k + 1 once frame k has been fetched). With `stream`, that request stream is served at the same time
    (run_served) and its summary returned beside the sessions'. Frame latency = server-side done time -
    submit time."""
    from . import workloads
    rs = abi.render_settings(width, height, max_depth=max_depth, seed=11)
    sv = abi.svgf_settings()
    sessions = [server.open_session(scene_id, width, height, sv) for _ in range(n_sessions)]
    cams = [workloads.orbit_cameras(desc, frames + warmup, width / height, start_deg=45.0 * k) for k in range(n_sessions)]
    lat = [[] for _ in range(n_sessions)]
    barrier = threading.Barrier(n_sessions + 1)

    def frame(k, f):
        rid = server.submit_frame(sessions[k], cams[k][f], cams[k][max(f - 1, 0)], rs)
        server.wait(rid, 600.0)
        _, st = server.fetch(rid, width, height)
        return st.done_s - st.submit_s

    def session(k):
        for f in range(warmup):
            frame(k, f)
        barrier.wait()
        for f in range(warmup, warmup + frames):
            lat[k].append(frame(k, f))

    threads = [threading.Thread(target=session, args=(k,)) for k in range(n_sessions)]
    for t in threads:
        t.start()
    barrier.wait()
    t0 = time.perf_counter()
    served = run_served(server, stream) if stream else None
    for t in threads:
        t.join()
    wall = time.perf_counter() - t0
    for sid in sessions:
        server.close_session(sid)
    ms = np.asarray([t for ts in lat for t in ts]) * 1e3
    out = {"sessions": n_sessions, "frames": int(ms.size), "width": width, "height": height, "spp": 1,
           "p50_ms": float(np.percentile(ms, 50)), "p99_ms": float(np.percentile(ms, 99)), "mean_ms": float(ms.mean()),
           "frames_per_s": ms.size / wall, "msamples_per_s": ms.size * width * height / wall / 1e6}
    if served is not None:
        out["stream"] = served
    return out


def run_plain(renderers, stream):
    """renderers: {scene id: native.Renderer with the scene uploaded}. Requests run one at a time in
    arrival order; latency = completion - arrival (queueing included)."""
    t0 = time.perf_counter()
    lat, samples = [], 0
    for r in stream:
        now = time.perf_counter() - t0
        if r["t"] > now:
            time.sleep(r["t"] - now)
        ren = renderers[r["scene"]]
        ren.resize(r["w"], r["h"])
        ren.reset()
        rs = abi.RenderSettings(r["w"], r["h"], r["path"], 1.0, abi.PT_TONEMAP_ACES, r["seed"])
        ren.render(r["cam"], rs, r["spp"])
        ren.download_image()
        done = time.perf_counter() - t0
        lat.append(done - r["t"])
        samples += r["w"] * r["h"] * r["spp"]
    makespan = (time.perf_counter() - t0) - stream[0]["t"]
    return _summary(lat, samples, makespan)


SWEEP_TRIANGLES = (36, 262144, 1048576, 4194304)


def sweep(rates=(10, 50, 100, 200, 500), max_requests=10000, max_seconds=60.0, budget_gb=150, seed=7, device=0, plain=True, out=None):
    """The serving configuration: a Poisson request stream over four resident scenes (the 36-triangle
    box and terrain scenes of 262,144, 1,048,576 and 4,194,304 triangles), one run per rate with
    min(max_requests, rate x max_seconds) requests, through the server and (optionally) through plain
    renderers one request at a time. Yields one dict per rate; both forms first take a warm-up burst of
    64 requests of another stream."""
    import json
    from . import workloads
    scenes = []
    for n in SWEEP_TRIANGLES:
        g = native.box_scene() if n == 36 else native.terrain_scene(n, 1)
        scenes.append((g, g.build()))
    server = native.Server(budget_bytes=int(budget_gb) << 30, device=device)
    ids = [server.add_scene(b.desc) for _, b in scenes]
    plain_r = {}
    if plain:
        for sid, (_, b) in zip(ids, scenes):
            r = native.Renderer(device)
            r.upload(b.desc)
            plain_r[sid] = r
    pairs = [(sid, b.desc) for sid, (_, b) in zip(ids, scenes)]
    warm = [dict(x, t=0.0) for x in workloads.request_stream(pairs, 64, 100.0, seed=seed + 1000)]
    run_served(server, warm)
    if plain:
        run_plain(plain_r, warm)
    for rate in rates:
        n = int(min(max_requests, rate * max_seconds))
        stream = workloads.request_stream(pairs, n, float(rate), seed=seed)
        rec = {"rate_per_s": rate, "requests": n, "served": run_served(server, stream)}
        if plain:
            rec["plain"] = run_plain(plain_r, stream)
        if out:
            print(json.dumps(rec), file=out, flush=True)
        yield rec
    server.close()
    for r in plain_r.values():
        r.close()


def main(argv=None):
    import argparse
    import sys
    ap = argparse.ArgumentParser(description="Serving sweep: Poisson streams over four resident scenes, served vs plain.")
    ap.add_argument("--rates", default="10,50,100,200,500")
    ap.add_argument("--max-requests", type=int, default=10000)
    ap.add_argument("--max-seconds", type=float, default=60.0)
    ap.add_argument("--no-plain", action="store_true")
    a = ap.parse_args(argv)
    rates = [float(x) for x in a.rates.split(",")]
    for _ in sweep(rates, a.max_requests, a.max_seconds, plain=not a.no_plain, out=sys.stdout):
        pass
    return 0


if __name__ == "__main__":
    import sys
    sys.exit(main())
