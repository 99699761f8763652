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
    """Submits each request at its arrival time; latency = server-side done time - submit time."""
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
    return _summary(lat, samples, last - first)


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
