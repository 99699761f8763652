"""A small, self-contained render for profilers (ncu): the 262,144-triangle terrain scene at a reduced
resolution, launched without CUDA graphs so every kernel is an ordinary launch.

    python -m photon_b200.profile_case [--width 960] [--height 540] [--spp 4] [--triangles 262144]
    python -m photon_b200.profile_case --denoise 3 --width 1600 --height 900   # real-time SVGF frames

At 960x540x4 the device holds ~0.6 GB (scene 21 MB, path pool, radiance buffer), well inside an
ncu capture's budget, and the path state (> 126 MB) still exceeds L2.
"""
import argparse
import sys

from . import abi, native


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--width", type=int, default=960)
    ap.add_argument("--height", type=int, default=540)
    ap.add_argument("--spp", type=int, default=4)
    ap.add_argument("--triangles", type=int, default=262144)
    ap.add_argument("--depth", type=int, default=12)
    ap.add_argument("--denoise", type=int, default=0, help="render this many real-time SVGF frames instead")
    ap.add_argument("--tuning", action="append", default=[], metavar="KNOB=VALUE",
                    help="a pt_tuning knob for the render (repeatable), e.g. --tuning pair_walk=6")
    a = ap.parse_args(argv)
    g = native.terrain_scene(a.triangles, 1)
    b = g.build()
    cam = g.camera(a.width / a.height)
    rs = abi.render_settings(a.width, a.height, max_depth=a.depth, seed=1)
    r = native.Renderer(0)
    r.upload(b.desc)
    r.resize(a.width, a.height)
    r.set_tuning(graph_bounces=0, **{k: int(v) for k, v in (t.split("=", 1) for t in a.tuning)})
    if a.denoise:
        from . import workloads
        cams = workloads.orbit_cameras(b.desc, a.denoise, a.width / a.height)
        for f in range(a.denoise):
            r.render_denoised(cams[f], cams[max(f - 1, 0)], rs, abi.svgf_settings())
        st = r.stats()
        print(f"rendered {a.denoise} denoised {a.width}x{a.height} frames, last {st.last_frame_ms:.2f} ms")
        r.close()
        return 0
    r.render(cam, rs, a.spp)
    st = r.stats()
    print(f"rendered {a.width}x{a.height}x{a.spp}: {st.bounce_iterations} iterations, {st.rays} rays, {st.last_frame_ms:.2f} ms")
    r.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
