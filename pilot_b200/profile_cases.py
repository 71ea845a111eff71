"""Fixed small cases for profiling one kernel at a time (ncu -k <kernel>).

    python -m pilot_b200.profile_cases --case light_march      # K1, 512^3 noise, M = 256
    python -m pilot_b200.profile_cases --case view_march       # K2, 512^3 noise, 1024^2, map cached
    python -m pilot_b200.profile_cases --case mlp_view         # learned-form view march, 1024^2
    python -m pilot_b200.profile_cases --case mlp_frame        # learned form frame: scene-light network, 1% probes
    python -m pilot_b200.profile_cases --case mlp_tc           # tcgen05 forward, 2^21 rows
    python -m pilot_b200.profile_cases --case batch            # 16-request persistent batch
    python -m pilot_b200.profile_cases --case precision_light  # precision-form K1, bf16 640^3
    python -m pilot_b200.profile_cases --case precision_view   # precision-form K2, bf16 640^3, 1024^2, map cached
    python -m pilot_b200.profile_cases --case bricks           # 512^3 noise as 2x2x2 bricks: K1, K5, K2, K6

Each case sets up its scene, runs the target kernel --reps times and exits 0;
device memory stays within a few GB. The tuning is fixed (8^3 vertex bricks,
skipping as stated per case) so that the launch sequence is the same every run.
"""
from __future__ import annotations

import argparse
import sys


def main(argv=None) -> int:
    import numpy as np
    import torch

    from . import beams as B
    from . import scenes

    ap = argparse.ArgumentParser()
    ap.add_argument("--case", required=True,
                    choices=["light_march", "view_march", "mlp_view", "mlp_frame", "mlp_tc", "batch",
                             "precision_light", "precision_view", "bricks"])
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--split", action="store_true", help="batch: map-build launch, then view launch")
    a = ap.parse_args(argv)
    torch.cuda.set_device(0)
    if a.case in ("light_march", "view_march", "mlp_view", "mlp_frame"):
        s = scenes.config1()
        fd = s.field_device()
        r = B.Renderer(0)
        r.set_volume(fd, origin=s.origin, spacing=s.spacing, value_range=s.value_range)
        s.configure(r)
        r.set_tuning(light_brick=8, empty_skip=False, view_skip=False)
        cam = s.camera()
        out = torch.empty((s.height, s.width, 4), device="cuda")
        if a.case == "light_march":
            for _ in range(a.reps):
                r.build_shadow_map(timings=False)
        elif a.case == "view_march":
            r.build_shadow_map(timings=False)
            r.set_reuse_shadow_map(True)
            for _ in range(a.reps):
                r.render(cam, out=out, timings=False)
        elif a.case == "mlp_frame":
            # the learned form as benchmarked: network trained for the scene's light, knot 32, 1% probes
            r.mlp_train(B.mlp_options(n_lights=1, scene_light=1))
            r.set_form(B.FORM_MLP, B.mlp_options(knot=32, probe_fraction=0.01))
            for _ in range(a.reps):
                r.render(cam, out=out, timings=False)
        else:
            r.mlp_train(B.mlp_options(samples_log2=18, epochs=1, batch=16384))
            r.set_form(B.FORM_MLP, B.mlp_options(knot=4, probe_fraction=0.0))
            for _ in range(a.reps):
                r.render(cam, out=out, timings=False)
    elif a.case == "mlp_tc":
        # the tcgen05 forward on 2^21 rows of device-resident features
        s = scenes.small(5, n=32, image=16, m=8)
        r = B.Renderer(0)
        r.set_volume(s.field_numpy(), origin=s.origin, spacing=s.spacing, value_range=s.value_range)
        s.configure(r)
        rng = np.random.default_rng(1)
        r.mlp_set_params(rng.normal(0, 0.1, B.lib().beams_mlp_param_count()).astype(np.float32))
        n = 1 << 21
        X = torch.empty((n, 112), device="cuda").uniform_(-1, 1).to(torch.bfloat16)
        T = torch.empty(n, device="cuda")
        for _ in range(a.reps):
            r.mlp_forward_tc_device(X, T)
    elif a.case in ("precision_light", "precision_view"):
        s = scenes.config2(n=640, image=1024, m=320)
        fd = s.field_device()
        r = B.Renderer(0)
        r.set_volume(fd, origin=s.origin, spacing=s.spacing, value_range=s.value_range)
        s.configure(r)
        r.set_form(B.FORM_PRECISION, B.BF16)
        r.set_tuning(light_brick=8, empty_skip=True, view_skip=True)
        if a.case == "precision_light":
            for _ in range(a.reps):
                r.build_shadow_map(timings=False)
        else:
            r.build_shadow_map(timings=False)
            r.set_reuse_shadow_map(True)
            out = torch.empty((s.height, s.width, 4), device="cuda")
            for _ in range(a.reps):
                r.render(s.camera(), out=out, timings=False)
    elif a.case == "bricks":
        s = scenes.config1()
        fd = s.field_device()
        cells = s.dims[0] - 1
        edges = [round(i * cells / 2) for i in range(3)]
        h = s.spacing
        bricks = []  # 2x2x2; neighbours share their face plane
        for z0, z1 in zip(edges[:-1], edges[1:]):
            for y0, y1 in zip(edges[:-1], edges[1:]):
                for x0, x1 in zip(edges[:-1], edges[1:]):
                    org = (s.origin[0] + x0 * h[0], s.origin[1] + y0 * h[1], s.origin[2] + z0 * h[2])
                    bricks.append((fd[z0:z1 + 1, y0:y1 + 1, x0:x1 + 1].contiguous(), org, h, s.value_range))
        del fd
        r = B.Renderer(0)
        r.set_bricks(bricks)
        s.configure(r)
        r.set_shadow_map_size(s.map_m // 2)
        cam = s.camera()
        out = torch.empty((s.height, s.width, 4), device="cuda")
        for _ in range(a.reps):
            r.render(cam, out=out, timings=False)
    else:  # batch
        sys.path.insert(0, str(__import__("pathlib").Path(__file__).resolve().parent.parent))
        import bench
        vols = bench.batch_volumes()
        rng = np.random.default_rng(11)
        n = 16
        sizes = [int(rng.choice(bench.BATCH_IMAGES)) for _ in range(n)]
        outs = [torch.empty((w, w, 4), device="cuda") for w in sizes]
        r = B.Renderer(0)
        r.set_color_map(scenes.tf_table())
        r.batch_set_volumes([(f, sc.origin, sc.spacing, sc.value_range) for sc, f in vols])
        r.set_batch_options(tile_w=32, tile_h=32, light_brick=8, skip=True, split=a.split)
        reqs = bench.batch_requests(B, vols, rng, n, outs)
        for _ in range(a.reps):
            r.render_batch(reqs, timings=False)
    torch.cuda.synchronize()
    print(f"profile case {a.case}: ok")
    return 0


if __name__ == "__main__":
    sys.exit(main())
