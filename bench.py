#!/usr/bin/env python
"""Benchmark of the Beams lighted volume renderer hot path on B200.

One step = one frame of the exact path at the 512^3 noise / 1024x1024 / M = 256
configuration (config 1): the light march that builds the 257^3
transmittance map (K1) and the view march that shades by it (K2), with the
field already resident in HBM. Synthetic seeded input; the 512 MiB field is
larger than L2, so no flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
  python bench.py --form precision [--field-dtype bf16|f16]   # config 2, 1024^3, 2048^2, M = 512
  python bench.py --form mlp [--knot 4] [--mlp-scene-light]    # learned form on the config 1 field
  python bench.py --form batch [--requests 64]                 # config 3: batched requests, one launch
  python bench.py --form bricks                                # config 3: 2x2x2 bricks of the 512^3 field
  python bench.py --profile-case light_march [--reps 3]        # one fixed small case per kernel, for ncu

N > 1 runs N independent replicas (the path does not shard across GPUs: there
is no exchange step), launched by torch.distributed.run; value is the total over
ranks divided by the slowest rank's time.

The line carries:
  value       lit samples/s over the timed frames (map build + view march),
  ms_per_step frame time (ms/frame),
  e2e         the same metric through the C ABI with host buffers: every step
              uploads the field from pinned host memory and reads the image back,
  roofline    the dominant kernel's algorithmic bytes / its CUDA-event time,
              against the measured HBM copy bandwidth,
  cpu_baseline the CPU oracle (the reference algorithm, OpenMP) on one whole
              frame when a sample says it fits the budget (the sample's
              extrapolation and its error beside it), else on the sample,
  learned     the metric's second half: the learned form on the same frame,
              with the specified network (32 training lights) and with a network
              trained for the rendered light; frames/s against the exact frame,
              PSNR against the FP64 oracle on crops, fallback tiles, tensor
              roofline (training is not timed).
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "lit samples/s & ms/frame @1024² on 1 B200; MLP vs exact shadow at ≥45 dB PSNR"
UNIT = "lit samples/s"
BYTES_LIGHT_SAMPLE = 32    # 8 field corners, float32
BYTES_MAP_VERTEX = 4       # one float32 opacity written per vertex
BYTES_LIT_SAMPLE = 64      # 8 field corners + 8 map corners, float32
BYTES_PIXEL = 16           # RGBA float32 written per ray


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic(kernel: str):
    """Per-launch DRAM bytes of a kernel from the committed ncu summaries, if any.
    Lines look like: `traffic_bytes_per_launch[k_light_march]: 123456`."""
    d = os.path.join(ROOT, "profiles")
    if not os.path.isdir(d):
        return None
    pat = re.compile(rf"traffic_bytes_per_launch\[{re.escape(kernel)}\]:\s*([0-9.eE+]+)")
    for name in sorted(os.listdir(d)):
        if not name.endswith((".md", ".txt")):
            continue
        with open(os.path.join(d, name)) as f:
            m = pat.search(f.read())
        if m:
            return float(m.group(1))
    return None


class ClockSampler:
    """Samples SM clock and throttle reasons through NVML while the timed region runs."""
    REASONS = {0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap", 0x8: "hw_slowdown",
               0x10: "sync_boost", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown",
               0x80: "hw_power_brake_slowdown", 0x100: "display_clock_setting"}

    def __init__(self, device_index: int, period_s: float = 0.02):
        self.samples, self.reasons, self.max_mhz = [], set(), None
        self.period = period_s
        self._stop = threading.Event()
        self._h = None
        try:
            import pynvml as N
            N.nvmlInit()
            self.N = N
            self._h = self._handle(device_index)
            self.max_mhz = N.nvmlDeviceGetMaxClockInfo(self._h, N.NVML_CLOCK_SM)
        except Exception as e:  # no NVML: report the absence, not a guess
            self.error = str(e)

    def _handle(self, idx):
        import torch
        N = self.N
        try:
            uuid = str(torch.cuda.get_device_properties(idx).uuid)
            return N.nvmlDeviceGetHandleByUUID(("GPU-" + uuid) if not uuid.startswith("GPU-") else uuid)
        except Exception:
            return N.nvmlDeviceGetHandleByIndex(idx)

    def _run(self):
        N = self.N
        while not self._stop.is_set():
            try:
                self.samples.append(N.nvmlDeviceGetClockInfo(self._h, N.NVML_CLOCK_SM))
                r = N.nvmlDeviceGetCurrentClocksEventReasons(self._h)
                for bit, name in self.REASONS.items():
                    if r & bit:
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(self.period)

    def __enter__(self):
        if self._h is not None:
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._h is not None:
            self._t.join()

    def summary(self):
        if self._h is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "note": "NVML unavailable"}
        busy = [s for s in self.samples if s > 0]
        return {"sm_mhz": statistics.median(busy) if busy else None, "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons - {"gpu_idle"}), "samples": len(self.samples)}


def max_over_ranks(ms: float, world: int, device: str = "cuda") -> float:
    """The slowest rank's time (all ranks take part; world == 1 returns ms)."""
    if world <= 1:
        return float(ms)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(world: int, steps: int, units_per_step: float, max_ms: float) -> float:
    """Whole-job throughput of N independent replicas: all units over the slowest rank's time."""
    return world * steps * units_per_step / (max_ms / 1e3)


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def build_scene(config: int):
    from pilot_b200 import scenes
    return {0: scenes.config0, 1: scenes.config1, 2: scenes.config2}[config]()


def workload_desc(s, config: int):
    return {"workload": f"config{config}: {s.dims[0]}^3 {s.kind} f32 field, {s.width}x{s.height} image, "
                        f"M={s.map_m} map ({s.map_m + 1}^3 vertices), view step 0.5 voxel, light step "
                        f"|extent|/128, alpha cut {s.cutoff}, {'point' if s.light_kind == 0 else 'directional'} light",
            "field": list(s.dims), "image": [s.width, s.height], "map_cells": s.map_m,
            "l2": "inputs larger than L2 (512 MiB field > 126 MB L2); no flush" if config == 1 else
                  "field 8 MiB fits L2: per-step L2 flush",
            "form": "exact"}


# ---------------------------------------------------------------------------
# CPU baseline / reference arm: the oracle (the reference algorithm restated in
# C++, float32 as the reference computes) on the host cores.
# ---------------------------------------------------------------------------
def cpu_sample_frame(scene, field, map_values, budget_s: float, threads: int, rng_seed: int = 0):
    """Times the oracle on a bounded sample of one frame and extrapolates.

    Light march: whole z-slabs of map vertices, evenly spread over z and each
    marched in the map's raster order (as a full build runs them). View march:
    evenly spread whole image rows, shading by map_values (the shading only
    scales colour, so the work does not depend on the map's values). Returns
    per-frame estimates."""
    from oracle.oracle import Oracle
    o = Oracle(scene, field=field, threads=threads)
    pd = scene.map_m + 1
    slab = pd * pd
    nvert = pd ** 3
    # calibrate on one slab and one row, then size the sample to the budget
    mid = pd // 2
    t0 = time.perf_counter()
    o.light_march_ids(np.arange(mid * slab, (mid + 1) * slab, dtype=np.int64))
    per_slab = time.perf_counter() - t0
    t0 = time.perf_counter()
    row = scene.height // 2
    o.view_march(map_values, window=(0, row, scene.width, 1))
    per_row = time.perf_counter() - t0
    nslabs = int(min(pd, max(1, 0.6 * budget_s / max(per_slab, 1e-9))))
    nrows = int(min(scene.height, max(1, 0.4 * budget_s / max(per_row, 1e-9))))
    off = np.random.default_rng(rng_seed).random()
    zs = np.unique(np.minimum(pd - 1, ((np.arange(nslabs) + off) * pd / nslabs).astype(np.int64)))
    ids = np.concatenate([np.arange(z * slab, (z + 1) * slab, dtype=np.int64) for z in zs])
    t0 = time.perf_counter()
    _, light_samples = o.light_march_ids(ids)  # one call: the slabs in raster order
    t_light = time.perf_counter() - t0
    # the rows as 8 evenly spread bands of whole rows, one call per band
    nb = min(8, nrows)
    bh = max(1, nrows // nb)
    y0s = np.unique(np.linspace(0, scene.height - bh, nb).round().astype(int))
    t0 = time.perf_counter()
    lit = 0
    for y in y0s:
        _, l = o.view_march(map_values, window=(0, int(y), scene.width, bh))
        lit += l
    t_view = time.perf_counter() - t0
    nrows = y0s.size * bh
    frame_s = t_light * nvert / ids.size + t_view * scene.height / nrows
    lit_frame = lit * scene.height / nrows
    return {"frame_s": frame_s, "lit_per_frame": lit_frame, "value": lit_frame / frame_s,
            "sample": f"{zs.size} of {pd} whole z-slabs of map vertices (raster order, evenly spread) + "
                      f"{y0s.size} bands of {bh} of {scene.height} image rows; timed {t_light + t_view:.1f} s, "
                      f"extrapolated to one frame",
            "t_light_s": t_light, "t_view_s": t_view, "light_samples_sampled": light_samples}


def cpu_full_frame(scene, field, threads: int):
    """One whole frame on the oracle: the light march over every map vertex,
    then the view march over every pixel shading by that map."""
    from oracle.oracle import Oracle
    o = Oracle(scene, field=field, threads=threads)
    t0 = time.perf_counter()
    m, light_samples = o.light_march()
    t1 = time.perf_counter()
    _, lit = o.view_march(m)
    t2 = time.perf_counter()
    return {"frame_s": t2 - t0, "light_s": t1 - t0, "view_s": t2 - t1, "lit_per_frame": lit,
            "light_samples": light_samples, "value": lit / (t2 - t0), "map": m}


def run_reference(args):
    world, rank, _ = dist_setup()
    if rank != 0:
        return 0
    from oracle.oracle import noise_field
    threads = os.cpu_count() or 1
    s = build_scene(args.config)
    if s.kind == "noise":
        field = noise_field(s.dims, s.params, s.octaves, s.base_freq, threads=threads)
    else:
        field = s.field_numpy()
    zero_map = np.zeros((s.map_m + 1,) * 3, np.float32)
    # one whole frame first (untimed): the yardstick of the per-step extrapolation
    full = cpu_full_frame(s, field, threads) if not args.no_full_frame else None
    per_step = max(1.0, min(10.0, 150.0 / max(1, args.steps + args.warmup)))
    results = []
    for i in range(args.warmup + args.steps):
        r = cpu_sample_frame(s, field, zero_map, per_step, threads, rng_seed=i)
        if i >= args.warmup:
            results.append(r)
    frame_s = float(np.mean([r["frame_s"] for r in results]))
    lit = float(np.mean([r["lit_per_frame"] for r in results]))
    value = lit / frame_s
    check = None
    if full is not None:
        check = {"full_frame_s": full["frame_s"], "full_frame_light_s": full["light_s"],
                 "full_frame_view_s": full["view_s"], "full_frame_value": full["value"],
                 "extrapolated_frame_s": frame_s,
                 "extrapolation_error": frame_s / full["frame_s"] - 1.0,
                 "lit_error": lit / full["lit_per_frame"] - 1.0}
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": frame_s * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded gradient noise generated on the CPU)",
            "config": workload_desc(s, args.config),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": results[-1]["sample"] + "; the reference cannot be built here (VTK-m, "
                                       "MPI absent), so its algorithm runs as the project's C++ restatement"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "full_frame_check": check}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def run_ours(args):
    import torch
    import torch.distributed as dist

    from pilot_b200 import beams as B

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    stream = torch.cuda.current_stream()
    s = build_scene(args.config)
    fd = s.field_device()
    r = B.Renderer(local, stream=stream.cuda_stream)
    r.set_volume(fd, origin=s.origin, spacing=s.spacing, value_range=s.value_range)
    s.configure(r)
    cam = s.camera()
    out = torch.empty((s.height, s.width, 4), dtype=torch.float32, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda") if args.config != 1 else None

    r.render(cam, out=out, timings=True)                  # builds the cell tables and quad field
    if args.no_autotune:  # the tuning the autotuner picks for this workload, fixed
        r.set_tuning(light_brick=8, empty_skip=False, view_skip=False)
        tuning = dict(r.get_tuning(), autotuned=False)
    else:
        tuning = r.autotune(cam)                          # launch choices only; results are identical
    _, t0 = r.render(cam, out=out, timings=True)          # counts for one frame (deterministic)
    lit_frame, light_frame = t0["lit_samples"], t0["light_samples"]
    launches_per_frame = t0["kernel_launches"]
    r.set_reuse_shadow_map(True)   # the explicit build below is the frame's map; render reuses it

    def frame(evs=None):
        if flush is not None:
            flush.zero_()
        if evs:
            evs[0].record(stream)
        r.build_shadow_map(timings=False)
        if evs:
            evs[1].record(stream)
        r.render(cam, out=out, timings=False)
        if evs:
            evs[2].record(stream)

    for _ in range(args.warmup):
        frame()
    torch.cuda.synchronize()
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    with sampler:
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        for i in range(args.steps):
            frame(evs[i])
        stop.record(stream)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    total_ms = start.elapsed_time(stop)
    if flush is not None:  # the flush is not part of a frame
        total_ms = sum(e[0].elapsed_time(e[2]) for e in evs)
    k1_ms = sum(e[0].elapsed_time(e[1]) for e in evs) / args.steps
    k2_ms = sum(e[1].elapsed_time(e[2]) for e in evs) / args.steps
    max_ms = max_over_ranks(total_ms, world)
    value = replica_value(world, args.steps, lit_frame, max_ms)

    # roofline of the dominant kernel
    peak, peak_kind = measured_peaks()
    nvert = (s.map_m + 1) ** 3
    npix = s.width * s.height
    k1_bytes = light_frame * BYTES_LIGHT_SAMPLE + nvert * BYTES_MAP_VERTEX
    k2_bytes = lit_frame * BYTES_LIT_SAMPLE + npix * BYTES_PIXEL
    if k1_ms >= k2_ms:
        kname, kbytes, kms = "k_light_march", k1_bytes, k1_ms
    else:
        kname, kbytes, kms = "k_view_march", k2_bytes, k2_ms
    achieved = kbytes / (kms / 1e3) / 1e9
    roofline = {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_kind, "traffic": profiled_traffic(kname),
                "algorithmic_bytes_per_launch": kbytes,
                "bytes_model": "light sample 32 B + 4 B/vertex; lit sample 64 B + 16 B/pixel",
                "k_light_march_ms": k1_ms, "k_view_march_ms": k2_ms,
                "k_light_march_GBps": k1_bytes / (k1_ms / 1e3) / 1e9,
                "k_view_march_GBps": k2_bytes / (k2_ms / 1e3) / 1e9}
    # compulsory footprint: every byte the launch must touch once (the 4-corner
    # quad field it reads, 16 B per cell, and the map it writes; for the view
    # march the quads, the map and the image)
    ncell = (s.dims[0] - 1) * (s.dims[1] - 1) * s.dims[2]
    unique = ncell * 16 + nvert * 4 if kname == "k_light_march" else ncell * 16 + nvert * 4 + npix * 16
    roofline["compulsory_bytes_per_launch"] = unique
    roofline["compulsory_frac"] = unique / (kms / 1e3) / 1e9 / peak

    # end to end through the C ABI with host buffers: every step uploads the
    # field from pinned host memory (beams_set_volume) and renders into pinned
    # host memory (BEAMS_OUT_HOST_ASYNC). Two renderers on two streams take the
    # steps in turn, so one step's upload overlaps the other's render, as a
    # double-buffered serving loop would run; a step's image is waited for
    # (beams_synchronize) before its renderer takes the next step.
    e2e = None
    if not args.no_e2e:
        host_field = fd.cpu().pin_memory()
        side = torch.cuda.Stream()
        r2 = B.Renderer(local, stream=side.cuda_stream)
        r2.set_volume(fd, origin=s.origin, spacing=s.spacing, value_range=s.value_range)
        s.configure(r2)
        r2.set_tuning(**{k: tuning[k] for k in ("light_brick", "empty_skip", "view_skip")})
        rs = (r, r2)
        host_outs = [torch.empty((s.height, s.width, 4), dtype=torch.float32).pin_memory() for _ in rs]
        r.set_reuse_shadow_map(False)

        def e2e_step(i):
            q = rs[i % 2]
            if i >= 2:
                q.synchronize()  # step i-2's image is in host_outs[i % 2]
            q.set_volume(host_field, dims=s.dims, origin=s.origin, spacing=s.spacing, value_range=s.value_range)
            q.render(cam, out=host_outs[i % 2], timings=False, host_async=True)

        for i in range(4):
            e2e_step(i)
        for q in rs:
            q.synchronize()
        ne = max(4, min(args.steps, 20))
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        w0 = time.perf_counter()
        for i in range(ne):
            e2e_step(i)
        for q in rs:
            q.synchronize()
        te_ms = max_over_ranks((time.perf_counter() - w0) * 1e3, world)
        e2e = {"value": replica_value(world, ne, lit_frame, te_ms), "unit": UNIT,
               "h2d_bytes_per_step": int(host_field.numel() * 4),
               "d2h_bytes_per_step": int(host_outs[0].numel() * 4),
               "ms_per_step": te_ms / ne,
               "path": "beams_set_volume(pinned host field) + beams_render(pinned host image, BEAMS_OUT_HOST_ASYNC) "
                       "per step on two renderers and streams in turn; wall clock, synchronised at both ends"}
        del r2
        r.set_reuse_shadow_map(True)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        field = fd.cpu().numpy()
        gpu_map = r.get_shadow_map(nvert).reshape((s.map_m + 1,) * 3)
        c = cpu_sample_frame(s, field, gpu_map, args.cpu_budget, threads)
        cpu = {"value": c["value"], "unit": UNIT, "cores": threads, "kind": "port", "sample": c["sample"],
               "ms_per_frame": c["frame_s"] * 1e3}
        # a whole frame when the sample says it fits the budget: it replaces the
        # extrapolation, which is kept beside it with its error
        if not args.no_full_frame and c["frame_s"] <= 4.0 * args.cpu_budget:
            f = cpu_full_frame(s, field, threads)
            cpu = {"value": f["value"], "unit": UNIT, "cores": threads, "kind": "port",
                   "sample": f"one whole frame: light march over all {nvert} map vertices, view march over all "
                             f"{npix} pixels ({f['frame_s']:.1f} s)",
                   "ms_per_frame": f["frame_s"] * 1e3, "light_ms": f["light_s"] * 1e3, "view_ms": f["view_s"] * 1e3,
                   "map_equals_gpu": bool(np.array_equal(f["map"], gpu_map)),
                   "extrapolated_from_sample": {"ms_per_frame": c["frame_s"] * 1e3, "sample": c["sample"],
                                                "error": c["frame_s"] / f["frame_s"] - 1.0}}

    # the exact form with the lazy map (beams_set_lazy_shadow_map): the same
    # frame with only the map vertices the view rays read built; the image must
    # equal the full map's bit for bit
    lazy = None
    exact_img = None
    if not args.no_lazy:
        r.set_reuse_shadow_map(False)
        r.render(cam, out=out, timings=False)
        exact_img = out.cpu().numpy()
        r.set_lazy_shadow_map(True)
        _, tl = r.render(cam, out=out, timings=True)
        same = bool(np.array_equal(out.cpu().numpy(), exact_img))
        lms, lclk = time_frames(lambda: r.render(cam, out=out, timings=False), args.steps, args.warmup, stream,
                                world, local)
        # the same field and light seen from 2 and 3 units instead of 1 (the
        # whole volume in view): full against lazy, a few frames each
        views = {}
        cdir = np.asarray(s.cam_pos, np.float64) - 0.5
        for dist in (2.0, 3.0):
            vpos = tuple(float(v) for v in 0.5 + cdir / np.linalg.norm(cdir) * dist)
            vcam = B.Renderer.camera(vpos, s.cam_look, s.cam_up, s.fov_y_deg, s.width, s.height)
            rec = {}
            for lz in (False, True):
                r.set_lazy_shadow_map(lz)
                _, tv = r.render(vcam, out=out, timings=True)
                rec["lazy" if lz else "full"] = out.cpu().numpy()
                vms, _ = time_frames(lambda: r.render(vcam, out=out, timings=False), 5, 2, stream, world, local)
                rec[("lazy" if lz else "full") + "_ms"] = vms / 5
                if lz:
                    rec["map_vertices_built"] = tv["map_vertices"]
                else:
                    rec["lit_samples"] = tv["lit_samples"]
            views[f"distance_{dist:g}"] = {"full_ms_per_frame": rec["full_ms"], "lazy_ms_per_frame": rec["lazy_ms"],
                                          "map_vertices_built": rec["map_vertices_built"],
                                          "lit_samples": rec["lit_samples"],
                                          "image_equals_full_map": bool(np.array_equal(rec["lazy"], rec["full"]))}
        # a light orbit around the fixed camera (the loop of the reference's Beams::Run): the
        # point light steps around the vertical axis every frame; with the marks
        # kept (mode 2) only the listed vertices are built again
        lpos0 = np.asarray(s.light, np.float64) - 0.5
        orbit = {}
        step = [0]

        def orbit_frame():
            a = 2.0 * np.pi * (step[0] % 24) / 24.0
            step[0] += 1
            c, sn = np.cos(a), np.sin(a)
            lp = (0.5 + c * lpos0[0] + sn * lpos0[2], 0.5 + lpos0[1], 0.5 - sn * lpos0[0] + c * lpos0[2])
            r.clear_lights()
            r.add_point_light(tuple(float(v) for v in lp), s.light_color, s.light_intensity)
            r.render(cam, out=out, timings=False)

        for mode, name in ((0, "full_map"), (1, "lazy"), (2, "lazy_kept_marks")):
            r.set_lazy_shadow_map(mode != 0, keep_marks=mode == 2)
            oms, _ = time_frames(orbit_frame, 24, 3, stream, world, local)
            orbit[name + "_ms_per_frame"] = oms / 24
            r.set_lazy_shadow_map(False)
        orbit["frames"] = "24 light positions around the vertical axis, 15 degrees apart, camera fixed"
        s.configure(r)
        r.set_lazy_shadow_map(False)
        lazy = {"ms_per_frame": lms / args.steps, "value": replica_value(world, args.steps, lit_frame, lms),
                "unit": UNIT, "map_build_ms": tl["map_build_ms"], "view_march_ms": tl["view_march_ms"],
                "map_vertices_built": tl["map_vertices"], "map_vertices": nvert,
                "lit_samples_equal": tl["lit_samples"] == lit_frame, "image_equals_full_map": same,
                "speedup_vs_full_map": (max_ms / args.steps) / (lms / args.steps), "clocks": lclk,
                "other_views": views, "light_orbit": orbit,
                "note": "a view march without shading marks the map cells the rays read, the light march builds "
                        "the marked cells' corners, then the view march; map_build_ms covers the marking"}

    # the metric's second half: the learned form on the same field, camera and
    # light, against this run's exact frame (the network as specified,
    # trained over 32 light directions, and a network trained for the rendered
    # light); training runs before each record's timed frames
    learned = None
    if not args.no_learned:
        r.set_reuse_shadow_map(False)
        if exact_img is None:
            r.render(cam, out=out, timings=False)
            exact_img = out.cpu().numpy()
        field_host = None
        if rank == 0 and not args.no_quality:
            field_host = field if cpu is not None else fd.cpu().numpy()
        learned = {}
        for name, lights, scene_light in (("lights32", 32, False), ("scene_light", 1, True)):
            rec, _, _, _, _ = learned_record(
                B, r, s, cam, out, exact_img, max_ms / args.steps, stream, world, local, lights=lights,
                scene_light=scene_light, knot=args.learned_knot, probe_fraction=args.probe_fraction,
                fallback_tol=args.fallback_tol, samples_log2=args.mlp_samples_log2, epochs=args.mlp_epochs,
                steps=max(10, min(args.steps, 50)), warmup=3, field_host=field_host, crops=args.crops,
                crop=args.crop, crop_stride=args.crop_stride, threads=os.cpu_count() or 1)
            rec["network"] = ("as specified: 2^24 samples over 32 light directions uniform on the sphere"
                              if lights == 32 else "2^24 samples for the rendered light only (fixed light, any camera)")
            if lazy is not None:
                rec["speedup_vs_exact_lazy_map"] = lazy["ms_per_frame"] / rec["ms_per_frame"]
                # the lazy record's wider views, rendered by this network
                rec["other_views"] = {}
                cdir = np.asarray(s.cam_pos, np.float64) - 0.5
                for vname, v in lazy["other_views"].items():
                    dist = float(vname.split("_")[1])
                    vpos = tuple(float(c) for c in 0.5 + cdir / np.linalg.norm(cdir) * dist)
                    vcam = B.Renderer.camera(vpos, s.cam_look, s.cam_up, s.fov_y_deg, s.width, s.height)
                    for _ in range(2):  # the frame order settles on the failing-tile count
                        _, tv = r.render(vcam, out=out, timings=True)
                    vms, _ = time_frames(lambda: r.render(vcam, out=out, timings=False), 5, 2, stream, world, local)
                    rec["other_views"][vname] = {"ms_per_frame": vms / 5, "fallback_tiles": tv["fallback_tiles"],
                                                 "speedup_vs_exact": v["full_ms_per_frame"] / (vms / 5),
                                                 "speedup_vs_exact_lazy_map": v["lazy_ms_per_frame"] / (vms / 5)}
            learned[name] = rec
        r.set_form(B.FORM_EXACT)

    # the other forms, each in its own configuration (one GPU, the default run only):
    # config 2 precision (no FP64 crops here), config 3 batch, the config-1 field as bricks
    forms = None
    if world == 1 and not args.no_forms:
        forms = {}
        for name, fn, over in (("precision_config2", run_form, dict(form="precision", config=2, no_quality=True)),
                               ("batch_config3", run_batch, dict(form="batch")),
                               ("bricks_2x2x2", run_bricks, dict(form="bricks"))):
            sub = argparse.Namespace(**dict(vars(args), steps=min(args.steps, 10), warmup=3, **over))
            try:
                rec = fn(sub, nested=True)
                forms[name] = {k: v for k, v in rec.items()
                               if k not in ("metric", "unit", "n_gpus", "higher_is_better", "scaling", "vs_baseline")}
            except Exception as ex:  # a failing form must not cost the headline line
                forms[name] = {"error": repr(ex)[:400]}
            torch.cuda.synchronize()
            torch.cuda.empty_cache()

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": max_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded 4-octave gradient noise, generated on the device)",
                "config": dict(workload_desc(s, args.config), parallelism=f"replicas x{world}", tuning=tuning),
                "ms_per_frame": max_ms / args.steps, "map_build_ms": k1_ms, "view_march_ms": k2_ms,
                "view_only_map_cached": {"ms_per_frame": k2_ms, "value": lit_frame / (k2_ms / 1e3), "unit": UNIT,
                                         "note": "the frame's view march, rendering with the frame's map reused"},
                "lit_samples_per_frame": lit_frame, "light_samples_per_frame": light_frame,
                "gpu_launches": launches_per_frame * args.steps,
                "roofline": roofline, "e2e": e2e, "cpu_baseline": cpu, "clocks": sampler.summary(),
                "exact_lazy_map": lazy, "learned": learned, "forms": forms}
        print(json.dumps(line), flush=True)
    r.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


# ---------------------------------------------------------------------------
# the other forms: --form precision (config 2) and --form mlp (config 1 field)
# ---------------------------------------------------------------------------
MLP_FLOP_PER_EVAL = 2 * (112 * 64 + 3 * 64 * 64 + 64)  # 39,040 FLOP per network evaluation


def measured_tensor_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("bf16_tflops", 1590.0)), "measured (burst)"
    return 1590.0, "fallback"


def time_frames(frame, steps, warmup, stream, world, local):
    """W untimed frames, then K frames between device events; max over ranks."""
    import torch
    import torch.distributed as dist
    for _ in range(warmup):
        frame()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    with sampler:
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(steps):
            frame()
        b.record(stream)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    return max_over_ranks(a.elapsed_time(b), world), sampler.summary()


def fp64_crops(s, field, images, crop, stride, ncrops, threads):
    """PSNR / max |d| of each image against the FP64 oracle (lazy map) on ncrops
    crop x crop windows, every stride-th pixel."""
    from oracle.oracle import Oracle, psnr
    o = Oracle(s, field=field, threads=threads)
    rng = np.random.default_rng(7)
    res = {k: [] for k in images}
    t0 = time.perf_counter()
    for c in range(ncrops):
        x0 = int(rng.integers(0, s.width - crop + 1)) if c else (s.width - crop) // 2
        y0 = int(rng.integers(0, s.height - crop + 1)) if c else (s.height - crop) // 2
        ref, _ = o.view_march_lazy_f64((x0, y0, crop, crop), stride=stride)
        for k, img in images.items():
            sub = img[y0:y0 + crop:stride, x0:x0 + crop:stride]
            res[k].append((psnr(sub, ref), float(np.abs(sub - ref).max()), float(np.abs(sub - ref).mean())))
    out = {k: {"psnr_db": float(np.mean([v[0] for v in r])), "max_abs": max(v[1] for v in r),
               "mean_abs": float(np.mean([v[2] for v in r]))} for k, r in res.items()}
    out["crops"] = f"{ncrops} crops of {crop}x{crop}, every {stride}th pixel, FP64 oracle with lazy map"
    out["oracle_s"] = time.perf_counter() - t0
    return out


def learned_record(B, r, s, cam, out, exact_img, exact_ms, stream, world, local, *, lights, scene_light, knot,
                   probe_fraction, fallback_tol, samples_log2, epochs, steps, warmup, field_host=None, crops=3,
                   crop=128, crop_stride=1, threads=1):
    """Trains the learned form's network (untimed), then times its frames (network
    view march + probe check + fallback) and reports speed against the exact
    frame, fallback tiles, the tensor roofline of the fused network march and the
    image error against the exact-map image and (field_host given) the FP64
    oracle. Leaves the renderer in the learned form."""
    from oracle.oracle import psnr
    rep = r.mlp_train(B.mlp_options(samples_log2=samples_log2, n_lights=lights, epochs=epochs,
                                    scene_light=int(scene_light)))
    opts = dict(knot=knot, probe_fraction=probe_fraction, fallback_tol=fallback_tol)
    # the network alone (no probes): its kernel time for the tensor roofline and its image
    r.set_form(B.FORM_MLP, B.mlp_options(**dict(opts, probe_fraction=0.0)))
    r.render(cam, out=out, timings=True)
    _, tn = r.render(cam, out=out, timings=True)
    net_img = out.cpu().numpy()
    r.set_form(B.FORM_MLP, B.mlp_options(**opts))
    _, tm = r.render(cam, out=out, timings=True)
    img = out.cpu().numpy()
    frame = lambda: r.render(cam, out=out, timings=False)  # noqa: E731  network + probes + fallback
    total_ms, clocks = time_frames(frame, steps, warmup, stream, world, local)
    tpeak, tsrc = measured_tensor_peak()
    flops = tn["mlp_samples"] * MLP_FLOP_PER_EVAL
    ach = flops / (tn["view_march_ms"] / 1e3) / 1e12
    ntiles = -(-s.width // 32) * -(-s.height // 32)
    ms = total_ms / steps
    rec = {"train": {k: rep[k] for k in ("datagen_ms", "train_ms", "holdout_rmse", "unlit_rmse", "mean_rmse", "steps",
                                         "samples")},
           "train_note": "training (data generation by the exact light march + Adam) runs before the timed frames",
           "lights": lights, "scene_light": bool(scene_light), "knot": knot, "probe_fraction": probe_fraction,
           "fallback_tol": fallback_tol, "fallback_tiles": tm["fallback_tiles"], "tiles": ntiles,
           "network_evaluations": tm["mlp_samples"], "ms_per_frame": ms, "frames_per_s": 1e3 / ms,
           "exact_ms_per_frame": exact_ms, "exact_frames_per_s": 1e3 / exact_ms,
           "speedup_vs_exact": exact_ms / ms, "network_only_ms": tn["total_ms"],
           "roofline": {"bound": "tensor", "kernel": "k_view_march_mlp", "achieved": ach, "peak": tpeak,
                        "unit": "TFLOP/s", "frac": ach / tpeak, "peak_source": tsrc,
                        "flops_model": f"{MLP_FLOP_PER_EVAL} FLOP per network evaluation",
                        "evaluations": tn["mlp_samples"], "kernel_ms": tn["view_march_ms"]},
           "psnr_vs_exact_map_full_frame": psnr(img, exact_img),
           "network_only_psnr_vs_exact_map": psnr(net_img, exact_img), "clocks": clocks,
           "launches_per_frame": tm["kernel_launches"]}
    # per-tile probe errors of the last frame: max |dRGBA| over each 32x32 tile's
    # probes against the exact light march (the fallback decision), as a histogram
    if probe_fraction > 0:
        P = max(1, int(round(1.0 / np.sqrt(min(probe_fraction, 1.0)))))
        off = P // 2
        nqx = (s.width - off - 1) // P + 1 if s.width > off else 0
        nqy = (s.height - off - 1) // P + 1 if s.height > off else 0
        if nqx * nqy > 0:
            perr = r.mlp_probe_errors(nqx * nqy).reshape(nqy, nqx)
            tx, ty = -(-s.width // 32), -(-s.height // 32)
            tmax = np.full((ty, tx), np.inf)
            seen = np.zeros((ty, tx), bool)
            for j in range(nqy):
                for i in range(nqx):
                    y, x = j * P + off, i * P + off
                    t0 = tmax[y // 32, x // 32]
                    tmax[y // 32, x // 32] = perr[j, i] if not seen[y // 32, x // 32] else max(t0, perr[j, i])
                    seen[y // 32, x // 32] = True
            edges = [0.0, 1e-3, 3e-3, 1e-2, 3e-2, 1e-1, 3e-1, np.inf]
            hist, _ = np.histogram(np.where(np.isfinite(tmax), tmax, 1e30), bins=edges)
            rec["tile_probe_error_histogram"] = {"edges": [str(e) for e in edges], "tiles": hist.tolist(),
                                                 "median": float(np.median(tmax)),
                                                 "note": "per 32x32 tile: max |dRGBA| of its probe pixels against "
                                                         "the exact light march; above fallback_tol falls back"}
    if field_host is not None:
        rec["vs_fp64"] = fp64_crops(s, field_host, {"learned_form": img, "network_only": net_img,
                                                    "exact": exact_img}, crop, crop_stride, crops, threads)
        rec["target_met"] = bool(rec["speedup_vs_exact"] >= 3.0 and rec["vs_fp64"]["learned_form"]["psnr_db"] >= 45.0)
    return rec, total_ms, clocks, tm, tn


def run_form(args, nested=False):
    """--form precision / mlp. nested: called from the default run (no process
    group of its own, returns the line instead of printing it)."""
    import torch
    import torch.distributed as dist

    from oracle.oracle import psnr
    from pilot_b200 import beams as B
    from pilot_b200 import scenes

    world, rank, local = dist_setup()
    if nested:
        world, rank = 1, 0
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    stream = torch.cuda.current_stream()
    cfg = args.config
    s = scenes.config2() if cfg == 2 else build_scene(cfg)
    fd = s.field_device()
    r = B.Renderer(local, stream=stream.cuda_stream)
    r.set_volume(fd, origin=s.origin, spacing=s.spacing, value_range=s.value_range)
    s.configure(r)
    cam = s.camera()
    out = torch.empty((s.height, s.width, 4), dtype=torch.float32, device="cuda")
    threads = os.cpu_count() or 1

    # the exact form in the same run: the speed and quality reference of the form
    r.set_form(B.FORM_EXACT)
    r.render(cam, out=out, timings=False)
    exact_tuning = r.autotune(cam)
    _, te = r.render(cam, out=out, timings=True)
    exact_img = out.cpu().numpy()
    lit_frame = te["lit_samples"]
    exact_ms, _ = time_frames(lambda: r.render(cam, out=out, timings=False), max(3, args.steps // 4), 2, stream,
                              world, local)
    exact_ms /= max(3, args.steps // 4)
    # the exact form with the lazy map (only the vertices the view reads)
    r.set_lazy_shadow_map(True)
    _, tlz = r.render(cam, out=out, timings=True)
    lazy_same = bool(np.array_equal(out.cpu().numpy(), exact_img))
    exact_lazy_ms, _ = time_frames(lambda: r.render(cam, out=out, timings=False), max(3, args.steps // 4), 2,
                                   stream, world, local)
    exact_lazy_ms /= max(3, args.steps // 4)
    r.set_lazy_shadow_map(False)
    exact_lazy = {"ms_per_frame": exact_lazy_ms, "map_vertices_built": tlz["map_vertices"],
                  "image_equals_full_map": lazy_same}
    extra, roofline = {}, None
    if args.form == "precision":
        dt = B.F16 if args.field_dtype == "f16" else B.BF16
        r.set_form(B.FORM_PRECISION, dt)
        r.render(cam, out=out, timings=False)
        extra["tuning"] = r.autotune(cam)
        _, tp = r.render(cam, out=out, timings=True)
        img = out.cpu().numpy()
        launches = tp["kernel_launches"]
        frame = lambda: r.render(cam, out=out, timings=False)  # noqa: E731  map build + view march
        total_ms, clocks = time_frames(frame, args.steps, args.warmup, stream, world, local)
        # the precision form with the lazy map
        r.set_lazy_shadow_map(True)
        _, tpl = r.render(cam, out=out, timings=True)
        prec_lazy_same = bool(np.array_equal(out.cpu().numpy(), img))
        prec_lazy_ms, _ = time_frames(frame, max(3, args.steps // 4), 2, stream, world, local)
        prec_lazy = {"ms_per_frame": prec_lazy_ms / max(3, args.steps // 4), "map_vertices_built": tpl["map_vertices"],
                     "image_equals_full_map": prec_lazy_same}
        r.set_lazy_shadow_map(False)
        _, tk = r.render(cam, out=out, timings=True)
        nvert = (s.map_m + 1) ** 3
        kb = tk["light_samples"] * 16 + nvert * 2  # bf16/f16 quads: 8 corners x 2 B; binary16 map
        roofline = {"bound": "hbm", "kernel": "k_light_march (precision)", "unit": "GB/s",
                    "achieved": kb / (tk["map_build_ms"] / 1e3) / 1e9, "traffic": None,
                    "bytes_model": "light sample 16 B (8 16-bit corners) + 2 B/vertex",
                    "k_light_march_ms": tk["map_build_ms"], "k_view_march_ms": tk["view_march_ms"]}
        dtype = args.field_dtype
        extra["precision"] = {"field_dtype": dtype, "exact_f32_ms_per_frame": exact_ms, "exact_tuning": exact_tuning,
                              "speedup_vs_exact_f32": exact_ms / (total_ms / args.steps),
                              "exact_f32_lazy_map": exact_lazy, "lazy_map": prec_lazy,
                              "psnr_vs_exact_f32_full_frame": psnr(img, exact_img)}
        if not args.no_quality and rank == 0:
            extra["precision"]["vs_fp64"] = fp64_crops(s, fd.cpu().numpy(), {"precision": img, "exact_f32": exact_img},
                                                       args.crop, args.crop_stride, args.crops, threads)
    else:  # mlp
        rec, total_ms, clocks, tm, tn = learned_record(
            B, r, s, cam, out, exact_img, exact_ms, stream, world, local, lights=args.mlp_lights,
            scene_light=args.mlp_scene_light, knot=args.knot, probe_fraction=args.probe_fraction,
            fallback_tol=args.fallback_tol, samples_log2=args.mlp_samples_log2, epochs=args.mlp_epochs,
            steps=args.steps, warmup=args.warmup,
            field_host=None if (args.no_quality or rank != 0) else fd.cpu().numpy(), crops=args.crops,
            crop=args.crop, crop_stride=args.crop_stride, threads=threads)
        launches = tm["kernel_launches"]
        roofline = dict(rec["roofline"], traffic=None)
        dtype = "bf16"
        tpeak = roofline["peak"]
        # the tcgen05 forward kernel on 2^22 device-resident rows (training's forward pass)
        nrow = 1 << 22
        X = torch.empty((nrow, 112), device="cuda").uniform_(-1, 1).to(torch.bfloat16)
        Tt = torch.empty(nrow, device="cuda")
        tc_ms, _ = time_frames(lambda: r.mlp_forward_tc_device(X, Tt), 10, 3, stream, world, local)
        tc_ms /= 10
        tc_tflops = nrow * MLP_FLOP_PER_EVAL / (tc_ms / 1e3) / 1e12
        del X, Tt
        rec["tcgen05_forward"] = {"rows": nrow, "ms": tc_ms, "tflops": tc_tflops,
                                  "frac_of_bf16_peak": tc_tflops / tpeak,
                                  "note": "dense forward kernel (TMEM accumulators), training's forward"}
        extra["learned"] = rec
    if roofline.get("peak") is None:
        peak, src = measured_peaks()
        roofline.update(peak=peak, frac=roofline["achieved"] / peak, peak_source=src)
    value = world * args.steps * lit_frame / (total_ms / 1e3)
    if rank == 0:
        wl = workload_desc(s, cfg) if cfg != 2 else {
            "workload": f"config2: {s.dims[0]}^3 64 blobs + 10% noise, {s.width}x{s.height} image, M={s.map_m} "
                        f"binary16 map, view step 0.25 voxel, alpha cut {s.cutoff}, point light",
            "field": list(s.dims), "image": [s.width, s.height], "map_cells": s.map_m,
            "l2": "inputs larger than L2 (2 GiB 16-bit field); no flush"}
        wl = dict(wl, form=args.form, parallelism=f"replicas x{world}")
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": dtype,
                "data": "synthetic (seeded fields generated on the device)", "config": wl,
                "lit_samples_per_frame": lit_frame, "gpu_launches": launches * args.steps,
                "roofline": roofline, "clocks": clocks, **extra}
        if nested:
            r.close()
            return line
        print(json.dumps(line), flush=True)
    r.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


# ---------------------------------------------------------------------------
# --form batch: 64 serving requests per graph replay (config 3): one persistent
# launch, or split into a map-build launch and a view launch, as the autotuner picks
# --form bricks: the 512^3 noise field as 2x2x2 bricks, stitched and composited
# ---------------------------------------------------------------------------
BATCH_SIZES = (64, 128, 256, 384)
BATCH_IMAGES = (256, 512, 1024)


def batch_volumes(seed=3):
    """Eight resident volumes: {64, 128, 256, 384}^3 x {blobs, noise}, generated on the device."""
    from pilot_b200 import scenes
    vols = []
    for i, n in enumerate(BATCH_SIZES):
        for kind in ("blobs", "noise"):
            sc = scenes.small(seed + 10 * i + (kind == "noise"), n=n, kind=kind)
            sc.base_freq = 4.0
            vols.append((sc, sc.field_device()))
    return vols


def batch_requests(B, vols, rng, nreq, outs):
    reqs = []
    for i in range(nreq):
        sc, _ = vols[i % len(vols)]
        n = sc.dims[0]
        w = outs[i].shape[1]
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        cam = B.Renderer.camera(tuple(0.5 + d), (0.5, 0.5, 0.5), (0, 1, 0) if abs(d[1]) < 0.9 else (1, 0, 0),
                                30.0, w, w)
        ld = rng.normal(size=3)
        ld /= np.linalg.norm(ld)
        light = tuple(0.5 + 2.0 * np.sqrt(3.0) * ld)
        reqs.append(B.Renderer.request(i % len(vols), cam, light, map_cells=n // 2, sample_distance=0.5 / (n - 1),
                                       termination_alpha=0.99, out=outs[i]))
    return reqs


def run_batch(args, nested=False):
    import torch

    from pilot_b200 import beams as B
    from pilot_b200 import scenes
    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    stream = torch.cuda.current_stream()
    vols = batch_volumes()
    rng = np.random.default_rng(11)
    nreq = args.requests
    sizes = [int(rng.choice(BATCH_IMAGES)) for _ in range(nreq)]
    outs = [torch.empty((w, w, 4), device="cuda") for w in sizes]
    r = B.Renderer(local, stream=stream.cuda_stream)
    r.set_color_map(scenes.tf_table())
    r.batch_set_volumes([(f, sc.origin, sc.spacing, sc.value_range) for sc, f in vols])
    reqs = batch_requests(B, vols, rng, nreq, outs)
    tuning = r.batch_autotune(reqs)
    for _ in range(args.warmup):
        r.render_batch(batch_requests(B, vols, rng, nreq, outs), timings=False)
    torch.cuda.synchronize()
    lit = launches = 0
    sampler = ClockSampler(local)
    with sampler:
        a, z = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(args.steps):  # new cameras and lights every step; the graph is replayed
            _, t = r.render_batch(batch_requests(B, vols, rng, nreq, outs), timings=True)
            lit += t["lit_samples"]
            launches += t["kernel_launches"]
        z.record(stream)
        torch.cuda.synchronize()
    total_ms = a.elapsed_time(z)
    # the other launch plan (one fused launch, or split) with the same options, for comparison
    tuned_opts = {k: tuning[k] for k in ("tile_w", "tile_h", "light_brick", "skip", "split")}
    r.set_batch_options(**dict(tuned_opts, split=not tuning["split"]))
    other_reqs = batch_requests(B, vols, rng, nreq, outs)
    for _ in range(3):
        r.render_batch(other_reqs, timings=False)
    torch.cuda.synchronize()
    a.record(stream)
    for _ in range(args.steps):
        r.render_batch(other_reqs, timings=False)
    z.record(stream)
    torch.cuda.synchronize()
    other_plan = {"split": not tuning["split"], "ms_per_batch": a.elapsed_time(z) / args.steps}
    r.set_batch_options(**tuned_opts)
    # the same requests one render at a time through the single-request API
    singles = []
    for sc, f in vols:
        q = B.Renderer(local, stream=stream.cuda_stream)
        q.set_volume(f, origin=sc.origin, spacing=sc.spacing, value_range=sc.value_range)
        q.set_color_map(scenes.tf_table())
        q.set_termination_alpha(0.99)
        q.set_sample_distance(0.5 / (sc.dims[0] - 1))
        q.set_shadow_map_size(sc.dims[0] // 2)
        singles.append(q)
    seq_reqs = batch_requests(B, vols, rng, nreq, outs)

    def sequential():
        for (rq, o) in seq_reqs:
            q = singles[rq.volume]
            q.clear_lights()
            q.add_point_light(tuple(rq.light), (1, 1, 1), 1.0)
            q.render(rq.camera, out=o, timings=False)
    sequential()
    torch.cuda.synchronize()
    a.record(stream)
    for _ in range(max(1, args.steps // 4)):
        sequential()
    z.record(stream)
    torch.cuda.synchronize()
    seq_ms = a.elapsed_time(z) / max(1, args.steps // 4)
    # The same comparison for small requests only (the 64^3 and 128^3 volumes,
    # 256^2 images), where one request alone cannot fill the GPU.
    small_outs = [torch.empty((256, 256, 4), device="cuda") for _ in range(nreq)]

    def small_requests():
        rq = batch_requests(B, vols, rng, nreq, small_outs)
        for q, _ in rq:
            q.volume = q.volume % 4
            n = vols[q.volume][0].dims[0]
            q.map_cells = n // 2
            q.sample_distance = 0.5 / (n - 1)
        return rq
    small_tuning = r.batch_autotune(small_requests())
    small_reqs = small_requests()
    for _ in range(3):
        r.render_batch(small_reqs, timings=False)
    torch.cuda.synchronize()
    a.record(stream)
    for _ in range(args.steps):
        r.render_batch(small_reqs, timings=False)
    z.record(stream)
    torch.cuda.synchronize()
    small_ms = a.elapsed_time(z) / args.steps
    seq_reqs = small_reqs
    sequential()
    torch.cuda.synchronize()
    a.record(stream)
    for _ in range(max(1, args.steps // 4)):
        sequential()
    z.record(stream)
    torch.cuda.synchronize()
    small_seq_ms = a.elapsed_time(z) / max(1, args.steps // 4)
    r.set_batch_options(**tuned_opts)
    # end to end: images to pinned host memory
    host = [torch.empty((w, w, 4)).pin_memory() for w in sizes]
    r.render_batch(batch_requests(B, vols, rng, nreq, host), timings=False)
    t0 = time.perf_counter()
    ne = max(3, min(args.steps, 10))
    lit_e = 0
    for _ in range(ne):
        _, t = r.render_batch(batch_requests(B, vols, rng, nreq, host), timings=True)
        lit_e += t["lit_samples"]
    e2e_s = time.perf_counter() - t0
    value = lit / (total_ms / 1e3)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded blob and noise volumes generated on the device)",
            "config": {"workload": f"config3: {nreq} requests per step over 8 resident volumes "
                                   f"{{64,128,256,384}}^3 x {{blobs, noise}}, images {{256,512,1024}}^2, M = N/2, "
                                   f"view step 0.5 voxel, alpha cut 0.99, new random camera and point light per "
                                   f"request every step; persistent launches replayed from a CUDA graph "
                                   f"({'map builds, then view marches' if tuning['split'] else 'one fused launch'})",
                       "form": "batch", "tuning": tuning, "parallelism": "1 GPU",
                       "l2": "volumes and maps total well above L2; no flush"},
            "requests_per_s": nreq * args.steps / (total_ms / 1e3),
            "sequential_ms_per_batch": seq_ms, "speedup_vs_sequential": seq_ms / (total_ms / args.steps),
            "other_launch_plan": other_plan,
            "small_requests": {"workload": f"{nreq} requests over the 64^3 and 128^3 volumes, 256^2 images",
                               "batch_ms": small_ms, "sequential_ms": small_seq_ms,
                               "speedup_vs_sequential": small_seq_ms / small_ms, "tuning": small_tuning},
            "gpu_launches": launches,
            "e2e": {"value": lit_e / e2e_s, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": int(sum(w * w * 16 for w in sizes)),
                    "note": "wall clock per batch: host request set-up, graph replay, images to pinned host memory"},
            "clocks": sampler.summary()}
    if nested:
        return line
    print(json.dumps(line), flush=True)
    return 0


def run_bricks(args, nested=False):
    import torch

    from oracle.oracle import psnr
    from pilot_b200 import beams as B
    from pilot_b200 import scenes
    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    stream = torch.cuda.current_stream()
    s = scenes.config1()
    fd = s.field_device()
    cam = s.camera()
    out = torch.empty((s.height, s.width, 4), device="cuda")
    r = B.Renderer(local, stream=stream.cuda_stream)
    r.set_volume(fd, origin=s.origin, spacing=s.spacing, value_range=s.value_range)
    s.configure(r)
    r.render(cam, out=out, timings=False)
    r.autotune(cam)
    whole_ms, _ = time_frames(lambda: r.render(cam, out=out, timings=False), 10, 3, stream, 1, local)
    whole_ms /= 10
    whole = out.cpu().numpy()
    r.set_lazy_shadow_map(True)
    whole_lazy_ms, _ = time_frames(lambda: r.render(cam, out=out, timings=False), 10, 3, stream, 1, local)
    whole_lazy_ms /= 10
    r.set_lazy_shadow_map(False)
    # 2x2x2 bricks; neighbours share their face plane (the reference's blocks)
    nx = s.dims[0]
    cells = nx - 1
    edges = [round(i * cells / 2) for i in range(3)]
    h = s.spacing
    bricks = []
    for z0, z1 in zip(edges[:-1], edges[1:]):
        for y0, y1 in zip(edges[:-1], edges[1:]):
            for x0, x1 in zip(edges[:-1], edges[1:]):
                sub = fd[z0:z1 + 1, y0:y1 + 1, x0:x1 + 1].contiguous()
                org = (s.origin[0] + x0 * h[0], s.origin[1] + y0 * h[1], s.origin[2] + z0 * h[2])
                bricks.append((sub, org, h, s.value_range))
    del fd
    r.set_bricks(bricks)
    s.configure(r)
    r.set_shadow_map_size(s.map_m // 2)  # each brick's map keeps the whole field's vertex spacing
    r.render(cam, out=out, timings=False)  # first frame: brick quads, tables and buffers
    _, tb = r.render(cam, out=out, timings=True)
    img = out.cpu().numpy()
    frame = lambda: r.render(cam, out=out, timings=False)  # noqa: E731
    total_ms, clocks = time_frames(frame, args.steps, args.warmup, stream, 1, local)
    value = tb["lit_samples"] * args.steps / (total_ms / 1e3)
    # the same bricks with the lazy map: only the stitched vertices the view reads
    r.set_lazy_shadow_map(True)
    _, tz = r.render(cam, out=out, timings=True)
    lazy_same = bool(np.array_equal(out.cpu().numpy(), img))
    lazy_ms, _ = time_frames(frame, args.steps, args.warmup, stream, 1, local)
    # a light orbit around the fixed camera: 12 point-light positions 30 degrees
    # apart, full maps, lazy maps, and lazy maps with each brick's marks kept
    lpos0 = np.asarray(s.light, np.float64) - 0.5
    step = [0]

    def orbit_frame():
        a = 2.0 * np.pi * (step[0] % 12) / 12.0
        step[0] += 1
        c, sn = np.cos(a), np.sin(a)
        lp = (0.5 + c * lpos0[0] + sn * lpos0[2], 0.5 + lpos0[1], 0.5 - sn * lpos0[0] + c * lpos0[2])
        r.clear_lights()
        r.add_point_light(tuple(float(v) for v in lp), s.light_color, s.light_intensity)
        r.render(cam, out=out, timings=False)

    orbit = {"frames": "12 light positions around the vertical axis, 30 degrees apart, camera fixed"}
    for mode, name in ((0, "full_maps"), (1, "lazy"), (2, "lazy_kept_marks")):
        r.set_lazy_shadow_map(mode != 0, keep_marks=mode == 2)
        oms, _ = time_frames(orbit_frame, 12, 3, stream, 1, local)
        orbit[name + "_ms_per_frame"] = oms / 12
    r.set_lazy_shadow_map(False)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded 4-octave gradient noise generated on the device)",
            "config": {"workload": "config3 bricks: the 512^3 noise field as 2x2x2 bricks of 256-257 points per axis, "
                                   "1024^2 image, per-brick M = 128; Phase 1 local maps, cross-brick stitch, "
                                   "per-brick view march, depth-ordered composite",
                       "form": "bricks", "parallelism": "1 GPU, 8 bricks", "l2": "inputs larger than L2; no flush"},
            "lit_samples_per_frame": tb["lit_samples"], "gpu_launches": tb["kernel_launches"] * args.steps,
            "phases_ms": {"maps_and_stitch": tb["map_build_ms"], "view_marches": tb["view_march_ms"],
                          "composite": tb["composite_ms"]},
            "undivided_ms_per_frame": whole_ms, "psnr_vs_undivided": psnr(img, whole), "clocks": clocks,
            "lazy_map": {"ms_per_frame": lazy_ms / args.steps, "undivided_ms_per_frame": whole_lazy_ms,
                         "map_vertices_built": tz["map_vertices"], "stitched_map_vertices": tb["map_vertices"],
                         "image_equals_full_maps": lazy_same, "light_orbit": orbit,
                         "phases_ms": {"maps_and_stitch": tz["map_build_ms"], "view_marches": tz["view_march_ms"]}}}
    r.close()
    if nested:
        return line
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# --profile-case: fixed small cases for profiling one kernel at a time (ncu -k):
#   light_march      K1, 512^3 noise, M = 256
#   view_march       K2, 512^3 noise, 1024^2, map cached
#   lazy_frame       exact frame with the lazy map: cell marking, masked K1, K2
#   mlp_view         learned-form view march, 1024^2
#   mlp_frame        learned form frame: scene-light network, 1% probes
#   mlp_frame32      learned form frame: the 32-light network, 1% probes (probe pixels first)
#   mlp_tc           tcgen05 forward, 2^21 rows
#   mlp_train        tcgen05 training steps (2^18 samples, 1 epoch, batches of 16384)
#   batch            16-request persistent batch (--split: map-build launch, then view launch)
#   precision_light  precision-form K1, bf16 640^3
#   precision_view   precision-form K2, bf16 640^3, 1024^2, map cached
#   precision_lazy   precision-form frame with the lazy map, bf16 640^3, 1024^2
#   bricks           512^3 noise as 2x2x2 bricks: K1, K5, K2, K6
#   bricks_lazy      the same with the lazy map (marks and lists before K5)
# Each case sets up its scene, runs the target kernel --reps times and exits 0;
# device memory stays within a few GB. The tuning is fixed (8^3 vertex bricks,
# skipping as stated per case) so that the launch sequence is the same every run.
# ---------------------------------------------------------------------------
PROFILE_CASES = ["light_march", "view_march", "lazy_frame", "mlp_view", "mlp_frame", "mlp_frame32", "mlp_tc", "mlp_train", "batch",
                 "precision_light", "precision_view", "precision_lazy", "bricks", "bricks_lazy"]


def run_profile_case(a):
    import numpy as np
    import torch

    from pilot_b200 import beams as B
    from pilot_b200 import scenes

    torch.cuda.set_device(0)
    if a.profile_case in ("light_march", "view_march", "lazy_frame", "mlp_view", "mlp_frame", "mlp_frame32"):
        s = scenes.config1()
        fd = s.field_device()
        r = B.Renderer(0)
        r.set_volume(fd, origin=s.origin, spacing=s.spacing, value_range=s.value_range)
        s.configure(r)
        r.set_tuning(light_brick=8, empty_skip=False, view_skip=False)
        cam = s.camera()
        out = torch.empty((s.height, s.width, 4), device="cuda")
        if a.profile_case == "light_march":
            for _ in range(a.reps):
                r.build_shadow_map(timings=False)
        elif a.profile_case == "view_march":
            r.build_shadow_map(timings=False)
            r.set_reuse_shadow_map(True)
            for _ in range(a.reps):
                r.render(cam, out=out, timings=False)
        elif a.profile_case == "lazy_frame":
            r.set_lazy_shadow_map(True)
            for _ in range(a.reps):
                r.render(cam, out=out, timings=False)
        elif a.profile_case == "mlp_frame":
            # the learned form as benchmarked: network trained for the scene's light, knot 32, 1% probes
            r.mlp_train(B.mlp_options(n_lights=1, scene_light=1))
            r.set_form(B.FORM_MLP, B.mlp_options(knot=32, probe_fraction=0.01))
            for _ in range(a.reps):
                r.render(cam, out=out, timings=False)
        elif a.profile_case == "mlp_frame32":
            # the network as specified (32 training lights): most tiles fall back, and
            # from the second frame on the probe pixels are marched first
            r.mlp_train(B.mlp_options(n_lights=32))
            r.set_form(B.FORM_MLP, B.mlp_options(knot=32, probe_fraction=0.01))
            for _ in range(a.reps):
                r.render(cam, out=out, timings=True)  # each frame's failing-tile count reaches the host
        else:
            r.mlp_train(B.mlp_options(samples_log2=18, epochs=1, batch=16384))
            r.set_form(B.FORM_MLP, B.mlp_options(knot=4, probe_fraction=0.0))
            for _ in range(a.reps):
                r.render(cam, out=out, timings=False)
    elif a.profile_case == "mlp_train":
        # training steps on the tensor cores on the 512^3 noise field
        s = scenes.config1()
        fd = s.field_device()
        r = B.Renderer(0)
        r.set_volume(fd, origin=s.origin, spacing=s.spacing, value_range=s.value_range)
        s.configure(r)
        r.render(s.camera(), timings=False)
        for _ in range(a.reps):
            r.mlp_train(B.mlp_options(samples_log2=18, epochs=1, batch=16384, n_lights=1, scene_light=1))
    elif a.profile_case == "mlp_tc":
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
    elif a.profile_case in ("precision_light", "precision_view", "precision_lazy"):
        s = scenes.config2(n=640, image=1024, m=320)
        fd = s.field_device()
        r = B.Renderer(0)
        r.set_volume(fd, origin=s.origin, spacing=s.spacing, value_range=s.value_range)
        s.configure(r)
        r.set_form(B.FORM_PRECISION, B.BF16)
        r.set_tuning(light_brick=8, empty_skip=True, view_skip=True)
        if a.profile_case == "precision_light":
            for _ in range(a.reps):
                r.build_shadow_map(timings=False)
        elif a.profile_case == "precision_lazy":
            r.set_lazy_shadow_map(True)
            out = torch.empty((s.height, s.width, 4), device="cuda")
            for _ in range(a.reps):
                r.render(s.camera(), out=out, timings=False)
        else:
            r.build_shadow_map(timings=False)
            r.set_reuse_shadow_map(True)
            out = torch.empty((s.height, s.width, 4), device="cuda")
            for _ in range(a.reps):
                r.render(s.camera(), out=out, timings=False)
    elif a.profile_case in ("bricks", "bricks_lazy"):
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
        r.set_lazy_shadow_map(a.profile_case == "bricks_lazy")
        cam = s.camera()
        out = torch.empty((s.height, s.width, 4), device="cuda")
        for _ in range(a.reps):
            r.render(cam, out=out, timings=False)
    else:  # batch
        vols = batch_volumes()
        rng = np.random.default_rng(11)
        n = 16
        sizes = [int(rng.choice(BATCH_IMAGES)) for _ in range(n)]
        outs = [torch.empty((w, w, 4), device="cuda") for w in sizes]
        r = B.Renderer(0)
        r.set_color_map(scenes.tf_table())
        r.batch_set_volumes([(f, sc.origin, sc.spacing, sc.value_range) for sc, f in vols])
        r.set_batch_options(tile_w=32, tile_h=32, light_brick=8, skip=True, split=a.split)
        reqs = batch_requests(B, vols, rng, n, outs)
        for _ in range(a.reps):
            r.render_batch(reqs, timings=False)
    torch.cuda.synchronize()
    print(f"profile case {a.profile_case}: ok")
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", type=int, default=None, choices=[0, 1, 2])
    ap.add_argument("--form", default="exact", choices=["exact", "precision", "mlp", "batch", "bricks"])
    ap.add_argument("--requests", type=int, default=64, help="batch form: requests per step")
    ap.add_argument("--field-dtype", default="bf16", choices=["bf16", "f16"], help="precision form")
    ap.add_argument("--knot", type=int, default=4, help="mlp form: network every knot lit samples")
    ap.add_argument("--probe-fraction", type=float, default=0.01)
    ap.add_argument("--fallback-tol", type=float, default=0.01)
    ap.add_argument("--mlp-lights", type=int, default=32)
    ap.add_argument("--mlp-scene-light", action="store_true")
    ap.add_argument("--mlp-samples-log2", type=int, default=24)
    ap.add_argument("--mlp-epochs", type=int, default=4)
    ap.add_argument("--no-quality", action="store_true", help="skip the FP64 oracle crops")
    ap.add_argument("--crops", type=int, default=None, help="FP64 crops (default 3; precision form 2)")
    ap.add_argument("--crop", type=int, default=None,
                    help="FP64 crop edge in pixels (default 128; precision form 512, as its config states)")
    ap.add_argument("--crop-stride", type=int, default=1)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="default line: skip the learned-form records")
    ap.add_argument("--no-lazy", action="store_true", help="default line: skip the lazy-map record")
    ap.add_argument("--no-forms", action="store_true",
                    help="default line: skip the precision, batch and bricks records")
    ap.add_argument("--learned-knot", type=int, default=32, help="default line: knot of the learned-form records")
    ap.add_argument("--no-autotune", action="store_true", help="fixed tuning (for launch lists under ncu)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=12.0, help="seconds of CPU work for cpu_baseline")
    ap.add_argument("--no-full-frame", action="store_true",
                    help="CPU legs: skip the whole-frame oracle run that checks the sample's extrapolation")
    ap.add_argument("--profile-case", default=None, choices=PROFILE_CASES,
                    help="run one fixed small case for a kernel profile (see PROFILE_CASES) and exit")
    ap.add_argument("--reps", type=int, default=3, help="--profile-case: repetitions of the target kernel")
    ap.add_argument("--split", action="store_true", help="--profile-case batch: split launch plan")
    args = ap.parse_args()
    if args.profile_case:
        return run_profile_case(args)
    args.warmup = max(3, args.warmup)  # at least 3 untimed warm-up frames
    if args.config is None:
        args.config = 2 if args.form == "precision" else 1
    if args.crop is None:
        args.crop = 512 if args.form == "precision" else 128
    if args.crops is None:
        args.crops = 2 if args.form == "precision" else 3
    if args.impl == "reference":
        return run_reference(args)
    if args.form == "batch":
        return run_batch(args)
    if args.form == "bricks":
        return run_bricks(args)
    if args.form != "exact":
        return run_form(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
