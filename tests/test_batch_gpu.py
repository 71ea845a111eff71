"""Batched form: many requests (own volume, camera, light, map size) in one
persistent launch replayed from a CUDA graph (or, split, one launch of map
builds and one of view marches); every image equals the single-request exact
render bit for bit."""
import numpy as np
import pytest
import torch

from pilot_b200 import beams as B
from pilot_b200 import scenes

pytestmark = pytest.mark.gpu


def _volumes():
    vs = []
    for seed, n, kind in ((1, 24, "blobs"), (2, 33, "noise"), (3, 40, "blobs")):
        s = scenes.small(seed, n=n, kind=kind)
        vs.append(s)
    return vs


def _requests(vols, rng, device_out):
    reqs, specs = [], []
    sizes = [(40, 32), (64, 64), (17, 23), (48, 40)]
    for i in range(9):
        vi = i % len(vols)
        s = vols[vi]
        w, h = sizes[i % len(sizes)]
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        cam = B.Renderer.camera(tuple(0.5 + 1.6 * d), (0.5, 0.5, 0.5), (0, 1, 0) if abs(d[1]) < 0.9 else (1, 0, 0),
                                30.0, w, h)
        ld = rng.normal(size=3)
        ld /= np.linalg.norm(ld)
        kind = i % 2
        light = tuple(ld) if kind == 1 else tuple(0.5 + 3.5 * ld)
        spec = dict(volume=vi, camera=cam, light=light, light_kind=kind, light_color=(1.0, 0.9, 0.8),
                    light_intensity=1.2, map_cells=(8, 12, 16)[i % 3],
                    sample_distance=(-1.0, 0.5 / (s.dims[0] - 1))[i % 2], termination_alpha=(1.0, 0.97)[i % 2])
        out = torch.zeros((h, w, 4), device="cuda") if (device_out and i % 3 != 1) else None
        reqs.append(B.Renderer.request(out=out, **spec))
        specs.append(spec)
    return reqs, specs


def _single(s, tf, spec):
    with B.Renderer(0) as r:
        r.set_volume(s.field_numpy(), origin=s.origin, spacing=s.spacing, value_range=s.value_range)
        r.set_color_map(tf)
        r.set_shadow_map_size(spec["map_cells"])
        if spec["light_kind"] == 0:
            r.add_point_light(spec["light"], spec["light_color"], spec["light_intensity"])
        else:
            r.add_directional_light(spec["light"], spec["light_color"], spec["light_intensity"])
        if spec["sample_distance"] > 0:
            r.set_sample_distance(spec["sample_distance"])
        r.set_termination_alpha(spec["termination_alpha"])
        img, t = r.render(spec["camera"])
    return img, t


def _as_np(o):
    return o if isinstance(o, np.ndarray) else o.cpu().numpy()


@pytest.mark.parametrize("opts", [dict(tile_w=16, tile_h=16, light_brick=8, use_graph=True),
                                  dict(tile_w=32, tile_h=8, light_brick=0, use_graph=True, skip=False),
                                  dict(tile_w=8, tile_h=32, light_brick=16, use_graph=False),
                                  dict(tile_w=32, tile_h=32, light_brick=64, use_graph=True, skip=False),
                                  dict(tile_w=64, tile_h=64, light_brick=32, use_graph=True),
                                  dict(tile_w=32, tile_h=32, light_brick=8, use_graph=True, split=True),
                                  dict(tile_w=16, tile_h=8, light_brick=0, use_graph=False, skip=False, split=True)])
def test_batch_equals_single_renders(cuda_device, opts):
    vols = _volumes()
    tf = scenes.tf_table()
    rng = np.random.default_rng(5)
    with B.Renderer(0) as r:
        r.set_color_map(tf)
        r.batch_set_volumes([(s.field_numpy(), s.origin, s.spacing, s.value_range) for s in vols])
        r.set_batch_options(**opts)
        for call in range(3):  # the graph is captured on the first call and replayed with new cameras
            reqs, specs = _requests(vols, rng, device_out=True)
            outs, t = r.render_batch(reqs)
            lit = 0
            for o, spec in zip(outs, specs):
                ref, ts = _single(vols[spec["volume"]], tf, spec)
                assert np.array_equal(_as_np(o), ref), (call, spec["volume"], opts)
                lit += ts["lit_samples"]
            assert t["lit_samples"] == lit and t["kernel_launches"] == (2 if opts.get("split") else 1)


def test_batch_rejects_bad_requests(cuda_device):
    vols = _volumes()
    with B.Renderer(0) as r:
        r.set_color_map(scenes.tf_table())
        with pytest.raises(B.BeamsError):
            r.render_batch([B.Renderer.request(0, B.Renderer.camera((0.5, 0.5, 2), (0.5, 0.5, 0.5), (0, 1, 0), 30, 8, 8),
                                               (1, 1, 1))])
        r.batch_set_volumes([(s.field_numpy(), s.origin, s.spacing, s.value_range) for s in vols])
        cam = B.Renderer.camera((0.5, 0.5, 2), (0.5, 0.5, 0.5), (0, 1, 0), 30, 8, 8)
        with pytest.raises(B.BeamsError):
            r.render_batch([B.Renderer.request(7, cam, (1, 1, 1))])
        with pytest.raises(B.BeamsError):
            r.render_batch([B.Renderer.request(0, cam, (1, 1, 1), map_cells=0)])
        with pytest.raises(B.BeamsError):
            r.set_batch_options(tile_w=12, tile_h=8)
        outs, _ = r.render_batch([B.Renderer.request(0, cam, (1, 1, 1))])
        assert outs[0].shape == (8, 8, 4)


def test_batch_autotune_keeps_images(cuda_device):
    vols = _volumes()
    tf = scenes.tf_table()
    rng = np.random.default_rng(9)
    with B.Renderer(0) as r:
        r.set_color_map(tf)
        r.batch_set_volumes([(s.field_numpy(), s.origin, s.spacing, s.value_range) for s in vols])
        reqs, specs = _requests(vols, rng, device_out=False)
        best = r.batch_autotune(reqs)
        # view tiles are whole 8x4 warp tiles
        assert best["tile_w"] % 8 == 0 and best["tile_h"] % 4 == 0 and best["batch_ms"] > 0
        outs, _ = r.render_batch(reqs)
        for o, spec in zip(outs, specs):
            ref, _ = _single(vols[spec["volume"]], tf, spec)
            assert np.array_equal(_as_np(o), ref)


def test_batch_tuning_cache_and_file(cuda_device, tmp_path):
    """The autotuner keeps its result per batch shape: the same shape with new
    cameras and lights is answered from the cache (no timing runs), and a saved
    cache file lets another renderer skip tuning too."""
    import time
    vols = _volumes()
    tf = scenes.tf_table()
    rng = np.random.default_rng(12)
    with B.Renderer(0) as r:
        r.set_color_map(tf)
        r.batch_set_volumes([(s.field_numpy(), s.origin, s.spacing, s.value_range) for s in vols])
        reqs, _ = _requests(vols, rng, device_out=False)
        t0 = time.perf_counter()
        first = r.batch_autotune(reqs)
        t_tune = time.perf_counter() - t0
        reqs2, _ = _requests(vols, rng, device_out=False)  # same shapes, new cameras and lights
        t0 = time.perf_counter()
        again = r.batch_autotune(reqs2)
        t_hit = time.perf_counter() - t0
        assert again == first and t_hit < t_tune / 5
        path = tmp_path / "tuning.txt"
        r.batch_tuning_save(path)
        r.batch_tuning_clear()
    with B.Renderer(0) as q:
        q.set_color_map(tf)
        q.batch_set_volumes([(s.field_numpy(), s.origin, s.spacing, s.value_range) for s in vols])
        q.batch_tuning_load(path)
        t0 = time.perf_counter()
        loaded = q.batch_autotune(reqs2)
        assert time.perf_counter() - t0 < t_tune / 5
        keys = ("tile_w", "tile_h", "light_brick", "skip", "split")
        assert {k: loaded[k] for k in keys} == {k: first[k] for k in keys}
        bad = tmp_path / "bad.txt"
        bad.write_text("beams-batch-tuning 2\nkey 7 4 8 0 0 1.0\n")
        with pytest.raises(B.BeamsError):
            q.batch_tuning_load(bad)
        bad.write_text("beams-batch-tuning 2\nkey 8 4 8 0 2 1.0\n")
        with pytest.raises(B.BeamsError):
            q.batch_tuning_load(bad)
        # a format-1 file (no split column) still loads, as one launch
        old = tmp_path / "v1.txt"
        key = path.read_text().splitlines()[1].split()[0]
        old.write_text(f"beams-batch-tuning 1\n{key} 16 8 0 1 2.5\n")
        q.batch_tuning_clear()
        q.batch_tuning_load(old)
        got = q.batch_autotune(reqs2)
        assert (got["tile_w"], got["tile_h"], got["light_brick"], got["skip"], got["split"]) == (16, 8, 0, False, False)
