"""Batched form against the oracle directly, on requests shaped like the batching
workload: resident volumes of 64^3, 128^3 and 384^3 (blobs and gradient noise),
images of 256^2, 512^2 and a 1024^2 image checked on a crop, map size N/2,
step 0.5 voxel, alpha cut 0.99, a random camera on the unit sphere around the
centre and a random light per request.

Bars (the exact form's): every request's image within max |dRGBA| <= 2e-3 of
the oracle's f32 march on the oracle's f32 map of the same request, >= 99.9% of
pixels bit-identical; the batch's lit-sample count equals the oracle's over
the full images. Both launch plans (one persistent launch, and the split plan)
are checked.
"""
import numpy as np
import pytest
import torch

from oracle.oracle import Oracle
from pilot_b200 import beams as B
from pilot_b200 import scenes

pytestmark = pytest.mark.gpu
TOL = 2e-3

# (volume size, kind, seed); the fields are generated on the device, as the
# batch workload does, and read back for the oracle
VOLUMES = [(64, "blobs", 3), (128, "noise", 14), (384, "noise", 34)]
# (volume index, image size, crop window or None, light kind)
REQUESTS = [(0, 256, None, 0), (1, 512, None, 0), (2, 512, None, 0), (1, 1024, (416, 416, 192, 192), 1),
            (0, 512, None, 1), (2, 256, None, 0)]


def _volumes():
    out = []
    for n, kind, seed in VOLUMES:
        sc = scenes.small(seed, n=n, kind=kind)
        sc.base_freq = 4.0
        fd = sc.field_device()
        torch.cuda.synchronize()
        sc.array = fd.cpu().numpy()
        out.append((sc, fd))
    return out


def _request_scene(sc, image, light_kind, rng):
    """The request as a scene for the oracle, plus its batch request arguments."""
    n = sc.dims[0]
    d = rng.normal(size=3)
    d /= np.linalg.norm(d)
    up = (0.0, 1.0, 0.0) if abs(d[1]) < 0.9 else (1.0, 0.0, 0.0)
    ld = rng.normal(size=3)
    ld /= np.linalg.norm(ld)
    light = tuple(float(x) for x in ld) if light_kind == 1 else \
        tuple(float(x) for x in 0.5 + 2.0 * np.sqrt(3.0) * ld)
    rs = scenes.Scene(name=f"req{n}", dims=sc.dims, kind=sc.kind, params=sc.params, tf=sc.tf,
                      light_kind=light_kind, light=light, map_m=n // 2, sample_distance=0.5 / (n - 1),
                      cutoff=0.99, cam_pos=tuple(float(x) for x in 0.5 + d), cam_up=up, width=image,
                      height=image, array=sc.array)
    return rs


@pytest.mark.parametrize("split", [False, True], ids=["one-launch", "split"])
def test_batch_matches_oracle_on_mixed_requests(cuda_device, split):
    vols = _volumes()
    rng = np.random.default_rng(77)
    tf = scenes.tf_table()
    with B.Renderer(0) as r:
        r.set_color_map(tf)
        r.batch_set_volumes([(fd, sc.origin, sc.spacing, sc.value_range) for sc, fd in vols])
        r.set_batch_options(tile_w=32, tile_h=32, light_brick=8, use_graph=True, split=split)
        reqs, rscenes = [], []
        for vi, image, crop, lk in REQUESTS:
            rs = _request_scene(vols[vi][0], image, lk, rng)
            out = torch.zeros((image, image, 4), device="cuda")
            reqs.append(B.Renderer.request(vi, rs.camera(), rs.light, light_kind=lk, map_cells=rs.map_m,
                                           sample_distance=rs.sample_distance, termination_alpha=rs.cutoff,
                                           out=out))
            rscenes.append((rs, crop))
        outs, t = r.render_batch(reqs)
        torch.cuda.synchronize()
    lit_full = 0
    for (rs, crop), out in zip(rscenes, outs):
        o = Oracle(rs)
        om, _ = o.light_march()
        img = out.cpu().numpy()
        if crop is None:
            oimg, lit = o.view_march(om)
            got = img
            lit_full += lit
        else:
            x0, y0, w, h = crop
            oimg, _ = o.view_march(om, window=crop)
            got = img[y0:y0 + h, x0:x0 + w]
        err = float(np.abs(got - oimg).max())
        same = float(np.mean(np.all(got == oimg, axis=-1)))
        print(f"{rs.name} {rs.width}^2 crop={crop}: max|d| {err:.2e}, identical {same:.5f}")
        assert err <= TOL, f"{rs.name} {rs.width}^2: max |d| {err}"
        assert same >= 0.999, f"{rs.name} {rs.width}^2: {same:.5f} bit-identical"
    # the crop request's lit samples are counted by the batch but not by the crop
    crop_reqs = [i for i, (_, c) in enumerate(rscenes) if c is not None]
    extra = 0
    for i in crop_reqs:
        rs, _ = rscenes[i]
        o = Oracle(rs)
        _, lit = o.view_march(o.light_march()[0])
        extra += lit
    assert t["lit_samples"] == lit_full + extra
