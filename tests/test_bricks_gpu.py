"""Multi-block scenes on one GPU: Phase 1 local maps, the cross-brick shadow
stitch (K5, the reference's Phases 2-3), per-brick view marches and the
depth-ordered composite (K6, the reference's GlobalComposite), against the
oracle's multi-block restatement. Tolerance: maps bit-exact, image max
|dRGBA| <= 2e-3 (expected bit-exact)."""
import numpy as np
import pytest

from oracle.oracle import Oracle, psnr, render_bricks
from pilot_b200 import beams as B
from pilot_b200 import scenes

pytestmark = pytest.mark.gpu
TOL = 2e-3


def shell_mask(pd):
    """Vertices (x fastest) with an index in {0, 1, pd-2, pd-1} on some axis."""
    i = np.arange(pd)
    edge = (i <= 1) | (i >= pd - 2)
    return (edge[:, None, None] | edge[None, :, None] | edge[None, None, :]).ravel()


def gpu_bricks(bricks):
    r = B.Renderer(0)
    r.set_bricks([(b.field_numpy(), b.origin, b.spacing, b.value_range) for b in bricks])
    bricks[0].configure(r)
    img, t = r.render(bricks[0].camera())
    return r, img, t


@pytest.mark.parametrize("kind,light_kind,splits", [("blobs", 0, (2, 2, 2)), ("noise", 1, (2, 2, 2)),
                                                      ("blobs", 0, (3, 1, 2))])
def test_bricks_match_oracle(cuda_device, kind, light_kind, splits):
    s = scenes.small(31, n=41, image=80, m=12, kind=kind, light_kind=light_kind)
    bricks = scenes.split_bricks(s, splits)
    r, img, t = gpu_bricks(bricks)
    orgba, _, olocal, ofinal, olit = render_bricks(bricks)
    for i, b in enumerate(bricks):
        nv = (b.map_m + 1) ** 3
        # Phase 1 builds the vertices the stitch reads: those within one layer of a brick face
        shell = shell_mask(b.map_m + 1)
        assert np.array_equal(r.get_brick_map(i, 0, nv)[shell], np.asarray(olocal[i]).ravel()[shell]), \
            f"brick {i} local map"
        assert np.array_equal(r.get_brick_map(i, 1, nv), ofinal[i]), f"brick {i} stitched map"
    err = np.abs(img - orgba)
    assert err.max() <= TOL and np.mean(np.all(img == orgba, axis=-1)) > 0.999
    assert t["lit_samples"] == olit
    # stitching darkens: every stitched vertex is at least as opaque as its local march
    for i, b in enumerate(bricks):
        assert np.all(ofinal[i] >= olocal[i] - 1e-6)


def test_one_brick_equals_single_volume(cuda_device):
    s = scenes.small(32, n=33, image=64, m=16)
    r, img, _ = gpu_bricks(scenes.split_bricks(s, (1, 1, 1)))
    with B.Renderer(0) as q:
        q.set_volume(s.field_numpy(), origin=s.origin, spacing=s.spacing, value_range=s.value_range)
        s.configure(q)
        ref, _ = q.render(s.camera())
    assert np.array_equal(img, ref)


def test_bricks_approximate_the_undivided_volume(cuda_device):
    s = scenes.small(33, n=65, image=96, m=32, kind="blobs")
    r, img, _ = gpu_bricks(scenes.split_bricks(s, (2, 2, 2)))
    full, _ = Oracle(s).view_march(None)
    p = psnr(img, full)
    print(f"2x2x2 bricks vs undivided volume: PSNR {p:.1f} dB")
    assert p > 25


def test_repeated_brick_frames_are_identical(cuda_device):
    """Each phase's brick launches run on side streams with per-brick counters:
    a second frame on the same renderer starts from zeroed counters and gives
    the same image and counts, also after the bricks are replaced."""
    s = scenes.small(34, n=41, image=72, m=12, kind="noise")
    bricks = scenes.split_bricks(s, (2, 2, 2))
    r, img, t = gpu_bricks(bricks)
    img2, t2 = r.render(bricks[0].camera())
    assert np.array_equal(img, img2)
    assert (t2["lit_samples"], t2["light_samples"]) == (t["lit_samples"], t["light_samples"])
    # the first frame also builds every brick's quads and cell tables (two launches per brick)
    assert t2["kernel_launches"] == t["kernel_launches"] - 2 * len(bricks)
    five = scenes.split_bricks(s, (5, 1, 1))
    r.set_bricks([(b.field_numpy(), b.origin, b.spacing, b.value_range) for b in five])
    img5, t5 = r.render(five[0].camera())
    orgba, _, _, _, olit = render_bricks(five)
    assert np.abs(img5 - orgba).max() <= TOL and t5["lit_samples"] == olit


@pytest.mark.parametrize("splits,fov", [((2, 2, 2), 30.0), ((3, 1, 2), 30.0), ((2, 2, 2), 8.0)])
def test_lazy_map_bricks_give_the_full_maps_image(cuda_device, splits, fov):
    """beams_set_lazy_shadow_map in a multi-block scene: each brick's view rays
    mark the cells of its stitched map they read and only their corners are
    stitched; a brick no pixel reaches stitches nothing. The lazy frame follows
    a frame under another light, so a vertex skipped but read would show."""
    s = scenes.small(35, n=41, image=80, m=12, kind="noise", light_kind=0)
    s.fov_y_deg = fov
    bricks = scenes.split_bricks(s, splits)
    for b in bricks:
        b.fov_y_deg = fov
    cam = bricks[0].camera()
    r, img, t = gpu_bricks(bricks)
    r.clear_lights()
    r.add_directional_light((0.3, 0.9, -0.3), (1.0, 0.2, 0.2), 1.0)
    r.render(cam)
    bricks[0].configure(r)
    r.set_lazy_shadow_map(True)
    lazy, tl = r.render(cam)
    assert np.array_equal(lazy, img), f"lazy brick frame differs by {np.max(np.abs(lazy - img))}"
    assert tl["lit_samples"] == t["lit_samples"]
    assert 0 < tl["map_vertices"] < t["map_vertices"]
    nv = (bricks[0].map_m + 1) ** 3
    with pytest.raises(B.BeamsError):
        r.get_brick_map(0, 1, nv)  # the stitched map is partial
    r.set_lazy_shadow_map(False)
    again, _ = r.render(cam)
    assert np.array_equal(again, img)
    assert r.get_brick_map(0, 1, nv).size == nv
    print(f"{splits} fov {fov}: {tl['map_vertices']} vertices built, full stitched maps {t['map_vertices']}")


def test_kept_brick_marks_over_a_light_orbit(cuda_device):
    """Mode 2 in a multi-block scene: each brick keeps its marks while the view
    is unchanged, so a moving light re-marks no brick (one launch fewer per
    brick the view reaches) and every frame equals the full stitched maps'."""
    s = scenes.small(36, n=41, image=72, m=12, kind="noise", light_kind=1)
    bricks = scenes.split_bricks(s, (2, 2, 2))
    cam = bricks[0].camera()
    r, _, _ = gpu_bricks(bricks)
    q, _, _ = gpu_bricks(bricks)
    r.set_lazy_shadow_map(True, keep_marks=True)
    counts = []
    for d in [(0.2, 0.9, 0.3), (-0.7, 0.1, 0.7), (0.5, -0.5, -0.7), (0.1, 0.2, -0.97)]:
        for x in (r, q):
            x.clear_lights()
            x.add_directional_light(d, (1.0, 0.9, 0.8), 1.2)
        a, ta = r.render(cam)
        b, tb = q.render(cam)
        assert np.array_equal(a, b), f"light {d}: differs by {np.max(np.abs(a - b))}"
        assert ta["lit_samples"] == tb["lit_samples"]
        counts.append(ta["kernel_launches"])
    assert counts[1] < counts[0] and counts[1] == counts[2] == counts[3]  # marked once
    cam2 = scenes.split_bricks(scenes.small(37, n=41, image=72, m=12, kind="noise"), (2, 2, 2))[0].camera()
    a, ta = r.render(cam2)  # a new view marks again
    b, _ = q.render(cam2)
    assert np.array_equal(a, b)
