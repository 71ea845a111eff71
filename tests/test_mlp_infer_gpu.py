"""Learned form, render side: the fused tensor-core view march against the
float64 network applied to the oracle's lit samples, knot interpolation, and
the trained network's gain over rendering without a shadow model."""
import numpy as np
import pytest

from oracle import mlp_oracle as M
from oracle.oracle import Oracle, psnr
from pilot_b200 import beams as B
from pilot_b200 import scenes

pytestmark = pytest.mark.gpu


def light_feature(s):
    c = np.array([0.5 * (0 + (s.dims[i] - 1) * s.spacing[i]) for i in range(3)])
    v = np.array(s.light, np.float64) - c if s.light_kind == 0 else -np.array(s.light, np.float64)
    return v / np.linalg.norm(v)


def oracle_mlp_image(s, P):
    """The float64 network shading the oracle's lit samples, composited in order."""
    o = Oracle(s)
    rec, cnt = o.record_samples()
    hi = np.array([(s.dims[i] - 1) * s.spacing[i] for i in range(3)])
    X = M.encode(rec[:, :3], np.repeat(light_feature(s)[None, :], rec.shape[0], 0), (0, 0, 0), hi)
    _, _, T = M.forward_backward(P, M.bf16(X), np.zeros(rec.shape[0]))
    lc = np.float32(s.light_intensity) * np.array(s.light_color, np.float32)
    img = np.zeros((s.height, s.width, 4), np.float32)
    k = 0
    for yy in range(s.height):
        for xx in range(s.width):
            c = np.zeros(4, np.float32)
            for _ in range(cnt[yy, xx]):
                r = rec[k]
                t = np.float32(T[k])
                for ch in range(3):
                    c[ch] = c[ch] + np.float32(min(max(r[3 + ch] * (t * lc[ch]), 0.0), 1.0)) * r[6]
                c[3] = r[6] + c[3]
                k += 1
            img[yy, xx] = c
    return img


def mlp_render(s, P=None, knot=1, r=None, probe_fraction=0.0):
    if r is None:
        r = B.Renderer(0)
        r.set_volume(s.field_numpy(), origin=s.origin, spacing=s.spacing, value_range=s.value_range)
        s.configure(r)
    if P is not None:
        r.mlp_set_params(P)
    r.set_form(B.FORM_MLP, B.mlp_options(knot=knot, probe_fraction=probe_fraction))
    img, t = r.render(s.camera())
    return img, t, r


def smooth_params(seed=7):
    rng = np.random.default_rng(seed)
    P = rng.normal(0, 0.08, M.N_PARAMS).astype(np.float32)
    P[M.OFF["B5"][0]] = 0.5
    return P


def test_mlp_render_matches_float64_network(cuda_device):
    s = scenes.small(61, n=32, image=40, m=8, kind="blobs")
    P = smooth_params()
    img, t, _ = mlp_render(s, P, knot=1)
    ref = oracle_mlp_image(s, P)
    err = np.abs(img - ref)
    print(f"mlp render vs float64 network: max {err.max():.2e} mean {err.mean():.2e}; "
          f"evals {t['mlp_samples']} lit {t['lit_samples']}")
    assert t["map_vertices"] == 0 and t["mlp_samples"] == t["lit_samples"]
    assert err.max() < 1e-2 and err.mean() < 1e-3
    # alpha does not depend on the shading: identical to the exact path's
    with B.Renderer(0) as q:
        q.set_volume(s.field_numpy(), origin=s.origin, spacing=s.spacing, value_range=s.value_range)
        s.configure(q)
        exact, _ = q.render(s.camera())
    assert np.array_equal(img[..., 3], exact[..., 3])


def test_mlp_knot_interpolation_close_to_every_sample(cuda_device):
    s = scenes.small(62, n=40, image=64, m=8, kind="noise")
    P = smooth_params(8)
    i1, t1, r = mlp_render(s, P, knot=1)
    i4, t4, _ = mlp_render(s, None, knot=4, r=r)
    p = psnr(i1, i4)
    print(f"knot 4 vs knot 1: PSNR {p:.1f} dB, evaluations {t4['mlp_samples']} vs {t1['mlp_samples']}")
    assert t4["mlp_samples"] < 0.4 * t1["mlp_samples"] and p > 40
    for k in (16, 32, 64):
        ik, tk, _ = mlp_render(s, None, knot=k, r=r)
        pk = psnr(i1, ik)
        print(f"knot {k} vs knot 1: PSNR {pk:.1f} dB, evaluations {tk['mlp_samples']}")
        assert np.array_equal(ik[..., 3], i1[..., 3]) and tk["mlp_samples"] < t4["mlp_samples"] and pk > 30


def test_trained_mlp_render_beats_no_shadow_model(cuda_device):
    s = scenes.small(63, n=48, image=64, m=24, kind="blobs", light_kind=0)
    r = B.Renderer(0)
    r.set_volume(s.field_numpy(), origin=s.origin, spacing=s.spacing, value_range=s.value_range)
    s.configure(r)
    rep = r.mlp_train(B.mlp_options(samples_log2=18, epochs=8, batch=2048, lr=3e-3))
    img, t, _ = mlp_render(s, None, knot=2, r=r)
    o = Oracle(s)
    ref64, _ = o.view_march(o.light_march(fp64=True)[0], fp64=True)
    s2 = scenes.small(63, n=48, image=64, m=24, kind="blobs", light_kind=0)
    s2.use_map = False
    unlit, _ = Oracle(s2).view_march(None)
    p_mlp, p_unlit = psnr(img, ref64), psnr(unlit, ref64)
    print(f"trained MLP (holdout rmse {rep['holdout_rmse']:.3f}): PSNR {p_mlp:.1f} dB vs unshadowed {p_unlit:.1f} dB")
    assert p_mlp > p_unlit + 3


# ---- per-tile fallback to the exact map -------------------------------------------
TILE = 32


def _renderer(s):
    r = B.Renderer(0)
    r.set_volume(s.field_numpy(), origin=s.origin, spacing=s.spacing, value_range=s.value_range)
    s.configure(r)
    return r


def _tile_max(err, h, w):
    ty, tx = -(-h // TILE), -(-w // TILE)
    out = np.full((ty, tx), -np.inf)
    for y in range(h):
        for x in range(w):
            out[y // TILE, x // TILE] = max(out[y // TILE, x // TILE], err[y, x])
    return out


def _probe_errors_cpu(s, mlp_img):
    """Every pixel composited with the exact light march's transmittance (float32
    oracle), against the network's image: max |dRGBA| per pixel."""
    o = Oracle(s)
    rec, cnt = o.record_samples()
    T = (np.float32(1) - o.point_opacity(rec[:, :3], fp64=False)).astype(np.float32)
    lc = np.float32(s.light_intensity) * np.array(s.light_color, np.float32)
    err = np.zeros((s.height, s.width), np.float32)
    k = 0
    for y in range(s.height):
        for x in range(s.width):
            c = np.zeros(4, np.float32)
            for _ in range(cnt[y, x]):
                r = rec[k]
                for ch in range(3):
                    c[ch] = c[ch] + np.float32(min(max(r[3 + ch] * (T[k] * lc[ch]), 0.0), 1.0)) * r[6]
                c[3] = r[6] + c[3]
                k += 1
            err[y, x] = np.abs(mlp_img[y, x] - c).max()
    return err


def _check_tiles(img, mlp_img, exact_img, flagged):
    h, w = img.shape[:2]
    for ty in range(flagged.shape[0]):
        for tx in range(flagged.shape[1]):
            sl = (slice(ty * TILE, min(h, (ty + 1) * TILE)), slice(tx * TILE, min(w, (tx + 1) * TILE)))
            want = exact_img if flagged[ty, tx] else mlp_img
            assert np.array_equal(img[sl], want[sl]), (ty, tx, bool(flagged[ty, tx]))


def test_mlp_fallback_every_pixel_probed(cuda_device):
    """probe_fraction 1: the device's probe errors equal the oracle's exact
    transmittance composite, and exactly the tiles above the tolerance carry
    the exact form's pixels."""
    s = scenes.small(64, n=32, image=72, m=8, kind="blobs")
    r = _renderer(s)
    exact_img, _ = r.render(s.camera())
    r.mlp_set_params(smooth_params(9))
    r.set_form(B.FORM_MLP, B.mlp_options(knot=2, probe_fraction=0.0))
    mlp_img, _ = r.render(s.camera())
    cpu_err = _probe_errors_cpu(s, mlp_img)
    tiles = _tile_max(cpu_err, s.height, s.width)
    tol = float(np.median(tiles))
    r.set_form(B.FORM_MLP, B.mlp_options(knot=2, probe_fraction=1.0, fallback_tol=tol))
    img, t = r.render(s.camera())
    gpu_err = r.mlp_probe_errors(s.width * s.height).reshape(s.height, s.width)
    assert np.array_equal(gpu_err, cpu_err), np.abs(gpu_err - cpu_err).max()
    flagged = tiles > tol
    print(f"tol {tol:.4f}: {flagged.sum()} of {flagged.size} tiles fall back")
    assert 0 < flagged.sum() < flagged.size and t["fallback_tiles"] == flagged.sum()
    # the lazy fallback builds only the map vertices the failing tiles' rays read
    assert 0 < t["map_vertices"] <= (s.map_m + 1) ** 3
    _check_tiles(img, mlp_img, exact_img, flagged)
    # a tolerance above every error keeps the network's image and builds no map
    r.set_form(B.FORM_MLP, B.mlp_options(knot=2, probe_fraction=1.0, fallback_tol=1e30))
    img2, t2 = r.render(s.camera())
    assert t2["fallback_tiles"] == 0 and t2["map_vertices"] == 0 and t2["light_samples"] == 0
    assert np.array_equal(img2, mlp_img)
    # tolerance 0 with a network far from the map: every tile with a visible probe falls back
    r.set_form(B.FORM_MLP, B.mlp_options(knot=2, probe_fraction=1.0, fallback_tol=0.0))
    img3, t3 = r.render(s.camera())
    _check_tiles(img3, mlp_img, exact_img, tiles > 0)


def test_mlp_fallback_one_percent_probes(cuda_device):
    s = scenes.small(65, n=40, image=96, m=10, kind="noise")
    r = _renderer(s)
    exact_img, _ = r.render(s.camera())
    r.mlp_set_params(smooth_params(10))
    r.set_form(B.FORM_MLP, B.mlp_options(knot=4, probe_fraction=0.0))
    mlp_img, _ = r.render(s.camera())
    r.set_form(B.FORM_MLP, B.mlp_options(knot=4, probe_fraction=0.01, fallback_tol=0.05))
    img, t = r.render(s.camera())
    P = 10
    n = len(range(P // 2, s.width, P))
    err = r.mlp_probe_errors(n * n).reshape(n, n)
    cpu = _probe_errors_cpu(s, mlp_img)[P // 2::P, P // 2::P]
    assert np.array_equal(err, cpu)
    tiles = np.full((3, 3), -np.inf)
    for j in range(n):
        for i in range(n):
            y, x = j * P + P // 2, i * P + P // 2
            tiles[y // TILE, x // TILE] = max(tiles[y // TILE, x // TILE], err[j, i])
    assert t["fallback_tiles"] == (tiles > 0.05).sum()
    _check_tiles(img, mlp_img, exact_img, tiles > 0.05)
    tol = float(np.median(tiles))
    r.set_form(B.FORM_MLP, B.mlp_options(knot=4, probe_fraction=0.01, fallback_tol=tol))
    img, t = r.render(s.camera())
    flagged = tiles > tol
    print(f"1% probes, tol {tol:.3f}: {flagged.sum()} of 9 tiles fall back; probe errors max {err.max():.3f}")
    assert 0 < flagged.sum() < 9 and t["fallback_tiles"] == flagged.sum()
    _check_tiles(img, mlp_img, exact_img, flagged)


def test_mlp_lazy_fallback_builds_only_the_failing_tiles_vertices(cuda_device):
    """A few failing tiles of a 256^2 image over a 64-cell map: the fallback
    marks and marches only the map vertices those tiles' view rays read, far
    fewer than the whole map, and the tiles still carry the exact form's pixels
    bit for bit (every vertex they read was built)."""
    s = scenes.small(66, n=48, image=256, m=64, kind="noise")
    r = _renderer(s)
    exact_img, te = r.render(s.camera())
    r.mlp_set_params(smooth_params(11))
    r.set_form(B.FORM_MLP, B.mlp_options(knot=2, probe_fraction=0.0))
    mlp_img, _ = r.render(s.camera())
    full = (s.map_m + 1) ** 3
    P = 4  # probe fraction 1/16: probes at (4i + 2, 4j + 2)
    n = len(range(P // 2, s.width, P))
    for q in (0.9, 0.5):
        r.set_form(B.FORM_MLP, B.mlp_options(knot=2, probe_fraction=1.0 / 16, fallback_tol=1e30))
        r.render(s.camera())
        err = r.mlp_probe_errors(n * n).reshape(n, n)
        nt = -(-s.width // TILE)
        tiles = np.full((nt, nt), -np.inf)
        for j in range(n):
            for i in range(n):
                y, x = j * P + P // 2, i * P + P // 2
                tiles[y // TILE, x // TILE] = max(tiles[y // TILE, x // TILE], err[j, i])
        tol = float(np.quantile(tiles[np.isfinite(tiles)], q))
        r.set_form(B.FORM_MLP, B.mlp_options(knot=2, probe_fraction=1.0 / 16, fallback_tol=tol))
        img, t = r.render(s.camera())
        flagged = tiles > tol
        print(f"quantile {q}: {flagged.sum()} of {flagged.size} tiles fall back, "
              f"{t['map_vertices']} of {full} map vertices built, light samples {t['light_samples']} "
              f"(whole map: {te['light_samples']})")
        assert t["fallback_tiles"] == flagged.sum() and flagged.sum() > 0
        assert 0 < t["map_vertices"] < full
        _check_tiles(img, mlp_img, exact_img, flagged)
    r.close()


def test_mlp_probe_first_order_gives_the_same_image(cuda_device):
    """Probe pixels first (the network then shades only the tiles that passed)
    and the network first give the same image bit for bit, the same fallback
    tiles and the same probe errors, at a tolerance where most tiles fail and
    at one where few do. A 200^2 image: 7 x 7 tiles with a ragged edge, 400
    probes (the last probe warp half full). The per-frame choice follows the
    last frame's fallback fraction."""
    s = scenes.small(67, n=40, image=200, m=24, kind="noise")
    r = _renderer(s)
    r.mlp_set_params(smooth_params(12))
    P = 10
    n = len(range(P // 2, s.width, P))
    r.mlp_set_probe_first(0)
    r.set_form(B.FORM_MLP, B.mlp_options(knot=4, probe_fraction=0.01, fallback_tol=1e30))
    r.render(s.camera())
    err = r.mlp_probe_errors(n * n).reshape(n, n)
    nt = -(-s.width // TILE)
    tiles = np.full((nt, nt), -np.inf)
    for j in range(n):
        for i in range(n):
            y, x = j * P + P // 2, i * P + P // 2
            tiles[y // TILE, x // TILE] = max(tiles[y // TILE, x // TILE], err[j, i])
    rows = {}
    for q in (0.2, 0.95):
        tol = float(np.quantile(tiles, q))
        flagged = int((tiles > tol).sum())
        out = {}
        for mode in (0, 1):
            r.mlp_set_probe_first(mode)
            r.set_form(B.FORM_MLP, B.mlp_options(knot=4, probe_fraction=0.01, fallback_tol=tol))
            img, t = r.render(s.camera())
            out[mode] = (img, t, r.mlp_probe_errors(n * n))
        print(f"quantile {q}: {flagged} of {tiles.size} tiles fall back; network rows "
              f"{out[0][1]['mlp_rows']} (network first) vs {out[1][1]['mlp_rows']} (probes first)")
        assert np.array_equal(out[0][0], out[1][0])
        assert out[0][1]["fallback_tiles"] == out[1][1]["fallback_tiles"] == flagged > 0
        assert out[0][1]["map_vertices"] == out[1][1]["map_vertices"]
        assert np.array_equal(out[0][2], out[1][2])
        rows[q] = (out[0][1]["mlp_rows"], out[1][1]["mlp_rows"], out[0][0])
    assert rows[0.2][1] < rows[0.2][0]
    # chosen per frame from the last frame's failing-tile count (the first auto
    # frame follows the last frame above, where few tiles failed)
    r.mlp_set_probe_first(-1)
    seq = []
    for q in (0.2, 0.2, 0.95, 0.95):
        r.set_form(B.FORM_MLP, B.mlp_options(knot=4, probe_fraction=0.01, fallback_tol=float(np.quantile(tiles, q))))
        img, t = r.render(s.camera())
        assert np.array_equal(img, rows[q][2])
        seq.append(t["mlp_rows"])
    assert seq == [rows[0.2][0], rows[0.2][1], rows[0.95][1], rows[0.95][0]]
    r.close()
