"""Cell-associated fields: the unlit march of SamplerCellAssoc
(beams/rendering/LightedVolumeRenderer.cxx:501-642), K2c k_view_march_cells,
against the oracle's restatement (oracle_view_march_cells_f32).

What the restatement pins: the cell value fetched once per cell with a clamped,
truncating TF index (:603-608); tx = ty = tz = 2 at the start, so the first
sample locates (:581-583); composite, advance, then the break before the
tx/ty/tz update (:617-631); the final clamp to 1 (:632-635).

Bars: max per-pixel |dRGBA| <= 2e-3 against the oracle's f32 mode, >= 99.9% of
pixels bit-identical, lit-sample (composite) counts equal; the error against
the oracle's f64 mode is reported.
"""
import numpy as np
import pytest

from oracle.oracle import Oracle, psnr
from pilot_b200 import beams as B
from pilot_b200 import scenes

pytestmark = pytest.mark.gpu
TOL = 2e-3


def cell_values(s, how="mean"):
    """(nz-1, ny-1, nx-1) cell-centred values of the scene's point field."""
    f = s.field_numpy().astype(np.float64)
    if how == "mean":
        c = sum(f[dz:f.shape[0] - 1 + dz, dy:f.shape[1] - 1 + dy, dx:f.shape[2] - 1 + dx]
                for dz in (0, 1) for dy in (0, 1) for dx in (0, 1)) / 8.0
    else:
        c = f[:-1, :-1, :-1]
    return np.ascontiguousarray(c, np.float32)


def jittered(n, seed):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(3):
        w = rng.uniform(0.4, 1.6, n - 1)
        c = np.concatenate([[0.0], np.cumsum(w)])
        out.append(np.float32(c / c[-1]))
    return tuple(out)


def render_cells(s, cells, value_range=None, coords=None):
    r = B.Renderer(0)
    vr = s.value_range if value_range is None else value_range
    r.set_volume(cells, dims=s.dims, origin=s.origin, spacing=s.spacing, value_range=vr, assoc=B.ASSOC_CELLS)
    if coords is not None:
        r.set_volume_coordinates(*coords)
    s.configure(r)
    img, t = r.render(s.camera())
    r.close()
    return img, t


def check(s, cells, img, t, tag):
    o = Oracle(s, field=cells)
    oimg, olit = o.view_march_cells()
    err = np.abs(img - oimg)
    same = float(np.mean(np.all(img == oimg, axis=-1)))
    assert err.max() <= TOL, f"{tag}: max |d| {err.max()}"
    assert same >= 0.999, f"{tag}: only {same:.4f} of pixels bit-identical"
    assert t["lit_samples"] == olit, f"{tag}: lit {t['lit_samples']} vs oracle {olit}"
    i64, _ = o.view_march_cells(fp64=True)
    print(f"{tag}: max|d| vs f32 oracle {err.max():.2e}, identical {same:.5f}, lit {olit}, "
          f"PSNR vs f64 {psnr(img, i64):.1f} dB")
    return oimg


CASES = [
    dict(seed=31, kind="blobs", grid="uniform", cutoff=1.0),
    dict(seed=32, kind="noise", grid="uniform", cutoff=0.99),
    dict(seed=33, kind="blobs", grid="rectilinear", cutoff=0.99),
    dict(seed=34, kind="noise", grid="rectilinear", cutoff=1.0),
]


@pytest.mark.parametrize("cfg", CASES, ids=lambda c: f"{c['kind']}-{c['grid']}-s{c['seed']}")
def test_cell_field_matches_oracle(cuda_device, cfg):
    s = scenes.small(cfg["seed"], n=36, image=96, m=8, kind=cfg["kind"])
    s.use_map = False
    s.cutoff = cfg["cutoff"]
    coords = jittered(s.dims[0], cfg["seed"]) if cfg["grid"] == "rectilinear" else None
    if coords is not None:
        s.coords = coords
    cells = cell_values(s)
    img, t = render_cells(s, cells, coords=coords)
    oimg = check(s, cells, img, t, f"cells {cfg}")
    assert oimg[..., 3].max() > 0 and t["lit_samples"] > 0


def test_cell_field_clamped_index_and_non_cubic(cuda_device):
    """Values outside the range clamp to the first and last TF entries (a NaN
    cell takes entry 0); the image is not a whole number of warp tiles and the
    grid is not cubic."""
    s = scenes.small(35, n=30, image=90, m=8, kind="noise")
    s.use_map = False
    nx, ny, nz = 30, 22, 17
    s.dims = (nx, ny, nz)
    s.height = 70
    rng = np.random.default_rng(35)
    cells = rng.uniform(-0.5, 1.5, (nz - 1, ny - 1, nx - 1)).astype(np.float32)
    cells[3, 4, 5] = np.nan
    img, t = render_cells(s, cells, value_range=(0.0, 1.0))
    check(s, cells, img, t, "cells clamped / non-cubic")
    # the same render with the field inside the range moved past both ends is the
    # same image as the field clamped to the ends explicitly
    img2, _ = render_cells(s, np.nan_to_num(np.clip(cells, 0.0, 1.0), nan=0.0), value_range=(0.0, 1.0))
    assert np.array_equal(img, img2)


def test_cell_field_explicit_uniform_coordinates(cuda_device):
    """Explicit coordinates equal to the generated ones give the same image."""
    s = scenes.small(36, n=28, image=64, m=8)
    s.use_map = False
    cells = cell_values(s, "corner")
    base, _ = render_cells(s, cells)
    c = np.float32(s.origin[0]) + np.float32(s.spacing[0]) * np.arange(s.dims[0], dtype=np.float32)
    img, _ = render_cells(s, cells, coords=(c, c.copy(), c.copy()))
    assert np.array_equal(img, base)
