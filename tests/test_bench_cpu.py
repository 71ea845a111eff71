"""The CPU legs of bench.py (the reference arm and the cpu_baseline): the
sample of whole z-slabs and row bands, its extrapolation to one frame, and the
whole-frame run it is checked against. CPU only (the oracle)."""
import numpy as np

import bench
from oracle.oracle import Oracle
from pilot_b200 import scenes


def test_sample_covering_the_frame_extrapolates_exactly():
    """With a budget larger than the frame the sample is every slab and every
    row: its lit-sample count equals the whole frame's."""
    s = scenes.small(91, n=20, image=48, m=8, kind="noise")
    field = s.field_numpy()
    full = bench.cpu_full_frame(s, field, threads=2)
    zero = np.zeros((s.map_m + 1,) * 3, np.float32)
    samp = bench.cpu_sample_frame(s, field, zero, budget_s=100.0, threads=2)
    assert samp["lit_per_frame"] == full["lit_per_frame"]
    assert f"{s.map_m + 1} of {s.map_m + 1} whole z-slabs" in samp["sample"]
    assert full["frame_s"] > 0 and samp["frame_s"] > 0


def test_partial_sample_is_whole_slabs_and_row_bands():
    s = scenes.small(92, n=24, image=64, m=15, kind="blobs")
    field = s.field_numpy()
    zero = np.zeros((s.map_m + 1,) * 3, np.float32)
    samp = bench.cpu_sample_frame(s, field, zero, budget_s=1e-6, threads=1, rng_seed=3)
    # the smallest sample: one slab and one band of one row
    assert "1 of 16 whole z-slabs" in samp["sample"] and "1 bands of 1 of 64" in samp["sample"]
    assert samp["frame_s"] > 0 and samp["lit_per_frame"] >= 0


def test_full_frame_map_is_the_oracle_map():
    s = scenes.small(93, n=20, image=32, m=8)
    field = s.field_numpy()
    full = bench.cpu_full_frame(s, field, threads=2)
    om, _ = Oracle(s, field=field).light_march()
    assert np.array_equal(full["map"], om)
    _, lit = Oracle(s, field=field).view_march(om)
    assert full["lit_per_frame"] == lit
