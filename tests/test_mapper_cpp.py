"""The C++ adapter (include/beams_mapper.hpp) compiled the way a reference-side
caller would use it: tests/cpp/mapper_snippet.cpp holds the integration notes'
call sequence (MapperLightedVolume setters, SetActiveColorTable, RenderCells)
and links libbeams_b200.so.

CPU: the snippet compiles with g++ -Wall -Werror against the adapter and links.
GPU: it renders a small seeded scene whose image matches the oracle within the
exact form's bar (max |dRGBA| <= 2e-3, >= 99.9% of pixels bit-identical) with
the oracle's lit-sample count, and the profiler set with SetProfiler holds the
two renders' frames in the reference's summary format.
"""
import subprocess
from pathlib import Path

import numpy as np
import pytest

from pilot_b200 import beams as B

ROOT = Path(__file__).resolve().parent.parent
SRC = ROOT / "tests" / "cpp" / "mapper_snippet.cpp"
TOL = 2e-3


def build_snippet(out_dir: Path) -> Path:
    lib = B._LIB_PATH
    exe = out_dir / "mapper_snippet"
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-I", str(ROOT / "include"), str(SRC),
           "-o", str(exe), "-L", str(Path(lib).parent), "-lbeams_b200", f"-Wl,-rpath,{Path(lib).parent}"]
    p = subprocess.run(cmd, capture_output=True, text=True)
    assert p.returncode == 0, p.stdout + p.stderr
    return exe


def test_mapper_snippet_compiles_and_links(tmp_path):
    B.lib()  # builds the library if needed
    exe = build_snippet(tmp_path)
    p = subprocess.run([str(exe)], capture_output=True, text=True)
    assert p.returncode == 2 and "usage" in p.stderr


@pytest.mark.gpu
def test_mapper_snippet_renders_like_the_oracle(cuda_device, tmp_path):
    from oracle.oracle import Oracle
    from pilot_b200 import scenes
    exe = build_snippet(tmp_path)
    s = scenes.small(41, n=36, image=80, m=18, kind="noise", light_kind=0)
    s.light_intensity = 2.0
    s.height = 72
    s.field_numpy().astype(np.float32).tofile(tmp_path / "field.bin")
    np.ascontiguousarray(s.tf, np.float32).tofile(tmp_path / "tf.bin")
    nx, ny, nz = s.dims
    args = [str(tmp_path), nx, ny, nz, s.map_m, *s.light, *s.cam_pos, *s.cam_up, s.fov_y_deg, s.width, s.height,
            s.sample_distance]
    p = subprocess.run([str(exe), *[repr(float(a)) if isinstance(a, float) else str(a) for a in args]],
                       capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stdout + p.stderr
    img = np.fromfile(tmp_path / "rgba.bin", np.float32).reshape(s.height, s.width, 4)
    o = Oracle(s)
    oimg, lit = o.view_march(o.light_march()[0])
    err = float(np.abs(img - oimg).max())
    assert err <= TOL, f"max |d| {err}"
    assert np.mean(np.all(img == oimg, axis=-1)) >= 0.999
    assert int(p.stdout.split()[0]) == lit
    # SetProfiler: the profiler's summary, one line per frame, indented per level
    lines = p.stderr.splitlines()
    names = [ln.split(":")[0] for ln in lines]
    assert names[:6] == ["Beams", "  Render", "    Phase 1", "    Phase 4", "    Phase 5", "  Second render"]
    assert names[6:] == ["    Render", "      Phase 1", "      Phase 4", "      Phase 5"]
    assert all("Min = " in ln and "Avg = " in ln for ln in lines)
