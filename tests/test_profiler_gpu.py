"""beams_set_profiler, the counterpart of MapperLightedVolume::SetProfiler
(MapperLightedVolume.h:57): every render reports the reference's frames
(Render > Phase 1, Phase 4, Phase 5) with their CUDA-event times, with or
without a timings struct, until the profiler is removed."""
import pytest

from pilot_b200 import beams as B
from pilot_b200 import scenes

pytestmark = pytest.mark.gpu


def test_profiler_reports_each_render_frames(cuda_device):
    s = scenes.small(71, n=40, image=64, m=16, kind="noise", light_kind=0)
    with B.Renderer(0) as r:
        r.set_volume(s.field_numpy(), origin=s.origin, spacing=s.spacing, value_range=s.value_range)
        s.configure(r)
        got = []
        r.set_profiler(lambda frame, depth, ms: got.append((frame, depth, ms)))
        _, t = r.render(s.camera())
        r.render(s.camera(), timings=False)
        frames = [("Render", 0), ("Phase 1", 1), ("Phase 4", 1), ("Phase 5", 1)]
        assert [(f, d) for f, d, _ in got] == frames * 2
        total, p1, p4, p5 = (ms for _, _, ms in got[:4])
        assert total == pytest.approx(t["total_ms"], rel=1e-6) and p1 == pytest.approx(t["map_build_ms"], rel=1e-6)
        assert p1 > 0 and p4 > 0 and p5 >= 0
        # the phases are consecutive event intervals of the render
        assert abs(p1 + p4 + p5 - total) <= 0.01 * total + 0.01
        r.set_profiler(None)
        r.render(s.camera(), timings=False)
        assert len(got) == 8
