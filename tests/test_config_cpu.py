"""Stage TOML reader and scene description (host code of the library; no GPU)."""
from pathlib import Path

import numpy as np
import pytest

from pilot_b200 import beams as B

ROOT = Path(__file__).resolve().parent.parent


def test_reference_style_stage_file_parses():
    d = B.load_config(ROOT / "pilot_b200" / "configs" / "stage.toml")
    assert d.provider_name == b"spheres" and d.provider_type == b"subdivided_spheres"
    assert list(d.cell_dims) == [128, 128, 128]
    assert d.width == 512 and d.composite_background == 1 and d.shadow_size_ratio == 0.5
    assert d.n_lights == 1 and list(d.lights[0].position) == [0.5, 5.0, 0.5] and d.lights[0].intensity == 2.0
    assert d.tf_points == 11 and d.tf_alpha[3] == pytest.approx(1.0) and d.tf_size == 256


def test_minimal_reference_stage_uses_defaults():
    # the reference's own descriptor: a provider table only (Stage.cxx:25-49)
    d = B.parse_config('[dataset_providers.sph]\ntype = "subdivided_spheres"\ncell_dims = [16, 24, 32]\n')
    assert list(d.cell_dims) == [16, 24, 32] and d.form == B.FORM_EXACT and d.termination_alpha == 1.0
    assert d.n_lights == 0 and d.tf_preset == b"cool to warm" and d.light_steps == 128.0


def test_values_arrays_and_tables():
    d = B.parse_config('''
# comment line
[dataset_providers."quoted name"]   # trailing comment
type = 'noise'                      # literal string
cell_dims = 1_000
seed = 7
base_freq = 2.5e0

[render]
width = 64
height = 48
sample_distance = 0.01
form = "mlp"

[camera]
position = [0.5, 0.5, 3]
look_at = [0.5, 0.5, 0.5]
up = [0, 1, 0]

[[light]]
type = "directional"
direction = [1, -1, 0]
[[light]]
position = [
    1.0,
    2.0,
    3.0,
]

[form]
knot = 2
probe_fraction = 0.05
''')
    assert d.provider_name == b"quoted name" and d.provider_type == b"noise" and d.cell_dims[0] == 1000
    assert d.seed == 7 and d.base_freq == 2.5 and d.form == B.FORM_MLP and d.camera_explicit == 1
    assert d.n_lights == 2 and d.lights[0].kind == 1 and list(d.lights[1].position) == [1.0, 2.0, 3.0]
    assert d.mlp_knot == 2 and d.mlp_probe_fraction == pytest.approx(0.05)


@pytest.mark.parametrize("text,msg", [
    ('[render]\nwidth = "a"\n', "line 2: 'width' must be an integer"),
    ('[render]\nfoo = 1\n', "line 2: unknown key 'foo'"),
    ('[nope]\nx = 1\n', "line 2: unknown table [nope]"),
    ('x = 1\n', "line 1: key 'x' outside any table"),
    ('[render]\nwidth = 10 20\n', "line 2: unexpected text after value"),
    ('[render]\nwidth = 1\nwidth = 2\n', "line 3: duplicate key 'width'"),
    ('[transfer_function]\npoints = [0, 1]\nalphas = [0]\n', "points and alphas differ in length"),
    ('[render]\nbackground = [1, 1, 1]\n', "'background' must have 4 elements"),
    ('[dataset_providers.a]\ntype = "cubes"\n', "unknown dataset provider type"),
    ('[render]\nwidth = {a = 1}\n', "inline tables are not supported"),
    ('[render\nwidth = 1\n', "line 1: malformed table header"),
    ('[render]\nname = "abc\n', "unterminated string"),
    ('[render]\ntermination_alpha = 1.5\n', "must be in (0, 1]"),
    ('[shadow_map]\nnum_steps = 0\n', "'num_steps' out of range"),
])
def test_config_errors_name_the_line(text, msg):
    with pytest.raises(B.BeamsError) as e:
        B.parse_config(text)
    assert msg in str(e.value) and e.value.status == 6  # BEAMS_ERR_CONFIG


def test_missing_file_is_a_config_error(tmp_path):
    with pytest.raises(B.BeamsError) as e:
        B.load_config(tmp_path / "nothing.toml")
    assert e.value.status == 6 and "cannot open" in str(e.value)


def test_cool_to_warm_table_and_alpha_points():
    d = B.parse_config('[transfer_function]\npoints = [0.2, 0.8]\nalphas = [0.0, 1.0]\nsize = 256\n')
    t = B.scene_color_table(d)
    # Moreland's diverging map: the endpoints and the unsaturated midpoint (~0.865 grey)
    assert np.allclose(t[0, :3], [0.230, 0.299, 0.754], atol=1e-3)
    assert np.allclose(t[-1, :3], [0.706, 0.016, 0.150], atol=1e-3)
    assert np.allclose(t[128, :3], 0.865, atol=0.01)
    v = np.arange(256) / 255.0
    assert np.allclose(t[:, 3], np.clip((v - 0.2) / 0.6, 0, 1), atol=1e-6)
    r = B.scene_color_table(B.parse_config('[transfer_function]\npreset = "ramp"\n'))
    assert np.allclose(r[0, :3], [0.23, 0.30, 0.75], atol=1e-6)


def test_vtk_file_provider_path_resolution(tmp_path):
    (tmp_path / "stage.toml").write_text('[dataset_providers.v]\ntype = "vtk_file"\nfile_name = "data/v.vtk"\n')
    d = B.load_config(tmp_path / "stage.toml")
    assert d.provider_type.decode() == "vtk_file"
    assert d.file_name.decode() == str(tmp_path / "data" / "v.vtk")
    d2 = B.parse_config('[dataset_providers.v]\ntype = "vtk_file"\nfile_name = "/abs/v.vtk"\n')
    assert d2.file_name.decode() == "/abs/v.vtk"
    with pytest.raises(B.BeamsError):
        B.parse_config('[dataset_providers.v]\ntype = "vtk_file"\nfile_name = ""\n')
