"""C-ABI library checks that need no GPU: it loads, exports every entry point
include/beams_b200.h declares, and reports a clean error where a GPU is needed."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

from pilot_b200 import beams as B

ROOT = Path(__file__).resolve().parent.parent


def declared(header: str):
    text = (ROOT / "include" / header).read_text()
    return sorted(set(re.findall(r"^\s*(?:beams_status|const char\*|int)\s+(beams_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    L = B.lib()
    names = declared("beams_b200.h")
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, f"not exported: {missing}"
    nm = subprocess.run(["nm", "-D", "--defined-only", str(B._LIB_PATH)], capture_output=True, text=True).stdout
    for n in names:
        assert re.search(rf"\bT {n}$", nm, re.M), f"{n} is not a defined text symbol"


def test_abi_version():
    assert B.lib().beams_abi_version() == 1


def test_create_without_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    st = B.lib().beams_create(C.byref(h), 0, None)
    assert st != 0 and not h.value
    assert B.lib().beams_last_error(None)


def test_null_arguments_are_rejected_without_a_device():
    L = B.lib()
    assert L.beams_create(None, 0, None) == 1
    assert L.beams_set_sample_distance(None, C.c_float(1.0)) == 1
    assert L.beams_destroy(None) == 0
    n = (C.c_int * 3)(1, 1, 1)
    assert L.beams_generate_blobs(None, n, None, 0, 1, None) == 1


# The ctypes mirrors of the header's structs, by C name.
MIRRORS = {"beams_mlp_options": "MlpOptions", "beams_mlp_report": "MlpReport", "beams_tuning": "Tuning",
           "beams_volume": "Volume", "beams_camera": "Camera", "beams_request": "Request",
           "beams_batch_options": "BatchOptions", "beams_config_light": "ConfigLight",
           "beams_scene_desc": "SceneDesc", "beams_timings": "Timings", "beams_vtk_field": "VtkField"}


def test_ctypes_structs_match_the_header(tmp_path):
    """Every struct the Python binding mirrors has the header's size and field
    offsets (a C program built with the host compiler prints them)."""
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "beams_b200.h"', "int main(void) {"]
    for cname, pyname in MIRRORS.items():
        lines.append(f'  printf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for field, _ in getattr(B, pyname)._fields_:
            lines.append(f'  printf("{cname} {field} %zu\\n", offsetof({cname}, {field}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    got = {}
    for ln in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines():
        cname, key, val = ln.split()
        got[(cname, key)] = int(val)
    for cname, pyname in MIRRORS.items():
        cls = getattr(B, pyname)
        assert got[(cname, "sizeof")] == C.sizeof(cls), cname
        for field, _ in cls._fields_:
            assert got[(cname, field)] == getattr(cls, field).offset, (cname, field)
