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
