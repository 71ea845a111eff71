"""Legacy VTK reader (beams_vtk_read), the input side of the reference's file
scenes (pilot/io/DataSetUtils.cxx:13-42). Host code: runs without a GPU.
Files are written here in the published legacy format, ASCII and BINARY
(big-endian), and read back exactly (float32 values, or the float32 rounding
of other types)."""
import numpy as np
import pytest

from pilot_b200 import beams as B

VTK_TYPES = {np.float32: "float", np.float64: "double", np.uint8: "unsigned_char", np.int16: "short",
             np.int32: "int", np.uint16: "unsigned_short"}


def write_vtk(path, data, binary, kind="STRUCTURED_POINTS", origin=(0, 0, 0), spacing=(1, 1, 1), coords=None,
              cells=False, dtype=np.float32, coord_dtype=np.float32, lookup=True):
    nz, ny, nx = data.shape
    dims = (nx + 1, ny + 1, nz + 1) if cells else (nx, ny, nz)
    out = bytearray()

    def put(text):
        out.extend(text.encode())

    def arr(a, dt):
        a = np.ascontiguousarray(a, dt)
        if binary:
            out.extend(a.astype(a.dtype.newbyteorder(">")).tobytes())
            put("\n")
        else:
            put(" ".join(repr(float(v)) if np.issubdtype(dt, np.floating) else str(int(v)) for v in a.ravel()) + "\n")
    put("# vtk DataFile Version 3.0\ntest volume\n" + ("BINARY" if binary else "ASCII") + "\n")
    put(f"DATASET {kind}\nDIMENSIONS {dims[0]} {dims[1]} {dims[2]}\n")
    if kind == "STRUCTURED_POINTS":
        put(f"ORIGIN {origin[0]} {origin[1]} {origin[2]}\nSPACING {spacing[0]} {spacing[1]} {spacing[2]}\n")
    else:
        for ax, c in zip("XYZ", coords):
            put(f"{ax}_COORDINATES {len(c)} {VTK_TYPES[coord_dtype]}\n")
            arr(c, coord_dtype)
    put(f"{'CELL_DATA' if cells else 'POINT_DATA'} {data.size}\nSCALARS density {VTK_TYPES[dtype]} 1\n")
    if lookup:
        put("LOOKUP_TABLE default\n")
    arr(data, dtype)
    path.write_bytes(bytes(out))


@pytest.mark.parametrize("binary", [False, True])
@pytest.mark.parametrize("dtype", [np.float32, np.float64, np.uint8, np.int16])
def test_structured_points_round_trip(tmp_path, binary, dtype):
    rng = np.random.default_rng(3)
    data = (rng.random((5, 6, 7)) * 200).astype(dtype)
    p = tmp_path / "v.vtk"
    write_vtk(p, data, binary, origin=(0.5, -1.0, 2.0), spacing=(0.25, 0.5, 1.0), dtype=dtype)
    v = B.vtk_read(p)
    assert v["dims"] == (7, 6, 5) and v["assoc"] == B.ASSOC_POINTS and v["coords"] is None
    assert v["origin"] == (0.5, -1.0, 2.0) and v["spacing"] == (0.25, 0.5, 1.0)
    assert np.array_equal(v["data"], data.astype(np.float32))
    assert v["range"] == (float(data.astype(np.float32).min()), float(data.astype(np.float32).max()))
    assert v["name"] == "density"


@pytest.mark.parametrize("binary", [False, True])
def test_rectilinear_grid_and_cell_data(tmp_path, binary):
    rng = np.random.default_rng(4)
    coords = [np.sort(rng.random(n)).astype(np.float32) + np.arange(n, dtype=np.float32) for n in (6, 5, 4)]
    data = rng.random((4, 5, 6)).astype(np.float32)
    p = tmp_path / "r.vtk"
    write_vtk(p, data, binary, kind="RECTILINEAR_GRID", coords=coords, coord_dtype=np.float64)
    v = B.vtk_read(p)
    assert v["dims"] == (6, 5, 4)
    for d in range(3):
        assert np.array_equal(v["coords"][d], coords[d])
    assert np.array_equal(v["data"], data)
    cells = rng.random((3, 4, 5)).astype(np.float32)
    q = tmp_path / "c.vtk"
    write_vtk(q, cells, binary, cells=True, lookup=False)
    c = B.vtk_read(q)
    assert c["assoc"] == B.ASSOC_CELLS and c["dims"] == (6, 5, 4) and np.array_equal(c["data"], cells)


def test_bad_files_are_rejected(tmp_path):
    p = tmp_path / "bad.vtk"
    p.write_text("not vtk\n")
    with pytest.raises(B.BeamsError):
        B.vtk_read(p)
    data = np.zeros((3, 3, 3), np.float32)
    write_vtk(p, data, False)
    text = p.read_text().replace("POINT_DATA 27", "POINT_DATA 26")
    p.write_text(text)
    with pytest.raises(B.BeamsError):
        B.vtk_read(p)
    write_vtk(p, data, True)
    p.write_bytes(p.read_bytes()[:-40])  # truncated binary payload
    with pytest.raises(B.BeamsError):
        B.vtk_read(p)
    with pytest.raises(B.BeamsError):
        B.vtk_read(tmp_path / "missing.vtk")
