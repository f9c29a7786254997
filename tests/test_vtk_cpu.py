"""Legacy-VTK particle output (the reference's per-step meshio files): the
writer's files read back to the same points and point data, binary and
ASCII, and carry the header a legacy-VTK reader expects."""
import numpy as np
import pytest

from geowarp_b200.vtk import read_particles_vtk, write_particles_vtk


@pytest.mark.parametrize("binary", [True, False])
def test_vtk_round_trip(tmp_path, binary):
    rng = np.random.default_rng(3)
    n = 37
    x = rng.normal(size=(n, 2))
    data = {"pressure": rng.normal(size=n), "displacement": rng.normal(size=(n, 2)),
            "stress": rng.normal(size=(n, 3, 3))}
    path = tmp_path / "particles.vtk"
    write_particles_vtk(path, x, data, binary=binary)
    head = open(path, "rb").read(200)
    assert head.startswith(b"# vtk DataFile Version 3.0\n")
    assert (b"BINARY" if binary else b"ASCII") in head and b"DATASET UNSTRUCTURED_GRID" in head
    pts, out = read_particles_vtk(path)
    assert np.array_equal(pts[:, :2], x) and np.all(pts[:, 2] == 0.0)
    assert np.array_equal(out["pressure"], data["pressure"])
    assert np.array_equal(out["displacement"][:, :2], data["displacement"])
    assert np.array_equal(out["stress"], data["stress"])


def test_vtk_rejects_mismatched_data(tmp_path):
    with pytest.raises(ValueError):
        write_particles_vtk(tmp_path / "bad.vtk", np.zeros((4, 3)), {"p": np.zeros(5)})


def test_vtk_bytes_follow_the_legacy_format(tmp_path):
    """Two particles with a scalar, a 2D vector and a tensor, checked against the
    bytes the legacy VTK format (version 3.0, UNSTRUCTURED_GRID) prescribes,
    spelled out here independently of the module's reader: header, POINTS as
    x y z doubles, one VTK_VERTEX (type 1) cell per point given as "1 i",
    POINT_DATA sections; the binary variant holds big-endian values, each
    block followed by a newline."""
    import struct
    from geowarp_b200.vtk import write_particles_vtk
    pts = np.array([[0.5, 1.25], [2.0, -3.0]])
    p = np.array([7.0, -1.5])
    u = np.array([[1.0, 2.0], [3.0, 4.0]])
    s = np.arange(18, dtype=np.float64).reshape(2, 3, 3)
    f = tmp_path / "a.vtk"
    write_particles_vtk(f, pts, {"p": p, "u": u, "sigma": s}, binary=False, title="t")
    expect = ("# vtk DataFile Version 3.0\nt\nASCII\nDATASET UNSTRUCTURED_GRID\n"
              "POINTS 2 double\n0.5 1.25 0\n2 -3 0\n"
              "CELLS 2 4\n1 0\n1 1\nCELL_TYPES 2\n1\n1\n"
              "POINT_DATA 2\nSCALARS p double 1\nLOOKUP_TABLE default\n7\n-1.5\n"
              "VECTORS u double\n1 2 0\n3 4 0\n"
              "TENSORS sigma double\n0 1 2 3 4 5 6 7 8\n9 10 11 12 13 14 15 16 17\n")
    assert f.read_bytes().decode() == expect
    fb = tmp_path / "b.vtk"
    write_particles_vtk(fb, pts, {"p": p}, binary=True, title="t")
    dbl = lambda *v: struct.pack(">%dd" % len(v), *v)
    i32 = lambda *v: struct.pack(">%di" % len(v), *v)
    expect_b = (b"# vtk DataFile Version 3.0\nt\nBINARY\nDATASET UNSTRUCTURED_GRID\n"
                b"POINTS 2 double\n" + dbl(0.5, 1.25, 0.0, 2.0, -3.0, 0.0) + b"\n"
                b"CELLS 2 4\n" + i32(1, 0, 1, 1) + b"\n"
                b"CELL_TYPES 2\n" + i32(1, 1) + b"\n"
                b"POINT_DATA 2\nSCALARS p double 1\nLOOKUP_TABLE default\n" + dbl(7.0, -1.5) + b"\n")
    assert fb.read_bytes() == expect_b
