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
