"""Legacy-VTK particle output.

The reference's problem scripts write the particle cloud after every load
step with meshio (e.g. problems/bar_compaction/bar_compaction_cpGIMP.py:
124-137: points plus point data such as stress or pore pressure).  meshio is
not a dependency here; this writes the same content as a legacy VTK
UNSTRUCTURED_GRID file: the particle positions, one VTK_VERTEX cell per
particle (so viewers show the points without a glyph filter), and the point
data arrays (scalars [N], vectors [N, 2|3], tensors [N, 3, 3]).
"""
import numpy as np

VTK_VERTEX = 1


def _host(a):
    if hasattr(a, "detach"):
        a = a.detach().cpu().numpy()
    return np.asarray(a)


def _pad3(v):
    """[N, 2] -> [N, 3] with a zero z component."""
    if v.shape[1] == 3:
        return v
    out = np.zeros((v.shape[0], 3), dtype=v.dtype)
    out[:, : v.shape[1]] = v
    return out


def write_particles_vtk(path, points, point_data=None, binary=True, title="geowarp_b200 particles"):
    """Write points [N, 2|3] and point_data {name: array} to a legacy VTK file.
    Arrays of shape [N] become SCALARS, [N, 2|3] VECTORS, [N, 3, 3] TENSORS;
    values are written as float64 (big-endian when binary)."""
    pts = _pad3(_host(points).astype(np.float64))
    n = pts.shape[0]
    fields = []
    for name, arr in (point_data or {}).items():
        a = _host(arr).astype(np.float64)
        if a.shape[0] != n:
            raise ValueError(f"point data '{name}' has {a.shape[0]} rows for {n} points")
        if " " in name:
            raise ValueError(f"point data name '{name}' contains a space")
        if a.ndim == 1:
            fields.append(("SCALARS", name, a.reshape(n, 1)))
        elif a.ndim == 2 and a.shape[1] in (2, 3):
            fields.append(("VECTORS", name, _pad3(a)))
        elif a.ndim == 3 and a.shape[1:] == (3, 3):
            fields.append(("TENSORS", name, a.reshape(n, 9)))
        else:
            raise ValueError(f"point data '{name}' has unsupported shape {a.shape}")

    def body(f, arr, dtype):
        if binary:
            f.write(np.ascontiguousarray(arr, dtype=dtype).astype(np.dtype(dtype).newbyteorder(">")).tobytes())
            f.write(b"\n")
        else:
            fmt = "%d" if np.dtype(dtype).kind == "i" else "%.17g"
            np.savetxt(f, np.asarray(arr).reshape(arr.shape[0], -1), fmt=fmt)

    with open(path, "wb") as f:
        f.write(b"# vtk DataFile Version 3.0\n")
        f.write(title[:255].encode() + b"\n")
        f.write(b"BINARY\n" if binary else b"ASCII\n")
        f.write(b"DATASET UNSTRUCTURED_GRID\n")
        f.write(f"POINTS {n} double\n".encode())
        body(f, pts, np.float64)
        f.write(f"CELLS {n} {2 * n}\n".encode())
        body(f, np.stack([np.ones(n, dtype=np.int32), np.arange(n, dtype=np.int32)], 1), np.int32)
        f.write(f"CELL_TYPES {n}\n".encode())
        body(f, np.full((n, 1), VTK_VERTEX, dtype=np.int32), np.int32)
        if fields:
            f.write(f"POINT_DATA {n}\n".encode())
        for kind, name, a in fields:
            if kind == "SCALARS":
                f.write(f"SCALARS {name} double 1\nLOOKUP_TABLE default\n".encode())
            else:
                f.write(f"{kind} {name} double\n".encode())
            body(f, a, np.float64)


def read_particles_vtk(path):
    """Read back what write_particles_vtk wrote: (points [N, 3], {name: array})."""
    with open(path, "rb") as f:
        data = f.read()
    pos = 0

    def line():
        nonlocal pos
        e = data.index(b"\n", pos)
        s = data[pos:e].decode()
        pos = e + 1
        return s

    line()
    line()
    binary = line().strip() == "BINARY"
    line()

    def block(count, dtype):
        nonlocal pos
        if binary:
            nb = count * np.dtype(dtype).itemsize
            a = np.frombuffer(data[pos:pos + nb], dtype=np.dtype(dtype).newbyteorder(">")).astype(dtype)
            pos += nb + 1
            return a
        vals = []
        while len(vals) < count:
            vals.extend(line().split())
        return np.array(vals, dtype=dtype)

    n = int(line().split()[1])
    pts = block(3 * n, np.float64).reshape(n, 3)
    line()
    block(2 * n, np.int32)
    line()
    block(n, np.int32)
    out = {}
    while pos < len(data):
        head = line().split()
        if not head or head[0] == "POINT_DATA":
            continue
        kind, name = head[0], head[1]
        if kind == "SCALARS":
            line()
            out[name] = block(n, np.float64)
        elif kind == "VECTORS":
            out[name] = block(3 * n, np.float64).reshape(n, 3)
        elif kind == "TENSORS":
            out[name] = block(9 * n, np.float64).reshape(n, 3, 3)
    return pts, out
