"""CPU checks of the C ABI: the library loads, exports every symbol the
header declares, and the ctypes structures match the C layouts; plus the
host-side pieces of the drop-in API."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "geowarp_b200.h")


def declared_functions():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^(?:int|int64_t|const char \*)\s*\**\s*(gw_\w+)\(", txt, re.M)))


def test_library_exports_every_declared_symbol():
    from geowarp_b200 import _lib
    from geowarp_b200.build import build
    build()
    lib = _lib.load()
    decl = declared_functions()
    assert len(decl) >= 20
    for name in decl:
        assert hasattr(lib, name), name
        assert name in _lib.SIGNATURES, name
    assert lib.gw_version() == 1
    assert lib.gw_status_string(-6).decode().startswith("index guard")


def test_struct_layouts_match_c():
    from geowarp_b200 import _lib
    structs = {"gw_grid_t": _lib.Grid, "gw_material_t": _lib.Material, "gw_step_t": _lib.Step,
               "gw_particles_t": _lib.Particles, "gw_bsr_t": _lib.Bsr, "gw_adjoint_t": _lib.Adjoint,
               "gw_mg_plan_t": _lib.MgPlan}
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void) {"]
    for cname, py in structs.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'printf("{cname}.{fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0; }")
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "l.c")
        exe = os.path.join(d, "l")
        open(src, "w").write("\n".join(lines))
        subprocess.run(["gcc", src, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split("\n")
    got = dict(l.split() for l in out if l)
    for cname, py in structs.items():
        assert int(got[cname]) == C.sizeof(py), cname
        for fname, _ in py._fields_:
            assert int(got[f"{cname}.{fname}"]) == getattr(py, fname).offset, (cname, fname)


def test_init_particles_match_reference_loops():
    from geowarp_b200.mpm.mpm_utils import init_particles_rectangle_2d, init_particles_rectangle_3d
    from oracle.mpm import init_particles_rectangle_2d as o2, init_particles_rectangle_3d as o3
    a = init_particles_rectangle_2d(0.78125, 0.78125, 1.5625, 13.28125, 0.78125, 6, 18, 2, 64)
    b = o2(0.78125, 0.78125, 1.5625, 13.28125, 0.78125, 6, 18, 2, 64)
    assert np.array_equal(a, b)
    a = init_particles_rectangle_3d(0.25, 0.25, 0.0, 1.25, 1.25, 1.0, 0.25, 6, 6, 6, 2, 512)
    b = o3(0.25, 0.25, 0.0, 1.25, 1.25, 1.0, 0.25, 6, 6, 6, 2, 512)
    assert np.array_equal(a, b)


def test_launch_adapter_matches_numpy_bc():
    import torch
    import cases
    from geowarp_b200 import launch
    nx, ny = 6, 20
    nn = (nx + 1) * (ny + 1)
    flags = torch.zeros(3 * nn, dtype=torch.bool)
    launch(cases.terzaghi_boundary_kernel, (nx + 1, ny + 1), [flags, nx, nn])
    ref = np.zeros(3 * nn, dtype=bool)
    cases.terzaghi_boundary_np(ref, nx, ny)
    assert np.array_equal(flags.numpy(), ref)


def test_engine_fails_loudly_without_cuda():
    import torch
    if torch.cuda.is_available():
        pytest.skip("CUDA present")
    import cases
    from geowarp_b200.solvers import quasi_static_solver_2d
    grid, parts, it, mat, load = cases.bar_dicts()
    with pytest.raises(RuntimeError, match="CUDA"):
        quasi_static_solver_2d(grid, parts, it, mat, load)


def test_unknown_material_raises():
    from geowarp_b200.engine import material_struct
    with pytest.raises(ValueError):
        material_struct(dict(material_name="Mohr-Coulomb"))


def test_vectorised_entry_points_reject_misaligned_vectors():
    """2x2 / 4x4 systems are gathered with 16-byte loads: a vector that is not
    16-byte aligned is rejected on the host, before any launch or access."""
    import ctypes as C
    import numpy as np
    from geowarp_b200 import _lib as L
    lib = L.load()
    buf = np.zeros(64, dtype=np.float64)
    base = buf.ctypes.data
    off = base + (16 - base % 16) % 16          # 16-byte aligned address inside buf
    A = L.Bsr()
    A.n_rows, A.nf, A.nnzb, A.mask_words = 2, 2, 2, 1
    p = C.c_void_p(off)
    A.row_ptr = A.cols = A.row2node = A.node2row = A.stencil = A.vals = p
    rc = lib.gw_bsr_spmv(C.byref(A), L.PREC_F64, C.c_void_p(off + 8), p, None)
    assert rc == L.GW_EINVAL
    assert b"vec_ok" in lib.gw_status_string(rc)
