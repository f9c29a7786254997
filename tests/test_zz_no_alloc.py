"""gw_bsr_krylov_solve_static: the Krylov solve for callers that cannot call
cudaMalloc (a host whose memory manager owns the device heap, or a path on
which device allocation is not allowed).  Its scratch is a file-scope device
array inside the library, so the call takes no workspace.  Each check compares
it with gw_bsr_krylov_solve, which takes a caller workspace, on the same
system.

The file name sorts last, so pytest collects it after every other test: a run
that stops at its first failure has run everything else before reaching it."""
import ctypes as C

import numpy as np
import pytest
import torch

import cases
from cases import rel_err

pytestmark = pytest.mark.gpu


def _bar_system(material, precision):
    """A J2 / Hencky bar after two load steps, with the Jacobian and residual of
    the first Newton iterate of step 3 assembled (block-CSR on the GPU)."""
    from geowarp_b200.solvers import quasi_static_solver_2d
    grid, parts, it, mat, load = cases.bar_dicts(material, height=6.25)
    s = quasi_static_solver_2d(grid, parts, it, mat, load, precision=precision)
    b = np.zeros(s.n_matrix_size, dtype=bool)
    cases.bar_boundary(b, grid["n_grid_x"], grid["n_grid_y"])
    s.dofStruct.boundary_flag_array[:] = torch.as_tensor(b, device=s.x_particles.device)
    for k in range(2):
        s.advance_one_step(k, 4)
    e = s.engine
    s._set_step_params()
    s.reset()
    e.sort_and_activate()
    e.build_system()
    e.assemble(s._mat, 2, 4, want_K=True)
    return e


def _solve(e, static, rtol=1e-12):
    from geowarp_b200 import _lib as L
    from geowarp_b200.engine import _p
    lib = L.load()
    n = e.n_rows * e.nf
    x = torch.zeros(n, dtype=torch.float64, device=e.device)
    A = e.bsr_struct()
    it, rr = C.c_int32(0), C.c_double(0.0)
    if static:
        rc = lib.gw_bsr_krylov_solve_static(C.byref(A), e.prec, L.KRYLOV_BICGSTAB, L.PRECOND_BLOCK, _p(e._R), _p(x), rtol,
                                            20000, C.byref(it), C.byref(rr), e.stream)
    else:
        ws = torch.zeros(lib.gw_krylov_workspace_bytes(e.n_rows, e.nf, e.prec), dtype=torch.uint8, device=e.device)
        rc = lib.gw_bsr_krylov_solve(C.byref(A), e.prec, L.KRYLOV_BICGSTAB, L.PRECOND_BLOCK, _p(e._R), _p(x), rtol, 20000,
                                     _p(ws), C.byref(it), C.byref(rr), e.stream)
    torch.cuda.synchronize()
    return rc, x, it.value, rr.value


@pytest.mark.parametrize("material,precision", [("J2", "fp64"), ("Hencky elasticity", "mixed")])
def test_static_scratch_solve_matches_workspace_solve(cuda, material, precision):
    e = _bar_system(material, precision)
    rc, x_ref, it_ref, rr_ref = _solve(e, static=False)
    assert rc == 0 and rr_ref <= 1e-12
    # two calls in a row: the second one finds the first one's contents in the
    # shared scratch and must give the same answer
    for _ in range(2):
        rc, x, it, rr = _solve(e, static=True)
        assert rc == 0
        assert it == it_ref
        assert rel_err(x.cpu().numpy(), x_ref.cpu().numpy()) < 1e-9


def test_static_scratch_rejects_oversize_systems(cuda):
    from geowarp_b200 import _lib as L
    lib = L.load()
    limit = lib.gw_krylov_static_max_unknowns()
    assert limit == 131072
    buf = torch.zeros(16, dtype=torch.float64, device=cuda)
    A = L.Bsr()
    A.n_rows, A.nf, A.nnzb, A.mask_words = limit // 2 + 1, 2, 1, 1
    p = C.c_void_p(buf.data_ptr())
    A.row_ptr = A.cols = A.row2node = A.node2row = A.stencil = A.vals = p
    it, rr = C.c_int32(0), C.c_double(0.0)
    # rejected on the host before any launch: nothing reads the small buffer
    rc = lib.gw_bsr_krylov_solve_static(C.byref(A), L.PREC_F64, L.KRYLOV_BICGSTAB, L.PRECOND_BLOCK, p, p, 1e-10, 10,
                                        C.byref(it), C.byref(rr), None)
    assert rc == L.GW_EINVAL
    assert b"static scratch limit" in lib.gw_status_string(rc)
