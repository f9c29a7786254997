"""Restarted GMRES on a system where it provably makes no progress stops on
stagnation (GW_TUNE_GMRES_STALL) instead of running to max_iter.

The system is the cyclic shift on 64 unknowns (row i holds a single 1 at
column i-1, row 0 at column 63) with b = e_0 and x0 = 0.  Its pattern has no
diagonal block, so the Jacobi preconditioner is the identity.  The Krylov space
of GMRES(30) from e_0 is span(e_0 .. e_29) and its image under A is
span(e_1 .. e_30), orthogonal to b: every cycle ends with x = 0 and the
residual exactly ||b|| = 1 (Hessenberg columns with one unit subdiagonal entry,
Givens rotations c = 0, s = 1, no division by anything but 1)."""
import ctypes as C

import pytest
import torch

pytestmark = pytest.mark.gpu

N, RESTART = 64, 30


def _shift_system(dev):
    from geowarp_b200 import _lib as L
    from geowarp_b200.engine import _p
    keep = {
        "row_ptr": torch.arange(N + 1, dtype=torch.int32, device=dev),
        "cols": ((torch.arange(N, dtype=torch.int32, device=dev) - 1) % N).to(torch.int32),
        "row2node": torch.arange(N, dtype=torch.int32, device=dev),
        "node2row": torch.arange(N, dtype=torch.int32, device=dev),
        "stencil": torch.zeros(N, dtype=torch.int32, device=dev),  # no blocks named: identity preconditioner
        "vals": torch.ones(N, dtype=torch.float64, device=dev),
    }
    A = L.Bsr()
    A.n_rows, A.nf, A.nnzb, A.mask_words = N, 1, N, 1
    for k, t in keep.items():
        setattr(A, k, _p(t))
    return A, keep


def _solve(lib, A, max_iter, dev):
    from geowarp_b200 import _lib as L
    from geowarp_b200.engine import _p
    b = torch.zeros(N, dtype=torch.float64, device=dev)
    b[0] = 1.0
    x = torch.zeros_like(b)
    ws = torch.zeros(lib.gw_gmres_workspace_bytes(N, 1, RESTART), dtype=torch.uint8, device=dev)
    it, rr = C.c_int32(0), C.c_double(0.0)
    rc = lib.gw_bsr_gmres_solve(C.byref(A), L.PREC_F64, L.PRECOND_DIAG, _p(b), _p(x), 1e-10, max_iter, RESTART,
                                _p(ws), C.byref(it), C.byref(rr), None)
    torch.cuda.synchronize()
    return rc, it.value, rr.value, x


def test_stagnating_gmres_stops_after_the_window(cuda):
    from geowarp_b200 import _lib as L
    lib = L.load()
    A, keep = _shift_system(cuda)
    default = lib.gw_tune_get(L.TUNE_GMRES_STALL)
    try:
        assert lib.gw_tune_set(L.TUNE_GMRES_STALL, 5) == L.GW_OK
        rc, it, rr, x = _solve(lib, A, 20000, cuda)
        assert rc == L.GW_ENOCONV
        assert lib.gw_gmres_last_stalled() == 1
        assert it == 5 * RESTART  # five full cycles, stopped at the start of the sixth
        assert rr == 1.0 and torch.count_nonzero(x) == 0

        # off: the solve runs to max_iter
        assert lib.gw_tune_set(L.TUNE_GMRES_STALL, 0) == L.GW_OK
        rc, it, rr, x = _solve(lib, A, 10 * RESTART, cuda)
        assert rc == L.GW_ENOCONV
        assert lib.gw_gmres_last_stalled() == 0
        assert it == 10 * RESTART
        assert rr == 1.0
    finally:
        lib.gw_tune_set(L.TUNE_GMRES_STALL, default)


def test_converging_solve_is_not_stopped(cuda):
    """The same ring with a diagonal of 2 (A = 2 I + shift: eigenvalues
    2 + the 64th roots of unity, so GMRES gains about a factor 2 per step) is
    solved to tolerance with the check at its tightest window of one cycle,
    and the flag stays clear."""
    from geowarp_b200 import _lib as L
    from geowarp_b200.engine import _p
    lib = L.load()
    rows = torch.arange(N, dtype=torch.int32)
    cols = torch.stack([(rows - 1) % N, rows], 1).reshape(-1)  # columns ascending except row 0
    keep = {
        "row_ptr": torch.arange(0, 2 * N + 1, 2, dtype=torch.int32).to(cuda),
        "cols": cols.to(torch.int32).to(cuda),
        "row2node": rows.to(cuda),
        "node2row": rows.to(cuda),
        "stencil": torch.zeros(N, dtype=torch.int32, device=cuda),
        "vals": torch.tensor([1.0, 2.0] * N, dtype=torch.float64, device=cuda),
    }
    A = L.Bsr()
    A.n_rows, A.nf, A.nnzb, A.mask_words = N, 1, 2 * N, 1
    for k, t in keep.items():
        setattr(A, k, _p(t))
    default = lib.gw_tune_get(L.TUNE_GMRES_STALL)
    try:
        assert lib.gw_tune_set(L.TUNE_GMRES_STALL, 1) == L.GW_OK
        rc, it, rr, x = _solve(lib, A, 20000, cuda)
    finally:
        lib.gw_tune_set(L.TUNE_GMRES_STALL, default)
    assert rc == L.GW_OK and rr <= 1e-10
    assert lib.gw_gmres_last_stalled() == 0
    # (2 I + S) x = e_0: x_i = (-1/2)^i x_0 with x_0 (2 - 2^-(N-1)) = 1
    x0 = 1.0 / (2.0 - 2.0 ** -(N - 1))
    expect = torch.tensor([x0 * (-0.5) ** i for i in range(N)], dtype=torch.float64)
    assert torch.allclose(x.cpu(), expect, rtol=0, atol=1e-9)
