"""Device index guards: a column index outside the matrix is skipped and
recorded (site and value), gw_guard_read reports and clears the record, the
Krylov entry point returns GW_ERANGE, and the context stays usable.

The corrupted index is an off-diagonal column of an assembled bar Jacobian;
the only kernels that read the column array (the row products of the SpMV
and of GMRES) check it before the gather, so nothing outside the vectors is
touched."""
import ctypes as C

import pytest
import torch

pytestmark = pytest.mark.gpu


def _assembled_bar():
    from geowarp_b200 import problems
    s = problems.bar_compaction_2d(precision="fp64")
    for k in range(2):
        s.advance_one_step(k, 50)
    e = s.engine
    s._set_step_params()
    s.reset()
    e.sort_and_activate()
    e.build_system()
    e.assemble(s._mat, 2, 50, want_K=True)
    torch.cuda.synchronize()
    return e


def _read_guard(lib, e):
    site, val = C.c_int32(0), C.c_int64(0)
    assert lib.gw_guard_read(C.byref(site), C.byref(val), e.stream) == 0
    return site.value, val.value


def test_out_of_range_column_is_skipped_and_reported(cuda):
    from geowarp_b200 import _lib as L
    from geowarp_b200.engine import _p
    lib = L.load()
    e = _assembled_bar()
    assert _read_guard(lib, e) == (0, 0)
    n, nf = e.n_rows * e.nf, e.nf
    g = torch.Generator(device="cpu").manual_seed(3)
    x = torch.randn(n, dtype=torch.float64, generator=g).to(e.device)
    y0 = torch.zeros_like(x)
    L.call("gw_bsr_spmv", C.byref(e.bsr_struct()), e.prec, _p(x), _p(y0), e.stream)

    # corrupt one off-diagonal column of a middle row
    rp = e._row_ptr.cpu()
    cols = e._cols.clone()
    r = e.n_rows // 2
    js = [j for j in range(int(rp[r]), int(rp[r + 1])) if int(cols[j]) != r]
    j = js[len(js) // 2]
    c_old = int(cols[j])
    bad = e.n_rows + 1000
    cols[j] = bad
    A = e.bsr_struct()
    A.cols = _p(cols)
    y1 = torch.zeros_like(x)
    L.call("gw_bsr_spmv", C.byref(A), e.prec, _p(x), _p(y1), e.stream)
    torch.cuda.synchronize()
    site, val = _read_guard(lib, e)
    assert site != 0 and val == bad
    assert lib.gw_guard_site_name(site)
    assert _read_guard(lib, e) == (0, 0)  # read clears the record

    # the skipped block is the only difference
    blk = e._vals.t[: e.nnzb * nf * nf * 8].view(torch.float64).view(e.nnzb, nf, nf)[j]  # FP64 bar
    expect = y0.clone()
    expect[r * nf:(r + 1) * nf] -= blk @ x[c_old * nf:(c_old + 1) * nf]
    assert torch.allclose(y1, expect, rtol=1e-12, atol=1e-12 * float(y0.abs().max()))

    # a Krylov solve over the corrupted matrix ends with GW_ERANGE and names the site
    sol = torch.zeros_like(x)
    it, rr = C.c_int32(0), C.c_double(0.0)
    ws = torch.zeros(lib.gw_gmres_workspace_bytes(e.n_rows, e.nf, 30), dtype=torch.uint8, device=e.device)
    rc = lib.gw_bsr_gmres_solve(C.byref(A), e.prec, 1, _p(e._R), _p(sol), 1e-10, 60, 30, _p(ws), C.byref(it),
                                C.byref(rr), e.stream)
    assert rc == L.GW_ERANGE
    assert b"index guard" in lib.gw_status_string(rc)
    assert _read_guard(lib, e) == (0, 0)

    # the context is still usable: the intact matrix gives the first product again
    y2 = torch.zeros_like(x)
    L.call("gw_bsr_spmv", C.byref(e.bsr_struct()), e.prec, _p(x), _p(y2), e.stream)
    torch.cuda.synchronize()
    assert torch.equal(y2, y0)
