"""Newton's starting iterate from the previous load step (mixed precision):
gw_predict_increment copies the previous converged increment onto the new
step's free DOFs only, and the predicted start changes how a load step is
solved, not what it converges to."""
import ctypes as C

import numpy as np
import pytest
import torch

from cases import rel_err

pytestmark = pytest.mark.gpu


def test_predict_increment_keeps_free_dofs_of_active_rows(cuda):
    from geowarp_b200 import _lib as L
    from geowarp_b200 import problems
    from geowarp_b200.engine import _p
    s = problems.bar_compaction_2d(precision="mixed", device=cuda)
    s.advance_one_step(0, 20)
    e = s.engine
    s._set_step_params()
    s.reset()
    e.sort_and_activate()
    e.build_system()
    g = torch.Generator(device="cpu").manual_seed(11)
    u_prev = torch.randn(e.n_nodes * e.nf, dtype=torch.float64, generator=g).to(cuda)
    e.u_new.fill_(0.0)
    L.call("gw_predict_increment", C.byref(e.bsr_struct()), _p(e.free_mask), _p(u_prev), _p(e.u_new), e.stream)
    torch.cuda.synchronize()
    fm = e.free_mask.cpu().numpy().astype(np.int64)
    rows = e.row2node[: e.n_rows].cpu().numpy()
    expect = np.zeros((e.n_nodes, e.nf))
    up = u_prev.cpu().numpy().reshape(e.n_nodes, e.nf)
    for f in range(e.nf):
        free = (fm[rows] >> f) & 1
        expect[rows, f] = np.where(free == 1, up[rows, f], 0.0)
    got = e.u_new.cpu().numpy().reshape(e.n_nodes, e.nf)
    assert np.array_equal(got, expect)
    assert (expect != 0).any() and ((fm[rows] & 3) != 3).any()  # both kinds of DOF present


def test_predicted_start_converges_to_the_same_state(cuda):
    from geowarp_b200 import problems
    out, first = {}, {}
    for on in (False, True):
        s = problems.bar_compaction_2d(precision="mixed", device=cuda, tol=1e-8)
        e = s.engine
        e.predict_increment = on
        for k in range(4):
            s.advance_one_step(k, 20)
        out[on] = ((s.x_particles - s.x0).cpu().numpy(), s.particle_Cauchy_stress_array.cpu().numpy())
        first[on] = {l[0]: l[2] for l in e.log if l[1] == 0}  # ||R|| of each step's first iterate
    assert rel_err(out[True][0], out[False][0]) < 1e-8
    assert rel_err(out[True][1], out[False][1]) < 1e-8
    assert first[True][0] == first[False][0]  # no previous step: both start from zero
    for k in (1, 2, 3):
        assert first[True][k] < 0.1 * first[False][k], (k, first[True][k], first[False][k])
