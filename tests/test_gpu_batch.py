"""Batched blocks (geowarp_b200.batch): instances packed into one grid must step
exactly like the same instances run one by one, forward and adjoint."""
import numpy as np
import pytest
import torch

from cases import rel_err

pytestmark = pytest.mark.gpu

SIZES = [(12, 8), (20, 10), (9, 14)]


def _fields(seed):
    from geowarp_b200 import batch
    return [np.log(1e7) + batch.gaussian_random_field(nx, ny, 2, 0.05, 0.5, 0.3, seed + q)
            for q, (nx, ny) in enumerate(SIZES)]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batched_blocks_step_like_separate_runs(cuda, precision):
    from geowarp_b200.batch import BatchedBlocks
    fields = _fields(11)
    bb = BatchedBlocks(SIZES, logE=np.concatenate(fields), precision=precision, tol=1e-7)
    # the mixed engine's inexact-Newton forcing scales each Krylov tolerance by
    # the whole system's ||R||, so packed and separate runs take other (equally
    # converged) iterates; the packing itself is checked with full solves
    bb.solver.engine.newton_forcing = None
    for k in range(3):
        bb.solver.advance_one_step(k, 6)
    d_batch = bb.displacement().cpu().numpy()
    for q, (size, f) in enumerate(zip(SIZES, fields)):
        one = BatchedBlocks([size], logE=f, precision=precision, tol=1e-7)
        one.solver.engine.newton_forcing = None
        for k in range(3):
            one.solver.advance_one_step(k, 6)
        d_one = one.displacement().cpu().numpy()
        assert rel_err(d_batch[bb.instance(q)], d_one) < 1e-9


def test_batched_gradient_is_the_sum_of_instance_gradients(cuda):
    from geowarp_b200.adjoint import DisplacementMisfit
    from geowarp_b200.batch import BatchedBlocks
    fields = _fields(21)
    rng = np.random.default_rng(4)
    bb = BatchedBlocks(SIZES, logE=np.concatenate(fields), tol=1e-9)
    bb.solver.engine.krylov_rtol = 1e-13
    target = torch.tensor(rng.normal(scale=1e-4, size=(bb.n_particles, 2)), device=cuda)
    logE = torch.tensor(np.concatenate(fields), device=cuda, requires_grad=True)
    loss = DisplacementMisfit.apply(logE, bb.solver, target, 6, 2, lambda s: bb.reset_state())
    loss.backward()
    g_batch = logE.grad.detach().cpu().numpy()
    total = 0.0
    for q, (size, f) in enumerate(zip(SIZES, fields)):
        one = BatchedBlocks([size], logE=f, tol=1e-9)
        one.solver.engine.krylov_rtol = 1e-13
        lq = torch.tensor(f, device=cuda, requires_grad=True)
        tq = target[bb.instance(q)].clone()
        l1 = DisplacementMisfit.apply(lq, one.solver, tq, 6, 2, lambda s, o=one: o.reset_state())
        l1.backward()
        total += float(l1)
        assert rel_err(g_batch[bb.instance(q)], lq.grad.detach().cpu().numpy()) < 1e-7
    assert abs(float(loss) - total) <= 1e-9 * abs(total)
