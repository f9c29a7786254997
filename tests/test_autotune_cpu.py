"""Launch-shape knobs and the autotuner's search, on the host: gw_tune_set /
gw_tune_get only touch host state, so the library answers them without a
GPU, and the search is driven by a synthetic cost with a known optimum."""
import pytest

from geowarp_b200 import _lib as L
from geowarp_b200 import autotune

DEFAULTS = {L.TUNE_PARTICLE_BLOCK: 256, L.TUNE_ADJOINT_BLOCK: 128, L.TUNE_ROW_WARPS: 8, L.TUNE_MG_COARSE: 160,
            L.TUNE_MG_ONE_SWEEP: 20, L.TUNE_MG_SWEEPS: 2, L.TUNE_MG_OMEGA: 70, L.TUNE_GS_CANCEL: 20,
            L.TUNE_MG_TAIL: 0, L.TUNE_MG_BF16: 0, L.TUNE_MG_FINE_SWEEPS: 1,
            L.TUNE_GMRES_STALL: 50}


@pytest.fixture
def lib():
    lib = L.load()
    yield lib
    for k, v in DEFAULTS.items():
        assert lib.gw_tune_set(k, v) == L.GW_OK


def test_knob_defaults_and_ranges(lib):
    for k, v in DEFAULTS.items():
        assert lib.gw_tune_get(k) == v
    assert lib.gw_tune_get(L.TUNE_COUNT) == -1
    bad = [(L.TUNE_PARTICLE_BLOCK, 288), (L.TUNE_PARTICLE_BLOCK, 48), (L.TUNE_ADJOINT_BLOCK, 0),
           (L.TUNE_ROW_WARPS, 0), (L.TUNE_ROW_WARPS, 33), (L.TUNE_MG_COARSE, 7), (L.TUNE_MG_COARSE, 161),
           (L.TUNE_MG_ONE_SWEEP, 0), (L.TUNE_MG_ONE_SWEEP, 21), (L.TUNE_MG_SWEEPS, 5), (L.TUNE_MG_OMEGA, 101),
           (L.TUNE_GS_CANCEL, -1), (L.TUNE_GS_CANCEL, 301), (L.TUNE_MG_TAIL, -1), (L.TUNE_MG_TAIL, (1 << 20) + 1),
           (L.TUNE_MG_BF16, 2), (L.TUNE_MG_FINE_SWEEPS, 0), (L.TUNE_MG_FINE_SWEEPS, 5),
           (L.TUNE_GMRES_STALL, -1), (L.TUNE_GMRES_STALL, 100001),
           (L.TUNE_COUNT, 1)]
    for k, v in bad:
        assert lib.gw_tune_set(k, v) == L.GW_EINVAL, (k, v)
        if k != L.TUNE_COUNT:
            assert lib.gw_tune_get(k) == DEFAULTS[k]  # a rejected value leaves the knob alone
    for k, v in [(L.TUNE_PARTICLE_BLOCK, 64), (L.TUNE_ADJOINT_BLOCK, 256), (L.TUNE_ROW_WARPS, 2),
                 (L.TUNE_MG_COARSE, 40), (L.TUNE_MG_ONE_SWEEP, 2)]:
        assert lib.gw_tune_set(k, v) == L.GW_OK
        assert lib.gw_tune_get(k) == v


def test_coordinate_search_finds_the_separable_optimum(lib):
    target = {"row_warps": 4, "mg_coarse": 80, "particle_block": 128, "adjoint_block": 64}

    def cost():
        cfg = autotune.current()
        return sum((cfg[n] - target[n]) ** 2 / float(target[n] or 1) for n in target) + 1.0

    calls = []
    best, table = autotune.tune(lambda: calls.append(1), reps=3, timer=lambda fn: (fn(), cost())[1])
    assert best == target
    assert autotune.current() == target          # the winners stay set
    assert set(table) == set(autotune.KNOBS)
    n_cands = sum(len(c) for _, c in autotune.KNOBS.values())
    assert len(calls) == n_cands * 4             # one untimed + three timed trials per candidate


def test_snapshot_restores_particle_state_and_newton_predictor():
    """A restored load step repeats the one it was taken before: the snapshot
    holds the particle state and the Newton predictor (the previous converged
    increment and its load step), and restoring hands the engine a copy, so the
    step run after it cannot overwrite the snapshot."""
    import types

    import torch
    eng = types.SimpleNamespace(**{n: torch.arange(6, dtype=torch.float64) + i for i, n in enumerate(autotune.STATE)})
    eng._u_prev = torch.full((4,), 2.0, dtype=torch.float64)
    eng._u_prev_step = 4
    snap = autotune.snapshot(eng)
    for n in autotune.STATE:
        getattr(eng, n).add_(100.0)
    eng._u_prev.fill_(-1.0)
    eng._u_prev_step = 5
    autotune.restore(eng, snap)
    for i, n in enumerate(autotune.STATE):
        assert torch.equal(getattr(eng, n), torch.arange(6, dtype=torch.float64) + i)
    assert eng._u_prev_step == 4 and torch.equal(eng._u_prev, torch.full((4,), 2.0, dtype=torch.float64))
    eng._u_prev.fill_(7.0)  # the next step's hold writes into the engine's copy only
    autotune.restore(eng, snap)
    assert torch.equal(eng._u_prev, torch.full((4,), 2.0, dtype=torch.float64))

    # an engine without a held increment restores to none
    eng._u_prev, eng._u_prev_step = None, None
    snap = autotune.snapshot(eng)
    eng._u_prev, eng._u_prev_step = torch.zeros(4), 3
    autotune.restore(eng, snap)
    assert eng._u_prev is None and eng._u_prev_step is None
