"""Host logic of the benchmark problems and of the benchmark's clock record:
the consolidation column's time schedule and Terzaghi's solution, the 3D
indentation dictionaries, and the filtering of clock samples to the timed
region."""
import numpy as np

from geowarp_b200 import problems


def test_consolidation_increments_grow_geometrically_to_the_end_time():
    H, dx, cv = 10.0, 0.05, 1e-7 * 1e7 * 0.7 / (1.3 * 0.4)
    dt0, t_end = 4.0 * dx * dx / cv, 2.0 * H * H / cv
    d = problems.consolidation_dts(200, dt0, t_end)
    assert d.shape == (200,)
    assert abs(d.sum() - t_end) <= 1e-12 * t_end
    r = d[1:] / d[:-1]
    assert np.allclose(r, r[0], rtol=1e-12) and r[0] > 1.0
    assert abs(d[0] * cv / (dx * dx) - 4.0) < 1e-6         # first mesh Fourier number
    grid, parts, it, mat, porous, load, dts, cv2, H2 = problems.consolidation_column_dicts()
    assert np.array_equal(dts, d) and abs(cv2 - cv) < 1e-12 * cv and H2 == H
    assert parts["n_particles"] == 800 and grid["n_grid_y"] == 202 and it["dt"] == d[0]


def test_terzaghi_pressure_limits():
    H, cv, q = 10.0, 1.3, 1e4
    z = np.linspace(0.0, H, 41)
    early = problems.terzaghi_pressure(z, 1e-6 * H * H / cv, H, cv, q, terms=2000)
    late = problems.terzaghi_pressure(z, 5.0 * H * H / cv, H, cv, q)
    assert abs(early[0]) < 1e-9 * q                          # drained face
    assert np.all(np.abs(early[4:] - q) < 0.02 * q)          # undrained interior at T -> 0
    assert np.all(np.abs(late) < 1e-4 * q)                   # fully consolidated
    mid = problems.terzaghi_pressure(z, 0.2 * H * H / cv, H, cv, q)
    assert np.all(np.diff(mid) >= -1e-9)                     # rises away from the drained face


def test_indentation_dicts_follow_the_block_and_indenter():
    g, p, it, mat, porous, load = problems.indentation_3d_dicts(block_cells=(20, 20, 12), grid_cells=(24, 24, 16),
                                                               indenter=0.1, depth=0.025, n_steps=50)
    assert p["n_particles"] == 20 * 20 * 12 * 8
    assert abs(g["end_z"] - 12 * 0.02) < 1e-12 and abs(g["end_x"] - (0.02 + 20 * 0.02)) < 1e-12
    assert abs(load["footing_region_max_x"] - load["footing_region_min_x"] - 0.1) < 1e-12
    assert abs(load["footing_incr_disp"] + 0.025 / 50) < 1e-15
    assert load["penalty_factor"] == mat["youngs_modulus"]
    assert abs(porous["mobility_constant"] - 1e-9) < 1e-24
    assert mat["material_name"] == "Drucker-Prager" and mat["tension_cutoff"] is False


def test_clock_sampler_keeps_only_the_timed_region(tmp_path):
    import datetime
    import bench
    cs = bench.ClockSampler(0)
    f = tmp_path / "clocks.csv"
    t0 = datetime.datetime(2026, 1, 1, 12, 0, 0)

    def row(sec, mhz, cap="Not Active"):
        stamp = (t0 + datetime.timedelta(seconds=sec)).strftime("%Y/%m/%d %H:%M:%S.%f")[:-3]
        return f"{stamp}, 0, {mhz}, 1965, 900.0, 0x0, Not Active, Not Active, Not Active, {cap}"

    f.write_text("\n".join([row(0.0, 1200), row(1.0, 1965), row(1.5, 1965, "Active"), row(3.0, 1000)]) + "\n")

    class F:
        name = str(f)
    cs.f = F()
    cs.t0 = (t0 + datetime.timedelta(seconds=0.5)).timestamp()
    cs.t1 = (t0 + datetime.timedelta(seconds=2.0)).timestamp()
    out = cs.summary()
    assert out["samples"] == 2 and out["sm_mhz"] == 1965.0 and out["reasons"] == ["sw_power_cap"]
    # a region shorter than the sampling interval keeps the nearest sample, flagged
    f.write_text("\n".join([row(0.0, 1200), row(3.0, 1000)]) + "\n")
    cs.t0 = (t0 + datetime.timedelta(seconds=0.4)).timestamp()
    cs.t1 = (t0 + datetime.timedelta(seconds=0.5)).timestamp()
    out = cs.summary()
    assert out["samples"] == 1 and out["sm_mhz"] == 1200.0 and "nearest" in out["note"]
