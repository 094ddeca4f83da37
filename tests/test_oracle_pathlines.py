"""CPU checks of the oracle's pathlines through time-varying fields (no
counterpart in the reference): frozen slices reproduce the steady
streamlines, the time axis follows the spatial rule, and a field linear in
time matches a numpy restatement step by step."""
import numpy as np

from dpa_b200 import UnsteadyGrid, fields, seeds

f32 = np.float32


def test_frozen_slices_give_the_steady_result(oracle):
    grid = fields.abc(24)
    frozen = UnsteadyGrid.from_data(np.stack([grid.data] * 4), grid.spacing, 0.5, grid.offset,
                                    time_origin=-0.25)
    offset, size = seeds.seed_box(grid)
    pos = seeds.generate_random(offset, size, 300, 0, aabb=([0, 0, 0], [6.2, 6.2, 6.2]),
                                seed=2).position
    for name in ("euler", "runge_kutta_4", "runge_kutta_cash_karp_54", "runge_kutta_4_true"):
        # 55 steps of 0.02 stay inside the span [-0.25, 1.25). The blend of
        # two equal slices, (1 - w) a + w a, is a to within an ulp or two,
        # not always exactly.
        steady = oracle.advect_round(oracle.OracleGrid.of(grid), name, 0.02, pos,
                                     np.full(300, 55, np.uint64))
        path = oracle.advect_pathlines(frozen, name, 0.02, pos, 0.0, np.full(300, 55, np.uint64))
        same = path.termination == steady.termination
        assert same.mean() > 0.98
        np.testing.assert_allclose(path.positions[same], steady.positions[same], rtol=0,
                                   atol=1e-4)
        # Time advances by one rounded addition of dt per step taken.
        for i in range(0, 300, 37):
            t = f32(0.0)
            for _ in range(int(path.steps[i])):
                t = f32(t + f32(0.02))
            assert path.times[i] == t


def test_time_span_ends_particles_out_of_bounds(oracle):
    data = np.zeros((3, 8, 8, 8, 3), np.float32)
    data[..., 2] = 1.0  # +x, everywhere and always
    g = UnsteadyGrid.from_data(data, (1, 1, 1), 0.5, time_origin=1.0)
    # Span [1.0, 2.0): a start at 0.9 is outside; 1.0 takes steps until t = 2.0.
    out = oracle.advect_pathlines(g, "euler", 0.25, [[1, 1, 1], [1, 1, 1]], [0.9, 1.0],
                                  [100, 100])
    assert list(out.termination) == [1, 1]
    assert list(out.steps) == [0, 4]
    assert list(out.times) == [f32(0.9), f32(2.0)]
    np.testing.assert_array_equal(out.positions[1], [2, 1, 1])


def test_linear_in_time_field_matches_numpy(oracle):
    # Slices hold constant fields whose value changes from slice to slice.
    rng = np.random.default_rng(1)
    vals = rng.normal(size=(5, 3)).astype(np.float32) * f32(0.3)
    data = np.broadcast_to(vals[:, None, None, None, :], (5, 16, 16, 16, 3)).copy()
    g = UnsteadyGrid.from_data(data, (1, 1, 1), 0.75)
    starts = np.array([[7.5, 7.5, 7.5], [6.0, 8.0, 7.0]], np.float32)
    out = oracle.advect_pathlines(g, "euler", 0.1, starts, [0.05, 0.33], [20, 20])
    for i in range(2):
        x, t = starts[i].copy(), f32([0.05, 0.33][i])
        for _ in range(20):
            s = int(np.floor(f32(t / f32(0.75))))
            w = f32(np.fmod(t, f32(0.75)) / f32(0.75))
            v = (f32(1) - w) * vals[s] + w * vals[s + 1]
            d = np.array([v[2], v[1], v[0]], np.float32)
            x = (f32(1) * x + f32(0.1) * d).astype(np.float32)
            t = f32(t + f32(0.1))
        np.testing.assert_array_equal(out.positions[i], x)
        assert out.times[i] == t
