"""CPU checks of the oracle against analytic known answers and the reference's
rules. The reference ships no tests or golden vectors and cannot be built
here, so these known answers are what anchor the oracle."""
import math

import numpy as np
import pytest

from dpa_b200 import fields, seeds


def test_contains_rule(oracle):
    # regular_grid.hpp:41-50: 0 <= floor((p - o) / h) <= n - 2 on every axis.
    g = oracle.OracleGrid(np.zeros((8, 8, 8, 3), np.float32), (1, 1, 1))
    assert oracle.contains(g, [0, 0, 0])
    assert oracle.contains(g, [6.999, 0.5, 3])
    assert not oracle.contains(g, [7.0, 0.5, 3])  # cell 7 = n - 1 is outside
    assert not oracle.contains(g, [-1e-6, 0.5, 3])
    assert oracle.contains(g, [-0.0, 0.5, 3])
    assert not oracle.contains(g, [np.nan, 0.5, 3])
    assert not oracle.contains(g, [np.inf, 0.5, 3])
    # An axis of one node has no cell (the reference compares the subscript
    # with shape - 1 = 0), so nothing is inside such a grid.
    flat = oracle.OracleGrid(np.zeros((4, 1, 4, 3), np.float32), (1, 1, 1))
    assert not oracle.contains(flat, [1.0, 0.0, 1.0])
    assert not oracle.contains(flat, [1.0, -0.0, 1.0])
    one = oracle.OracleGrid(np.zeros((2, 2, 2, 3), np.float32), (1, 1, 1))
    assert oracle.contains(one, [0.5, 0.5, 0.999])
    assert not oracle.contains(one, [0.5, 0.5, 1.0])


def test_trilinear_is_exact_on_linear_fields(oracle):
    rng = np.random.default_rng(5)
    grad = rng.normal(size=(3, 3))
    const = rng.normal(size=3)
    grid = fields.linear(9, grad, const, spacing=(0.5, 0.25, 1.0), offset=(1.0, -2.0, 0.5))
    g = oracle.OracleGrid.of(grid)
    pts = grid.offset + rng.random((200, 3)) * (np.asarray(grid.shape) - 1.001) * grid.spacing
    for p in pts.astype(np.float32):
        got = oracle.interpolate(g, p)
        want = const + grad @ p.astype(np.float64)
        np.testing.assert_allclose(got, want, rtol=0, atol=2e-5)


def test_interpolation_uses_fmod_weights_with_floor_start(oracle):
    # A position whose quotient rounds up to an integer: start index from the
    # rounded quotient, weight from the exact fmod (close to 1), as the
    # reference computes them (regular_grid.hpp:58-59).
    h = np.float32(2 * math.pi / 63)
    data = np.zeros((8, 8, 8, 3), np.float32)
    data[..., 0] = np.arange(8, dtype=np.float32)[:, None, None]
    g = oracle.OracleGrid(data, (h, h, h))
    for i in range(1, 6):
        p = np.nextafter(np.float32(h * np.float32(i)), np.float32(0))
        q = np.float32(p / h)
        w = np.float32(np.fmod(p, h) / h)
        s = int(np.floor(q))
        want = np.float32((np.float32(1) - w) * np.float32(s) + w * np.float32(s + 1))
        got = oracle.interpolate(g, [p, np.float32(0.1), np.float32(0.1)])[0]
        assert got == want


def test_constant_field_exit_step(oracle):
    # Constant flow of +1 along x (stored reversed: component 2 drives x), step
    # 0.25 with unit spacing: every position is exact, so the exit step is known.
    n = 16
    data = np.zeros((n, n, n, 3), np.float32)
    data[..., 2] = 1.0
    g = oracle.OracleGrid(data, (1, 1, 1))
    p0 = np.array([[0.5, 3.5, 3.5]], np.float32)
    for integ in ("euler", "runge_kutta_4"):
        r = oracle.advect_round(g, integ, 0.25, p0, [1000], record=True)
        # contained while x < n - 1 = 15: x = 0.5 + 0.25 k, leaves at k = 58.
        assert r.steps[0] == 58
        assert r.termination[0] == 1
        assert r.remaining[0] == 1000 - 58
        assert r.positions[0, 0] == np.float32(0.5 + 0.25 * 58)
        assert r.vertices.shape[0] == 58 + 2
        assert np.all(r.vertices[-1] == -2.0)
        np.testing.assert_array_equal(r.indices[0::2], np.arange(58, dtype=np.uint32))


def test_zero_velocity_and_out_of_bounds_start(oracle):
    g = oracle.OracleGrid(np.zeros((8, 8, 8, 3), np.float32), (1, 1, 1))
    r = oracle.advect_round(g, "runge_kutta_4", 0.1, [[1, 1, 1], [9, 1, 1]], [5, 5], record=True)
    assert list(r.termination) == [2, 1]
    assert list(r.steps) == [0, 0]
    assert list(r.remaining) == [5, 5]  # not decremented on a failed iteration
    assert r.vertices.shape == (4, 3)  # [p0, T, p1, T]
    assert r.indices.size == 0
    assert np.all(r.colors == 0)


def test_is_zero_tolerance_is_eigen_dummy_precision(oracle):
    data = np.zeros((4, 4, 4, 3), np.float32)
    data[..., 2] = np.float32(1e-5)
    g = oracle.OracleGrid(data, (1, 1, 1))
    assert oracle.advect_round(g, "euler", 1.0, [[1, 1, 1]], [3]).termination[0] == 2
    data[..., 2] = np.nextafter(np.float32(1e-5), np.float32(1))
    g = oracle.OracleGrid(data, (1, 1, 1))
    assert oracle.advect_round(g, "euler", 1.0, [[1, 1, 1]], [3]).termination[0] == 0


def test_index_and_color_rules(oracle):
    # Two curves in one round: [a0 a1 a2 T] [b0 b1 T]. Pairs never cross a
    # terminal; color of vertex 1 has no "prev" (vertex_index > 1 rule).
    T = [-2, -2, -2]
    v = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], T, [5, 5, 5], [4, 4, 4], T], np.float32)
    idx = np.zeros(14, np.uint32)
    n = oracle.lib().oracle_generate_indices(oracle._ptr(v), 7, 0, oracle._ptr(idx))
    assert list(idx[:n]) == [0, 1, 1, 2, 4, 5]
    col = np.zeros(7, np.float32)
    oracle.lib().oracle_generate_colors(oracle._ptr(v), 7, oracle._ptr(col))
    assert col[0] == 0.0  # prev zero, next (1,0,0): dot +0 -> atan2(0, +0) = 0
    assert col[1] == 0.0  # index 1: no prev by the reference's rule
    assert col[2] == 0.0  # prev (0,1,0), next zero
    assert col[3] == 0.0  # terminal
    # b0: prev is zero (after a terminal), next = normalize(-1,-1,-1): all
    # products -0 -> dot = -0 -> atan2(+0, -0) = pi.
    assert col[4] == np.float32(math.pi)
    assert col[5] == np.float32(math.pi)  # prev (-1,-1,-1)/sqrt3, next zero: dot -0
    assert col[6] == 0.0


def test_color_right_angle(oracle):
    T = [-2, -2, -2]
    v = np.array([[9, 9, 9], [0, 0, 0], [1, 0, 0], [1, 1, 0], T], np.float32)
    col = np.zeros(5, np.float32)
    oracle.lib().oracle_generate_colors(oracle._ptr(v), 5, oracle._ptr(col))
    assert col[2] == pytest.approx(math.pi / 2, abs=1e-6)


def test_prune_removes_invalid_sentinels(oracle):
    v = np.array([[0, 0, 0], [-1, -1, -1], [1, 2, 3], [-1, -1, 0], [-1, -1, -1]], np.float32)
    kept = oracle.lib().oracle_prune(oracle._ptr(v), 5)
    assert kept == 3
    np.testing.assert_array_equal(v[:3], [[0, 0, 0], [1, 2, 3], [-1, -1, 0]])


def test_lattice_matches_host_generator(oracle):
    grid = fields.abc(33)
    offset, size = seeds.seed_box(grid)
    stride = (grid.spacing * np.float32(2)).astype(np.float32)
    pos, shape = oracle.lattice_seeds(offset, size, stride)
    host = seeds.generate(offset, size, stride, 10)
    assert shape == (16, 16, 16)
    np.testing.assert_array_equal(pos, host.position)
    # last axis fastest
    assert pos[1, 2] > pos[0, 2] and pos[1, 0] == pos[0, 0]
    box = ([0.5, 0.5, 0.5], [2.0, 3.0, 4.0])
    pos2, shape2 = oracle.lattice_seeds(offset, size, stride, box)
    host2 = seeds.generate(offset, size, stride, 10, aabb=box)
    np.testing.assert_array_equal(pos2, host2.position)


def test_ftle_of_linear_flow_map(oracle):
    # Flow map x -> A x on a lattice: interior J = A, so FTLE = ln(sigma_max(A)) / T.
    A = np.array([[2.0, 0.1, 0.0], [0.0, 0.5, 0.0], [0.3, 0.0, 1.0]])
    n, stride = 16, 1.0
    pos, shape = oracle.lattice_seeds([0, 0, 0], [n, n, n], [stride] * 3)
    final = (pos.astype(np.float64) @ A.T).astype(np.float32)
    ftle, info = oracle.ftle((n, n, n), (0, 0, 0), (1, 1, 1), (1, 1, 1), 10, 0.5, pos, final)
    assert info == {"collisions": 0, "holes": 0, "outside": 0}
    sigma = np.linalg.svd(A, compute_uv=False)[0]
    want = math.log(sigma) / 5.0
    np.testing.assert_allclose(ftle[1:-1, 1:-1, 1:-1], want, rtol=1e-5)
    # Border: one-sided difference divided by 2h halves that column of J.
    Ab = A.copy()
    Ab[:, 0] *= 0.5
    want_b = math.log(np.linalg.svd(Ab, compute_uv=False)[0]) / 5.0
    assert ftle[0, 5, 5] == pytest.approx(want_b, rel=1e-5)
    lat, _ = oracle.ftle((n, n, n), (0, 0, 0), (1, 1, 1), (1, 1, 1), 10, 0.5, pos, final, 1)
    np.testing.assert_array_equal(lat, ftle)


def test_ftle_reference_mapping_collisions(oracle):
    # With spacing 2 pi / 255 and stride 2, rounding maps some lattice planes
    # to the previous cell (ftle_estimator.cpp:42), leaving holes.
    n = 256
    h = np.float32(2 * math.pi / (n - 1))
    offset = np.zeros(3, np.float32)
    size = (h * np.float32(n)) * np.ones(3, np.float32)
    stride = (h * np.float32(2)) * np.ones(3, np.float32)
    pos, shape = oracle.lattice_seeds(offset, size, stride)
    assert shape == (128, 128, 128)
    _, info = oracle.ftle((n, n, n), offset, (h, h, h), (2, 2, 2), 250, 0.02, pos, pos)
    assert info["holes"] > 0 and info["collisions"] > 0
    # Planes 51, 97, 102 and 107 land on their predecessors on every axis.
    good = 128 - 4
    assert info["holes"] == 128 ** 3 - good ** 3


def test_fp64_oracle_tracks_analytic_abc(oracle):
    grid = fields.abc(128)
    g = oracle.OracleGrid.of(grid)
    rng = np.random.default_rng(0)
    p0 = (1.0 + rng.random((64, 3)) * 4.0)
    lo, hi = [0, 0, 0], [2 * math.pi * 126 / 127] * 3
    ana = oracle.advect64_abc(math.sqrt(3), math.sqrt(2), 1.0, lo, hi, 0.01, p0, [50] * 64)
    num = oracle.advect64(g, "runge_kutta_4_true", 0.01, p0, [50] * 64)
    ok = (ana.termination == 0) & (num.termination == 0)
    assert ok.sum() > 40
    err = np.abs(ana.positions[ok] - num.positions[ok]).max()
    assert err < 5e-3  # trilinear discretization error at h = 2 pi / 127


def test_fp32_rk4_equals_euler_in_exact_arithmetic(oracle):
    # Reference semantics: four identical stages, so RK4 is Euler up to the
    # rounding of the weighted sum.
    grid = fields.curl_noise(32, 3.0, 7)
    g = oracle.OracleGrid.of(grid)
    rng = np.random.default_rng(1)
    p0 = 4 + rng.random((32, 3)).astype(np.float32) * 20
    a = oracle.advect_round(g, "runge_kutta_4", 0.25, p0, [20] * 32)
    b = oracle.advect_round(g, "euler", 0.25, p0, [20] * 32)
    ok = (a.termination == 0) & (b.termination == 0)
    np.testing.assert_allclose(a.positions[ok], b.positions[ok], atol=1e-3)
