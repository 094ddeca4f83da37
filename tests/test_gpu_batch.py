"""Step budgets (resumable launches), batched seed sets, CUDA-graph replay and
the autotuner: every form must give the bit-identical results of one plain
dpa_advect_device call."""
import ctypes as C

import numpy as np
import pytest

import dpa_b200
from dpa_b200 import _native as N
from dpa_b200 import fields, seeds
from bitwise import assert_same

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup(ctx):
    import torch
    grid = fields.curl_noise(64, 4.0, 21)
    field = ctx.field(grid)
    offset, size = seeds.seed_box(grid)
    pos = seeds.generate_random(offset, size, 20000, 1, seed=31).position
    rng = np.random.default_rng(3)
    rem = rng.integers(0, 500, size=20000).astype(np.int64)
    p0 = torch.from_numpy(pos).cuda()
    r0 = torch.from_numpy(rem).cuda()
    yield grid, field, p0, r0
    field.close()


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def reference_run(ctx, field, p0, r0, integrator="runge_kutta_4"):
    import torch
    pos, rem = p0.clone(), r0.clone()
    term = torch.zeros(p0.shape[0], dtype=torch.uint8, device="cuda")
    opts = N.AdvectOptions(N.INTEGRATORS[integrator], 0.25, 0, 0, 0, 1, 0)
    ctx.check(ctx._lib.dpa_advect_device(ctx.handle, field.handle, C.byref(opts), p0.shape[0],
                                         _ptr(pos), _ptr(rem), _ptr(term), None))
    ctx.synchronize()
    return pos.cpu().numpy(), rem.cpu().numpy(), term.cpu().numpy()


def test_step_budget_resumes_to_the_same_result(ctx, setup):
    import torch
    grid, field, p0, r0 = setup
    want = reference_run(ctx, field, p0, r0)
    pos, rem = p0.clone(), r0.clone()
    term = torch.zeros(p0.shape[0], dtype=torch.uint8, device="cuda")
    opts = N.AdvectOptions(N.INTEGRATORS["runge_kutta_4"], 0.25, 0, 0, 0, 1, 37)
    launches = 0
    while True:
        ctx.check(ctx._lib.dpa_advect_device(ctx.handle, field.handle, C.byref(opts),
                                             p0.shape[0], _ptr(pos), _ptr(rem), _ptr(term), None))
        ctx.synchronize()
        launches += 1
        t = term.cpu().numpy()
        if not np.any(t == 3):
            break
        assert launches < 100
    assert launches >= 500 // 37
    assert_same(pos.cpu().numpy(), want[0])
    assert_same(rem.cpu().numpy(), want[1])
    assert_same(term.cpu().numpy(), want[2])


def test_batched_sets_match_one_call(ctx, setup):
    grid, field, p0, r0 = setup
    want = reference_run(ctx, field, p0, r0)
    offsets = np.array([0, 10, 3000, 3000, 12345, 20000], np.uint64)
    pos, rem = p0.clone(), r0.clone()
    import torch
    term = torch.zeros(p0.shape[0], dtype=torch.uint8, device="cuda")
    steps = np.zeros(5, np.uint64)
    opts = N.AdvectOptions(N.INTEGRATORS["runge_kutta_4"], 0.25, 0, 0, 0, 1, 0)
    ctx.check(ctx._lib.dpa_advect_batch_device(
        ctx.handle, field.handle, C.byref(opts), 5, offsets.ctypes.data_as(N._U64P), _ptr(pos),
        _ptr(rem), _ptr(term), steps.ctypes.data_as(N._U64P), None))
    ctx.synchronize()
    assert_same(pos.cpu().numpy(), want[0])
    taken = r0.cpu().numpy() - want[1]
    for s in range(5):
        assert steps[s] == taken[offsets[s]:offsets[s + 1]].sum()


def test_graph_replay_matches_one_call(ctx, setup):
    import torch
    grid, field, p0, r0 = setup
    want = reference_run(ctx, field, p0, r0)
    pos, rem = p0.clone(), r0.clone()
    term = torch.zeros(p0.shape[0], dtype=torch.uint8, device="cuda")
    opts = N.AdvectOptions(N.INTEGRATORS["runge_kutta_4"], 0.25, 0, 0, 0, 1, 0)
    graph = C.c_void_p()
    ctx.check(ctx._lib.dpa_graph_create_advect(ctx.handle, field.handle, C.byref(opts),
                                               p0.shape[0], _ptr(pos), _ptr(rem), _ptr(term),
                                               C.byref(graph)))
    for _ in range(2):
        pos.copy_(p0)
        rem.copy_(r0)
        torch.cuda.synchronize()
        ctx.check(ctx._lib.dpa_graph_launch(ctx.handle, graph, None))
        ctx.synchronize()
        assert_same(pos.cpu().numpy(), want[0])
        assert_same(term.cpu().numpy(), want[2])
    ctx.check(ctx._lib.dpa_graph_destroy(ctx.handle, graph))


def test_graph_replays_after_a_larger_call_on_its_context(ctx, setup):
    # A graph keeps its own scratch: a call on the same context with four
    # times the particles (which regrows the context's scratch) between two
    # replays changes neither replay.
    import torch
    grid, field, p0, r0 = setup
    want = reference_run(ctx, field, p0, r0)
    pos, rem = p0.clone(), r0.clone()
    term = torch.zeros(p0.shape[0], dtype=torch.uint8, device="cuda")
    opts = N.AdvectOptions(N.INTEGRATORS["runge_kutta_4"], 0.25, 0, 0, 0, 1, 0)
    graph = C.c_void_p()
    ctx.check(ctx._lib.dpa_graph_create_advect(ctx.handle, field.handle, C.byref(opts),
                                               p0.shape[0], _ptr(pos), _ptr(rem), _ptr(term),
                                               C.byref(graph)))
    big_want = None
    for _ in range(2):
        pos.copy_(p0)
        rem.copy_(r0)
        torch.cuda.synchronize()
        ctx.check(ctx._lib.dpa_graph_launch(ctx.handle, graph, None))
        ctx.synchronize()
        assert_same(pos.cpu().numpy(), want[0])
        assert_same(rem.cpu().numpy(), want[1])
        assert_same(term.cpu().numpy(), want[2])
        big = reference_run(ctx, field, p0.repeat(4, 1), r0.repeat(4))
        if big_want is None:
            big_want = big
        for x, y in zip(big, big_want):
            assert_same(x, y)
    for x, y in zip(big_want, want):
        assert_same(x, np.concatenate([y] * 4))
    ctx.check(ctx._lib.dpa_graph_destroy(ctx.handle, graph))


def test_autotune_keeps_results_identical(ctx, setup):
    grid, field, p0, r0 = setup
    want = reference_run(ctx, field, p0, r0)
    saved = N.Tuning()
    ctx.check(ctx._lib.dpa_context_get_tuning(ctx.handle, C.byref(saved)))
    best = N.Tuning()
    opts = N.AdvectOptions(N.INTEGRATORS["runge_kutta_4"], 0.25, 0, 0, 0, 1, 0)
    ctx.check(ctx._lib.dpa_autotune_advect(ctx.handle, field.handle, C.byref(opts), p0.shape[0],
                                           _ptr(p0), _ptr(r0), 100, C.byref(best)))
    assert best.claim in (16, 32) and best.order in (0, 16, 64)
    assert best.measured_ms > 0
    got = reference_run(ctx, field, p0, r0)
    for g, w in zip(got, want):
        assert_same(g, w)
    bad = N.Tuning(0, 0, 16, 0.0)
    with pytest.raises(dpa_b200.DpaError):
        ctx.check(ctx._lib.dpa_context_set_tuning(ctx.handle, C.byref(bad)))
    ctx.check(ctx._lib.dpa_context_set_tuning(ctx.handle, C.byref(saved)))


@pytest.fixture(scope="module")
def many(ctx, oracle):
    # More particles than resident lanes, every one starting inside the grid.
    import torch
    grid = fields.curl_noise(64, 4.0, 22)
    field = ctx.field(grid)
    offset, size = seeds.seed_box(grid)
    n = 400_000
    pos = seeds.generate_random(offset, size, n, 1, aabb=([0, 0, 0], [63, 63, 63]), seed=5).position
    want = oracle.advect_round(oracle.OracleGrid.of(grid), "runge_kutta_4", 0.25, pos,
                               np.full(n, 60, np.uint64))
    yield field, torch.from_numpy(pos).cuda(), torch.full((n,), 60, dtype=torch.int64,
                                                          device="cuda"), want
    field.close()


@pytest.mark.parametrize("claim,blocks,order", [(32, 0, 16), (16, 1, 64), (4, 2, 0),
                                                (128, 0, 8), (16, 0, 33), (64, 3, 1)])
def test_results_do_not_depend_on_launch_parameters(ctx, many, claim, blocks, order):
    # Claims smaller and larger than a warp, small grids, every processing order.
    field, pos, rem, want = many
    saved = N.Tuning()
    ctx.check(ctx._lib.dpa_context_get_tuning(ctx.handle, C.byref(saved)))
    assert (saved.claim, saved.blocks_per_sm, saved.order) == (16, 0, 64)
    t = N.Tuning(claim, blocks, order, 0.0)
    ctx.check(ctx._lib.dpa_context_set_tuning(ctx.handle, C.byref(t)))
    try:
        got = reference_run(ctx, field, pos, rem)
    finally:
        ctx.check(ctx._lib.dpa_context_set_tuning(ctx.handle, C.byref(saved)))
    assert_same(got[0], want.positions)
    assert_same(got[1].astype(np.uint64), want.remaining)
    assert_same(got[2], want.termination)


def test_host_round_with_step_budget_reports_in_flight(ctx, setup):
    grid, field, p0, r0 = setup
    pos = p0.cpu().numpy()[:100].copy()
    rem = np.full(100, 50, np.uint64)
    term = np.zeros(100, np.uint8)
    opts = N.AdvectOptions(N.INTEGRATORS["euler"], 0.25, 0, 0, 0, 1, 10)
    ctx.check(ctx._lib.dpa_advect_round(ctx.handle, field.handle, C.byref(opts), 100,
                                        pos.ctypes.data_as(C.c_void_p),
                                        rem.ctypes.data_as(C.c_void_p),
                                        term.ctypes.data_as(C.c_void_p), N.CURVE_SINK(), None))
    assert set(np.unique(term)) <= {1, 2, 3}
    assert np.all(rem[term == 3] == 40)
    opts = N.AdvectOptions(N.INTEGRATORS["euler"], 0.25, 1, 0, 1, 1, 10)
    assert ctx._lib.dpa_advect_round(ctx.handle, field.handle, C.byref(opts), 100,
                                     pos.ctypes.data_as(C.c_void_p),
                                     rem.ctypes.data_as(C.c_void_p), None, N.CURVE_SINK(),
                                     None) == 1
