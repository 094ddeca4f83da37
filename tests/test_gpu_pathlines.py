"""Pathlines through a time-varying field on the GPU (dpa_advect_pathlines_device
and the request server), bit-exact against the oracle's pathlines."""
import ctypes as C

import numpy as np
import pytest

import dpa_b200
from dpa_b200 import _native as N
from dpa_b200 import advect_pathlines, fields, seeds
from dpa_b200.serve import Server
from bitwise import assert_same

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gyre(ctx):
    grid = fields.double_gyre((64, 32, 32), slices=8)
    f32 = ctx.field(grid)
    f16 = ctx.field(grid, "f16")
    yield grid, f32, f16
    f32.close()
    f16.close()


def _seeds(n, seed):
    rng = np.random.default_rng(seed)
    lo = np.array([0.02, 0.02, 0.02])
    hi = np.array([1.98, 0.98, 0.98])
    return (lo + rng.random((n, 3)) * (hi - lo)).astype(np.float32)


def _check(got, want):
    assert_same(got.termination, want.termination)
    assert_same(got.remaining_iterations, want.remaining)
    assert_same(got.position, want.positions)
    assert_same(got.time, want.times)


@pytest.mark.parametrize("integrator", ["runge_kutta_4", "euler", "runge_kutta_4_true",
                                        "runge_kutta_cash_karp_54", "adams_bashforth_2",
                                        "runge_kutta_dormand_prince_5"])
def test_pathlines_match_the_oracle(ctx, oracle, gyre, integrator):
    grid, field, _ = gyre
    pos = _seeds(4000, 1)
    starts = np.random.default_rng(2).uniform(0.0, 6.0, 4000).astype(np.float32)
    # Step 0.05 for up to 150 steps: some particles run past the last slice
    # (time 10), some leave through the walls, the rest complete.
    want = oracle.advect_pathlines(grid, integrator, 0.05, pos, starts, np.full(4000, 150, np.uint64))
    got = advect_pathlines(ctx, field, pos, starts, 150, integrator, 0.05)
    _check(got, want)
    assert set(np.unique(want.termination)) >= {0, 1}


def test_half_storage_pathlines_match_the_rounded_field(ctx, oracle, gyre):
    grid, _, field = gyre
    rounded = dpa_b200.UnsteadyGrid.from_data(grid.data.astype(np.float16).astype(np.float32),
                                              grid.spacing, grid.time_spacing, grid.offset,
                                              grid.time_origin)
    pos = _seeds(3000, 3)
    want = oracle.advect_pathlines(rounded, "runge_kutta_4", 0.05, pos, 1.0,
                                   np.full(3000, 120, np.uint64))
    got = advect_pathlines(ctx, field, pos, 1.0, 120, "runge_kutta_4", 0.05)
    _check(got, want)


def test_edge_record_pathlines_match_the_oracle(ctx, oracle, gyre):
    grid = gyre[0]
    field = ctx.field(grid, "f32_edges")
    try:
        pos = _seeds(3000, 6)
        want = oracle.advect_pathlines(grid, "runge_kutta_4", 0.05, pos, 0.5,
                                       np.full(3000, 120, np.uint64))
        got = advect_pathlines(ctx, field, pos, 0.5, 120, "runge_kutta_4", 0.05)
        _check(got, want)
    finally:
        field.close()


def test_step_budgets_resume_at_the_stored_time(ctx, oracle, gyre):
    grid, field, _ = gyre
    pos = _seeds(2000, 4)
    want = oracle.advect_pathlines(grid, "runge_kutta_4_true", 0.05, pos, 0.5,
                                   np.full(2000, 90, np.uint64))
    import torch
    p = torch.from_numpy(pos).cuda()
    t = torch.full((2000,), 0.5, dtype=torch.float32, device="cuda")
    r = torch.full((2000,), 90, dtype=torch.int64, device="cuda")
    term = torch.zeros(2000, dtype=torch.uint8, device="cuda")
    opts = N.AdvectOptions(N.INTEGRATORS["runge_kutta_4_true"], 0.05, 0, 0, 0, 1, 13)
    ptr = lambda x: C.c_void_p(x.data_ptr())
    for _ in range(20):
        ctx.check(ctx._lib.dpa_advect_pathlines_device(ctx.handle, field.handle, C.byref(opts),
                                                       2000, ptr(p), ptr(t), ptr(r), ptr(term),
                                                       None))
        ctx.synchronize()
        if not np.any(term.cpu().numpy() == 3):
            break
    assert_same(p.cpu().numpy(), want.positions)
    assert_same(t.cpu().numpy(), want.times)
    assert_same(term.cpu().numpy(), want.termination)


def test_steady_calls_refuse_a_time_varying_field(ctx, gyre):
    grid, field, _ = gyre
    adv = dpa_b200.ParticleAdvector(ctx, 10, "none", "runge_kutta_4", 0.05, False, False)
    with pytest.raises(dpa_b200.DpaError) as e:
        adv.advect(field, dpa_b200.Particles.create(_seeds(10, 5), 5))
    assert e.value.status == 1
    slices = C.c_uint32()
    t0, dt = C.c_float(), C.c_float()
    ctx.check(ctx._lib.dpa_field_time_info(field.handle, C.byref(slices), C.byref(t0), C.byref(dt)))
    assert (slices.value, t0.value, dt.value) == (8, 0.0, np.float32(10.0 / 7))


def test_served_pathlines_match_the_direct_call(ctx, gyre):
    grid, field, _ = gyre
    noise = fields.curl_noise(32, 3.0, 9)
    steady = ctx.field(noise)
    offset, size = seeds.seed_box(noise)
    with Server(ctx, particle_capacity=30000, vertex_capacity=2_000_000, steps_per_tick=24,
                max_requests=8) as server:
        g = server.add_field(field)
        n = server.add_field(steady)
        plan = [(g, _seeds(5000, 6), 2.5, 200, False), (n, None, 0.0, 150, False),
                (g, _seeds(300, 7), 7.25, 100, True), (g, _seeds(8000, 8), 0.0, 60, False)]
        ids = {}
        for fid, pos, t0, iters, record in plan:
            if pos is None:
                pos = seeds.generate_random(offset, size, 4000, 0, seed=3).position
            ids[server.submit(fid, pos, iters, "runge_kutta_4", 0.05, record, start_time=t0)] = (
                fid, pos, t0, iters, record)
        results = {}
        while len(results) < len(plan):
            res = server.poll(wait_ms=5000)
            assert res is not None
            results[res.id] = res
    for rid, (fid, pos, t0, iters, record) in ids.items():
        res = results[rid]
        f = field if fid == g else steady
        want = advect_pathlines(ctx, f, pos, t0, iters, "runge_kutta_4", 0.05)
        assert_same(res.positions, want.position)
        assert_same(res.times, want.time)
        assert_same(res.termination, want.termination)
        if record:
            assert res.vertices.shape[0] > len(pos)
            assert_same(res.vertices[0], pos[0])
    steady.close()
