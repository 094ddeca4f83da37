"""The request server: every result is the same alone and in a mix of
concurrent requests (bit for bit), requests that do not fit wait for room,
and requests that can never fit are refused. The mix holds requests of 4096
seeds or more, which the server sweeps in the Morton order of their seeds,
and smaller ones, swept in submission order."""
import time

import numpy as np
import pytest

import dpa_b200
from dpa_b200 import ParticleAdvector, Particles, fields, seeds
from dpa_b200.serve import Server
from bitwise import assert_same

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def resident(ctx):
    abc = fields.abc(48)
    noise = fields.curl_noise(64, 4.0, 8)
    f_abc = ctx.field(abc)
    f_noise = ctx.field(noise)
    yield {"abc": (abc, f_abc), "noise": (noise, f_noise)}
    f_abc.close()
    f_noise.close()


def alone(ctx, field, positions, iterations, integrator, step, record):
    adv = ParticleAdvector(ctx, max(len(positions), 1), "none", integrator, step, False, record,
                           use_64_bit_indices=False)
    return adv.advect(field, Particles.create(positions, iterations))


def make_requests(resident):
    rng = np.random.default_rng(11)
    reqs = []
    for i in range(14):
        name = "abc" if i % 2 else "noise"
        grid, field = resident[name]
        offset, size = seeds.seed_box(grid)
        count = int(rng.integers(50, 6000))
        iters = int(rng.integers(20, 300))
        step = 0.02 if name == "abc" else 0.25
        record = bool(i % 3 == 0)
        integ = ["runge_kutta_4", "euler", "runge_kutta_4"][i % 3]
        pos = seeds.generate_random(offset, size, count, iters, seed=100 + i).position
        reqs.append(dict(name=name, positions=pos, iterations=iters, step=step, record=record,
                         integrator=integ))
    return reqs


def test_results_are_the_same_alone_and_in_the_mix(ctx, resident):
    reqs = make_requests(resident)
    with Server(ctx, particle_capacity=40000, vertex_capacity=4_000_000, steps_per_tick=32,
                max_requests=64) as server:
        ids = {}
        fid = {name: server.add_field(f) for name, (_, f) in resident.items()}
        for r in reqs:
            rid = server.submit(fid[r["name"]], r["positions"], r["iterations"], r["integrator"],
                                r["step"], r["record"])
            ids[rid] = r
        results = {}
        while len(results) < len(reqs):
            res = server.poll(wait_ms=2000)
            assert res is not None, server.stats()
            results[res.id] = res
        stats = server.stats()
    assert stats["completed"] == len(reqs) and stats["ticks"] > 1
    # Where admission and the finishers spent their time.
    assert 0 < stats["peak_slots"] <= 40000 and stats["peak_vertices"] <= 4_000_000
    assert stats["peak_finishing"] >= 1 and stats["finish_seconds"] > 0
    for rid, r in ids.items():
        res = results[rid]
        assert res.status == 0
        want = alone(ctx, resident[r["name"]][1], r["positions"], r["iterations"],
                     r["integrator"], r["step"], r["record"])
        assert_same(res.positions, want.inactive_particles.position)
        assert_same(res.termination, want.inactive_particles.termination)
        assert_same(res.remaining, want.inactive_particles.remaining_iterations)
        if r["record"]:
            curve = want.integral_curves[0]
            assert_same(res.vertices, curve.vertices)
            assert_same(res.indices, curve.indices)
            assert_same(res.colors, curve.colors)
        assert res.queued <= res.admitted <= res.finished


def test_ftle_request_matches_the_stage_api(ctx, resident):
    grid, field = resident["abc"]
    offset, size = seeds.seed_box(grid)
    stride = (grid.spacing * np.float32(2)).astype(np.float32)
    lattice = seeds.generate(offset, size, stride, 30)
    with Server(ctx, particle_capacity=20000, steps_per_tick=16, max_requests=4) as server:
        fid = server.add_field(field)
        server.submit(fid, lattice.position, 30, step_size=0.02, ftle=True,
                      seed_stride=(2, 2, 2))
        res = server.poll(wait_ms=5000)
    assert res is not None and res.status == 0
    out = alone(ctx, field, lattice.position, 30, "runge_kutta_4", 0.02, False)
    want = dpa_b200.estimate_ftle(ctx, field, 30, (2, 2, 2), 0.02, out.inactive_particles)
    assert_same(res.ftle, want.data)


def test_admission_waits_for_room_and_refuses_what_never_fits(ctx, resident):
    grid, field = resident["noise"]
    offset, size = seeds.seed_box(grid)
    with Server(ctx, particle_capacity=5000, vertex_capacity=100_000, steps_per_tick=64,
                max_requests=2) as server:
        fid = server.add_field(field)
        with pytest.raises(dpa_b200.DpaError) as e:
            server.submit(fid, np.zeros((6000, 3), np.float32), 10)
        assert e.value.status == 3
        with pytest.raises(dpa_b200.DpaError):
            server.submit(fid, np.zeros((1000, 3), np.float32), 200, record=True)
        ids = [server.submit(fid, seeds.generate_random(offset, size, 3000, 50, seed=s).position,
                             50) for s in range(5)]
        got = []
        while len(got) < 5:
            res = server.poll(wait_ms=5000)
            assert res is not None
            got.append(res)
    assert sorted(r.id for r in got) == sorted(ids)
    # 3000-particle requests in a 5000-slot arena run one at a time, in order.
    order = [r.id for r in sorted(got, key=lambda r: r.admitted)]
    assert order == sorted(ids)


@pytest.mark.timeout(300)
def test_many_concurrent_requests_all_complete(ctx, resident):
    # Many requests whose particles leave the grid at very different steps,
    # small ticks and an arena under a fifth of the plan's particles, so that
    # slot ranges are reused while ticks run: every request must complete
    # with the results it has alone, and with its counter exact.
    grid, field = resident["noise"]
    offset, size = seeds.seed_box(grid)
    pool = seeds.generate_random(offset, size, 200_000, 0, seed=77).position
    rng = np.random.default_rng(5)
    plan = []
    for i in range(80):
        count = int(np.exp(rng.uniform(np.log(50), np.log(50_000))))
        start = int(rng.integers(0, len(pool) - count))
        plan.append((pool[start:start + count], int(rng.integers(10, 800)), bool(i % 4 == 0)))
    assert sum(len(p) for p, _, _ in plan) > 5 * 90_000
    with Server(ctx, particle_capacity=90_000, vertex_capacity=30_000_000, steps_per_tick=16,
                max_requests=32) as server:
        fid = server.add_field(field)
        ids = {}
        for pos, iters, record in plan:
            if record and len(pos) * (iters + 2) > 30_000_000:
                record = False
            ids[server.submit(fid, pos, iters, record=record)] = (pos, iters, record)
        got = {}
        deadline = time.time() + 240
        while len(got) < len(plan) and time.time() < deadline:
            r = server.poll(wait_ms=100)
            if r is not None:
                got[r.id] = r
        stats = server.stats()
    assert len(got) == len(plan), stats
    for rid in ids:
        pos, iters, record = ids[rid]
        want = alone(ctx, field, pos, iters, "runge_kutta_4", 0.25, record)
        assert_same(got[rid].positions, want.inactive_particles.position)
        assert_same(got[rid].termination, want.inactive_particles.termination)
        assert got[rid].particle_steps == int(
            (iters - want.inactive_particles.remaining_iterations.astype(np.int64)).sum())


def test_server_takes_memoryless_steppers_and_refuses_the_others(ctx, resident):
    grid, field = resident["abc"]
    offset, size = seeds.seed_box(grid)
    pos = seeds.generate_random(offset, size, 500, 80, seed=8).position
    with Server(ctx, particle_capacity=5000, vertex_capacity=1_000_000, steps_per_tick=16,
                max_requests=4) as server:
        fid = server.add_field(field)
        for name in ("runge_kutta_dormand_prince_5", "adams_bashforth_2",
                     "adams_bashforth_moulton_2"):
            with pytest.raises(dpa_b200.DpaError) as e:
                server.submit(fid, pos, 80, name, 0.02)
            assert e.value.status == 2
        server.submit(fid, pos, 80, "runge_kutta_cash_karp_54", 0.02, record=True)
        res = server.poll(wait_ms=5000)
    assert res is not None and res.status == 0
    want = alone(ctx, field, pos, 80, "runge_kutta_cash_karp_54", 0.02, True)
    assert_same(res.positions, want.inactive_particles.position)
    assert_same(res.vertices, want.integral_curves[0].vertices)


def test_deadlines_and_cancels_drop_requests_and_spare_the_rest(ctx, resident):
    """Failure handling on the host: a running request past its deadline, a
    waiting request past its deadline and a cancelled request come back with
    DPA_ERROR_TIMEOUT / DPA_ERROR_CANCELLED between ticks (no kernel waits
    on the host), while the other requests of the mix finish bit-exact with
    their results alone. Short tick budgets keep the long requests in flight
    across many ticks."""
    grid, field = resident["noise"]
    offset, size = seeds.seed_box(grid)
    box = ([0.0] * 3, [float(s - 1) for s in grid.shape])
    long_pos = seeds.generate_random(offset, size, 20000, 0, aabb=box, seed=61).position
    small = [seeds.generate_random(offset, size, 300 + 50 * i, 0, aabb=box, seed=70 + i).position
             for i in range(4)]
    with Server(ctx, particle_capacity=30000, vertex_capacity=0, steps_per_tick=8,
                max_requests=16, max_bypass_ms=5000) as server:
        fid = server.add_field(field)
        # Runs (many ticks of 8 steps) past its 30 ms deadline.
        timed_out = server.submit(fid, long_pos, 200000, step_size=0.01, deadline_ms=30)
        # No room while the long request runs; its deadline passes in the queue.
        waiting = server.submit(fid, long_pos[:15000], 100, deadline_ms=10)
        cancelled = server.submit(fid, small[0], 10_000_000, step_size=0.001)
        keep = [server.submit(fid, s, 150) for s in small[1:]]
        time.sleep(0.05)
        assert server.cancel(cancelled)
        assert not server.cancel(123456)
        results = {}
        while len(results) < 3 + len(keep):
            res = server.poll(wait_ms=5000)
            assert res is not None, server.stats()
            results[res.id] = res
        assert not server.cancel(keep[0])  # already returned
    r = results[timed_out]
    assert r.status == 7  # DPA_ERROR_TIMEOUT, dropped while running
    assert r.positions.shape == (20000, 3)
    assert (r.termination == 4).any() and r.particle_steps > 0
    assert r.vertices is None and r.ftle is None
    assert results[waiting].status == 7 and results[waiting].positions.shape == (0, 3)
    assert results[cancelled].status == 8  # DPA_ERROR_CANCELLED
    for rid, s in zip(keep, small[1:]):
        assert results[rid].status == 0
        want = alone(ctx, field, s, 150, "runge_kutta_4", 0.25, False)
        assert_same(results[rid].positions, want.inactive_particles.position)
        assert_same(results[rid].termination,
                                      want.inactive_particles.termination)


def test_small_requests_pass_a_large_one_that_waits_for_room(ctx, resident):
    """Admission scans the queue: while a large request waits for slots, the
    small requests behind it that fit start (and finish) before it, and each
    result is the same as alone."""
    grid, field = resident["noise"]
    offset, size = seeds.seed_box(grid)
    box = ([0.0] * 3, [float(s - 1) for s in grid.shape])
    big = seeds.generate_random(offset, size, 12000, 0, aabb=box, seed=81).position
    small = [seeds.generate_random(offset, size, 200, 0, aabb=box, seed=90 + i).position
             for i in range(3)]
    with Server(ctx, particle_capacity=20000, vertex_capacity=0, steps_per_tick=8,
                max_requests=16, small_request_seeds=1000, reserved_percent=10,
                max_bypass_ms=10000) as server:
        fid = server.add_field(field)
        first = server.submit(fid, big, 3000, step_size=0.01)   # runs
        second = server.submit(fid, big, 300, step_size=0.01)   # no room: waits
        smalls = [server.submit(fid, s, 100) for s in small]    # pass it
        order = []
        results = {}
        while len(results) < 2 + len(smalls):
            res = server.poll(wait_ms=5000)
            assert res is not None, server.stats()
            results[res.id] = res
            order.append(res.id)
    assert order.index(second) > max(order.index(s) for s in smalls)
    assert all(results[s].admitted < results[second].admitted for s in smalls)
    for rid, s in zip(smalls, small):
        want = alone(ctx, field, s, 100, "runge_kutta_4", 0.25, False)
        assert_same(results[rid].positions, want.inactive_particles.position)
    want = alone(ctx, field, big, 300, "runge_kutta_4", 0.01, False)
    assert_same(results[second].positions, want.inactive_particles.position)


def test_an_overdue_request_holds_large_ones_and_lets_small_ones_pass(ctx, resident):
    """Once the oldest waiting request is past max_bypass_ms, a younger large
    request that would fit waits behind it, while small requests still pass
    within the reserved share; results are the same as alone."""
    grid, field = resident["noise"]
    offset, size = seeds.seed_box(grid)
    box = ([0.0] * 3, [float(s - 1) for s in grid.shape])
    big = seeds.generate_random(offset, size, 12000, 0, aabb=box, seed=81).position
    mid = seeds.generate_random(offset, size, 1500, 0, aabb=box, seed=82).position
    small = [seeds.generate_random(offset, size, 200, 0, aabb=box, seed=90 + i).position
             for i in range(3)]
    with Server(ctx, particle_capacity=20000, vertex_capacity=0, steps_per_tick=8,
                max_requests=16, small_request_seeds=1000, reserved_percent=10,
                max_bypass_ms=1) as server:
        fid = server.add_field(field)
        first = server.submit(fid, big, 30000, step_size=0.01)  # runs
        second = server.submit(fid, big, 300, step_size=0.01)   # no room: waits, overdue
        time.sleep(0.01)
        third = server.submit(fid, mid, 200)                    # fits, but is large
        smalls = [server.submit(fid, s, 100) for s in small]    # pass it
        results = {}
        while len(results) < 3 + len(smalls):
            res = server.poll(wait_ms=10000)
            assert res is not None, server.stats()
            results[res.id] = res
        stats = server.stats()
    assert all(r.status == 0 for r in results.values())
    assert stats["overdue_scans"] > 0
    assert all(results[s].admitted < results[second].admitted for s in smalls)
    assert results[third].admitted >= results[second].admitted
    for rid, s in zip(smalls, small):
        want = alone(ctx, field, s, 100, "runge_kutta_4", 0.25, False)
        assert_same(results[rid].positions, want.inactive_particles.position)
    want = alone(ctx, field, mid, 200, "runge_kutta_4", 0.25, False)
    assert_same(results[third].positions, want.inactive_particles.position)
