"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Bar: final positions, termination reasons and steps, pruned curve vertices
and index buffers are bit-exact; colors agree within 2e-6 rad (atan2f of
CUDA and of the host libm may differ in the last bits; the exact special
cases, 0 and pi, must match exactly)."""
import math

import numpy as np
import pytest

import dpa_b200
from dpa_b200 import ParticleAdvector, Particles, fields, seeds
from bitwise import assert_same

pytestmark = pytest.mark.gpu

COLOR_ATOL = 2e-6


def _seeds_in_box(grid, count, seed, box=None):
    offset, size = seeds.seed_box(grid)
    return seeds.generate_random(offset, size, count, 0, aabb=box, seed=seed).position


def compare(ctx, oracle, grid, positions, iterations, integrator, step, ppr, record,
            storage="f32", index64=False, morton=True, staging=None, host_chunk=None):
    """Runs the GPU rounds and the oracle rounds on the same input."""
    oracle_data = grid.data
    if storage == "f16":
        oracle_data = grid.data.astype(np.float16).astype(np.float32)
    elif storage == "bf16":
        import torch
        oracle_data = torch.from_numpy(grid.data).to(torch.bfloat16).float().numpy()
    og = oracle.OracleGrid(oracle_data, grid.spacing, grid.offset)
    rem = np.broadcast_to(np.asarray(iterations, np.uint64), (positions.shape[0],)).copy()
    want, want_rounds = oracle.advect_rounds(og, integrator, step, positions, rem, ppr, record,
                                             index64)
    if staging:
        ctx.set_staging_limit(staging)
    if host_chunk:
        ctx.check(ctx._lib.dpa_context_set_host_chunk_limit(ctx.handle, host_chunk))
    field = ctx.field(grid, storage)
    adv = ParticleAdvector(ctx, ppr, "none", integrator, step, False, record,
                           use_64_bit_indices=index64, morton_order=morton)
    got = adv.advect(field, Particles.create(positions, rem))
    if staging:
        ctx.set_staging_limit(1 << 30)
    if host_chunk:
        ctx.check(ctx._lib.dpa_context_set_host_chunk_limit(ctx.handle, 256 << 20))
    assert_same(got.inactive_particles.termination, want.termination)
    assert_same(got.inactive_particles.remaining_iterations, want.remaining)
    assert_same(got.inactive_particles.position, want.positions)
    if record:
        assert len(got.integral_curves) == len(want_rounds)
        for c, r in zip(got.integral_curves, want_rounds):
            assert_same(c.vertices, r.vertices)
            assert c.indices.dtype == r.indices.dtype
            assert_same(c.indices, r.indices)
            np.testing.assert_allclose(c.colors, r.colors, rtol=0, atol=COLOR_ATOL)
            special = (r.colors == 0) | (r.colors == np.float32(math.pi))
            assert_same(c.colors[special], r.colors[special])
    return got, want


@pytest.mark.parametrize("integrator", ["runge_kutta_4", "euler", "runge_kutta_4_true"])
def test_abc_recording_matches_oracle(ctx, oracle, integrator):
    grid = fields.abc(64)
    box = ([0, 0, 0], [2 * math.pi] * 3)
    pos = _seeds_in_box(grid, 512, 0, box)
    compare(ctx, oracle, grid, pos, 300, integrator, 0.01, 512, True)


def test_abc_default_seed_box_has_out_of_bounds_starts(ctx, oracle):
    # The default seed box reaches one cell past the valid domain, so some
    # particles leave at step 0 with a two-vertex curve.
    grid = fields.abc(32)
    pos = _seeds_in_box(grid, 2048, 3)
    got, want = compare(ctx, oracle, grid, pos, 50, "runge_kutta_4", 0.05, 2048, True)
    assert np.sum((want.termination == 1) & (want.steps == 0)) > 0


def test_multiple_rounds_take_the_tail(ctx, oracle):
    grid = fields.abc(32)
    pos = _seeds_in_box(grid, 1000, 4, ([0, 0, 0], [2 * math.pi] * 3))
    got, _ = compare(ctx, oracle, grid, pos, 80, "runge_kutta_4", 0.02, 300, True)
    assert got.rounds == 4
    assert [c.vertices.shape[0] > 0 for c in got.integral_curves] == [True] * 4


def test_u64_indices_and_small_staging_pieces(ctx, oracle):
    grid = fields.abc(32)
    pos = _seeds_in_box(grid, 777, 5, ([0, 0, 0], [2 * math.pi] * 3))
    compare(ctx, oracle, grid, pos, 120, "runge_kutta_4", 0.02, 777, True, index64=True,
            staging=12 * 122 * 50)
    compare(ctx, oracle, grid, pos, 120, "runge_kutta_4", 0.02, 777, True, index64=False,
            staging=12 * 122 * 7)


@pytest.mark.parametrize("index64", [False, True])
def test_curve_chunks_through_small_pinned_halves(ctx, oracle, index64):
    # A host chunk limit of 4 KiB splits every piece's curve into many chunks
    # (vertices and indices split at different places), copied through the
    # two pinned halves while the sink takes the previous chunk.
    grid = fields.abc(32)
    pos = _seeds_in_box(grid, 600, 12, ([0, 0, 0], [2 * math.pi] * 3))
    compare(ctx, oracle, grid, pos, 150, "runge_kutta_4", 0.02, 600, True, index64=index64,
            staging=12 * 152 * 200, host_chunk=4096)


def test_curl_noise_power_of_two_spacing_end_positions(ctx, oracle):
    grid = fields.curl_noise(64, 4.0, 1)
    pos = _seeds_in_box(grid, 4096, 1)
    got, want = compare(ctx, oracle, grid, pos, 400, "runge_kutta_4", 0.25, 4096, False)
    assert np.sum(want.termination == 0) > 500


def test_non_power_of_two_unit_like_spacing(ctx, oracle):
    grid = fields.curl_noise(48, 3.0, 9, spacing=0.7)
    pos = _seeds_in_box(grid, 2048, 2)
    compare(ctx, oracle, grid, pos, 200, "runge_kutta_4", 0.2, 2048, False)


@pytest.mark.parametrize("storage", ["f16", "bf16"])
def test_half_storage_is_exact_on_the_rounded_field(ctx, oracle, storage):
    # The device widens 16-bit nodes to FP32 exactly and then runs the same
    # arithmetic, so it matches the oracle on the rounded field bit for bit.
    grid = fields.curl_noise(64, 4.0, 11)
    pos = _seeds_in_box(grid, 2048, 6)
    compare(ctx, oracle, grid, pos, 300, "runge_kutta_4", 0.25, 2048, False, storage=storage)


@pytest.mark.parametrize("case", ["abc_record", "noise_rk4", "spacing_0.7", "anisotropic",
                                  "cash_karp"])
def test_edge_record_storage_matches_the_f32_oracle(ctx, oracle, case):
    # F32_EDGES holds the F32 values as one 32-byte record per cell edge:
    # the same bits as F32 storage, so the oracle on the unrounded field.
    if case == "abc_record":
        grid = fields.abc(32)
        pos = _seeds_in_box(grid, 1500, 3, box=([0, 0, 0], [2 * math.pi] * 3))
        compare(ctx, oracle, grid, pos, 300, "runge_kutta_4", 0.01, 1000, True,
                storage="f32_edges")
    elif case == "noise_rk4":
        grid = fields.curl_noise(64, 4.0, 11)
        pos = _seeds_in_box(grid, 12000, 6)
        compare(ctx, oracle, grid, pos, 300, "runge_kutta_4", 0.25, 12000, False,
                storage="f32_edges")
    elif case == "spacing_0.7":
        grid = fields.curl_noise(48, 3.0, 9, spacing=0.7)
        pos = _seeds_in_box(grid, 2048, 2)
        compare(ctx, oracle, grid, pos, 200, "runge_kutta_4", 0.2, 2048, False,
                storage="f32_edges")
    elif case == "anisotropic":
        data = fields.curl_noise(40, 3.0, 4).data[:, :17, :5].copy()
        grid = dpa_b200.RegularGrid.from_data(data, (0.5, 2.0, 0.25), (1.0, -3.0, 0.5))
        pos = _seeds_in_box(grid, 3000, 12)
        compare(ctx, oracle, grid, pos, 150, "euler", 0.1, 3000, False, storage="f32_edges")
    else:
        grid = fields.curl_noise(32, 3.0, 5)
        pos = _seeds_in_box(grid, 2000, 13)
        compare(ctx, oracle, grid, pos, 200, "runge_kutta_cash_karp_54", 0.25, 2000, False,
                storage="f32_edges")


def test_morton_order_does_not_change_results(ctx, oracle):
    # 12,000 particles: calls with fewer than 8192 run in input order anyway.
    grid = fields.curl_noise(32, 3.0, 2)
    pos = _seeds_in_box(grid, 12000, 8)
    a, _ = compare(ctx, oracle, grid, pos, 100, "euler", 0.3, 12000, True, morton=True)
    b, _ = compare(ctx, oracle, grid, pos, 100, "euler", 0.3, 12000, True, morton=False)
    assert_same(a.inactive_particles.position, b.inactive_particles.position)


def test_edge_cases(ctx, oracle):
    grid = fields.abc(16)
    field = ctx.field(grid)
    # empty round
    adv = ParticleAdvector(ctx, 10, "none", "runge_kutta_4", 0.01, False, True)
    out = adv.advect(field, Particles.create(np.zeros((0, 3), np.float32), 10))
    assert out.rounds == 0 and len(out.inactive_particles) == 0
    # zero remaining, outside, NaN, exactly on the upper boundary
    top = np.float32(grid.spacing[0] * np.float32(14))
    pos = np.array([[1, 1, 1], [50, 1, 1], [np.nan, 1, 1], [top, 1, 1], [1, 1, 1]], np.float32)
    rem = np.array([0, 5, 5, 5, 5], np.uint64)
    og = oracle.OracleGrid.of(grid)
    want = oracle.advect_round(og, "runge_kutta_4", 0.01, pos, rem, record=True)
    got = adv.advect(field, Particles(pos.copy(), rem.copy(), pos.copy()))
    assert_same(got.inactive_particles.termination, want.termination)
    assert_same(got.inactive_particles.remaining_iterations, want.remaining)
    c = got.integral_curves[0]
    assert_same(c.vertices, want.vertices)
    assert_same(c.indices, want.indices)
    # zero field: zero-velocity termination at step 0
    zero = dpa_b200.RegularGrid.from_data(np.zeros((8, 8, 8, 3), np.float32), (1, 1, 1))
    zf = ctx.field(zero)
    out = ParticleAdvector(ctx, 4, "none", "euler", 0.1, False, False).advect(
        zf, Particles.create(np.full((3, 3), 2.0, np.float32), 9))
    assert list(out.inactive_particles.termination) == [2, 2, 2]
    assert list(out.inactive_particles.remaining_iterations) == [9, 9, 9]


OTHER_INTEGRATORS = ["modified_midpoint", "runge_kutta_cash_karp_54",
                     "runge_kutta_dormand_prince_5", "runge_kutta_fehlberg_78",
                     "adams_bashforth_2", "adams_bashforth_moulton_2"]


@pytest.mark.parametrize("integrator", OTHER_INTEGRATORS)
def test_other_odeint_steppers_match_oracle(ctx, oracle, integrator):
    # Recorded curves over several rounds, then end positions on a
    # power-of-two grid with FP16 storage (the multiplicative cell lookup).
    grid = fields.abc(48)
    pos = _seeds_in_box(grid, 700, 3, ([0, 0, 0], [2 * math.pi] * 3))
    compare(ctx, oracle, grid, pos, 200, integrator, 0.02, 256, True)
    noise = fields.curl_noise(64, 4.0, 6)
    pos = _seeds_in_box(noise, 3000, 4)
    compare(ctx, oracle, noise, pos, 400, integrator, 0.25, 3000, False, storage="f16")


@pytest.mark.parametrize("integrator", ["runge_kutta_dormand_prince_5", "adams_bashforth_2",
                                        "adams_bashforth_moulton_2"])
def test_steppers_with_memory_refuse_step_budgets(ctx, integrator):
    import ctypes as C
    import torch
    from dpa_b200 import _native as N
    grid = fields.abc(8)
    field = ctx.field(grid)
    pos = torch.ones((2, 3), dtype=torch.float32, device="cuda")
    rem = torch.full((2,), 3, dtype=torch.int64, device="cuda")
    opts = N.AdvectOptions(N.INTEGRATORS[integrator], 0.1, 0, 0, 0, 0, 2)
    rc = ctx._lib.dpa_advect_device(ctx.handle, field.handle, C.byref(opts), 2,
                                    C.c_void_p(pos.data_ptr()), C.c_void_p(rem.data_ptr()), None,
                                    None)
    assert rc == 2
    rc = ctx._lib.dpa_advect_device_no_alloc(ctx.handle, field.handle, C.byref(opts), 2,
                                             C.c_void_p(pos.data_ptr()),
                                             C.c_void_p(rem.data_ptr()), None, None)
    assert rc == 2
    field.close()


def test_device_api_matches_host_api(ctx, oracle):
    import ctypes as C
    import torch
    from dpa_b200 import _native as N
    grid = fields.curl_noise(64, 4.0, 3)
    pos = _seeds_in_box(grid, 3000, 9)
    field = ctx.field(grid)
    adv = ParticleAdvector(ctx, 3000, "none", "runge_kutta_4", 0.25, False, False)
    host = adv.advect(field, Particles.create(pos, 200))
    dp = torch.from_numpy(pos.copy()).cuda()
    dr = torch.full((3000,), 200, dtype=torch.int64, device="cuda")
    dt = torch.zeros(3000, dtype=torch.uint8, device="cuda")
    opts = adv.options(False)
    ctx.check(ctx._lib.dpa_advect_device(ctx.handle, field.handle, C.byref(opts), 3000,
                                         C.c_void_p(dp.data_ptr()), C.c_void_p(dr.data_ptr()),
                                         C.c_void_p(dt.data_ptr()), None))
    ctx.synchronize()
    assert_same(dp.cpu().numpy(), host.inactive_particles.position)
    assert_same(dr.cpu().numpy().astype(np.uint64),
                                  host.inactive_particles.remaining_iterations)
    assert_same(dt.cpu().numpy(), host.inactive_particles.termination)


@pytest.mark.parametrize("mapping,storage", [("reference", "f32"), ("lattice", "f32"),
                                             ("lattice", "f32_edges")])
def test_ftle_matches_oracle(ctx, oracle, mapping, storage):
    grid = fields.abc_perturbed(64, seed=2)
    field = ctx.field(grid, storage)
    offset, size = seeds.seed_box(grid)
    stride = np.float32(2)
    parts = seeds.generate(offset, size, (grid.spacing * stride).astype(np.float32), 60)
    adv = ParticleAdvector(ctx, len(parts), "none", "runge_kutta_4", 0.02, False, False)
    out = adv.advect(field, parts).inactive_particles
    got = dpa_b200.estimate_ftle(ctx, field, 60, (2, 2, 2), 0.02, out, mapping)
    want, info = oracle.ftle(grid.shape, grid.offset, grid.spacing, (2, 2, 2), 60, 0.02,
                             out.original_position, out.position, 0 if mapping == "reference" else 1)
    assert got.data.shape == want.shape == (32, 32, 32)
    finite = np.isfinite(want)
    assert_same(np.isfinite(got.data), finite)
    np.testing.assert_allclose(got.data[finite], want[finite], rtol=1e-3, atol=1e-6)


def test_degenerate_and_anisotropic_grids(ctx, oracle):
    rng = np.random.default_rng(12)
    # One cell (2 x 2 x 2 nodes); an axis of a single node (no cell is inside);
    # an anisotropic grid with a negative offset and mixed spacings, one of
    # them a power of two; power-of-two spacings with non-zero offsets.
    cases = [
        (rng.normal(size=(2, 2, 2, 3)).astype(np.float32), (0.5, 0.5, 0.5), (0.0, 0.0, 0.0)),
        (rng.normal(size=(4, 1, 4, 3)).astype(np.float32), (1.0, 1.0, 1.0), (0.0, 0.0, 0.0)),
        (rng.normal(size=(9, 5, 13, 3)).astype(np.float32), (0.3, 2.0, 0.125),
         (-1.25, 3.0, -0.5)),
        # power-of-two spacings with non-zero offsets: the one-FMA location
        (rng.normal(size=(7, 11, 6, 3)).astype(np.float32), (0.5, 0.25, 2.0),
         (-1.5, -0.75, 4.0)),
    ]
    for data, spacing, offset in cases:
        grid = dpa_b200.RegularGrid.from_data(data, spacing, offset)
        lo = np.asarray(offset, np.float32)
        hi = lo + np.asarray(spacing, np.float32) * (np.asarray(data.shape[:3]) - 1)
        pos = (lo + rng.random((300, 3)) * (hi - lo) * 1.02 - 0.01 * (hi - lo)).astype(np.float32)
        compare(ctx, oracle, grid, pos, 40, "runge_kutta_4", 0.05, 300, True)


def _locate_mode(ctx, field):
    import ctypes as C
    mode = C.c_int32()
    ctx.check(ctx._lib.dpa_field_locate_mode(field.handle, C.byref(mode)))
    return mode.value


@pytest.mark.parametrize("spacing", [2 * math.pi / 63, 0.7, 1.0 / 3.0])
def test_reciprocal_division_matches_ieee_division_and_oracle(ctx, oracle, spacing):
    """Non-power-of-two spacings divide by the rounded reciprocal once the
    device has checked it against IEEE division for every float dividend;
    results are bit-exact with the IEEE-division kernels and with the oracle."""
    data = fields.curl_noise(40, 3.0, 13).data
    grid = dpa_b200.RegularGrid.from_data(data, (spacing, spacing, spacing), (0.25, -0.5, 0.0))
    pos = _seeds_in_box(grid, 3000, 14)
    step = float(np.float32(0.3 * spacing))
    og = oracle.OracleGrid(grid.data, grid.spacing, grid.offset)
    rem = np.full(pos.shape[0], 250, np.uint64)
    want = oracle.advect_round(og, "runge_kutta_4", step, pos, rem, record=True)
    modes = []
    try:
        for ieee in (0, 1):
            ctx.check(ctx._lib.dpa_context_set_ieee_division(ctx.handle, ieee))
            field = ctx.field(grid)
            modes.append(_locate_mode(ctx, field))
            adv = ParticleAdvector(ctx, pos.shape[0], "none", "runge_kutta_4", step, False, True)
            got = adv.advect(field, Particles.create(pos, rem))
            field.close()
            assert_same(got.inactive_particles.position, want.positions)
            assert_same(got.inactive_particles.termination, want.termination)
            assert_same(got.integral_curves[0].vertices, want.vertices)
            assert_same(got.integral_curves[0].indices, want.indices)
    finally:
        ctx.check(ctx._lib.dpa_context_set_ieee_division(ctx.handle, 0))
    # The split reciprocal is exact for these divisors (an exhaustive host
    # check of all 2^32 dividends agrees), so the default is mode 1.
    assert modes == [1, 0], modes


@pytest.mark.parametrize("storage", ["f32", "f16", "f32_edges"])
@pytest.mark.parametrize("integrator", ["runge_kutta_4", "runge_kutta_cash_karp_54"])
def test_two_particles_per_lane_and_block_sizes_match_oracle(ctx, oracle, storage, integrator):
    """Every launch shape the autotuner may pick -- 64 to 256 threads per
    block, one or two particles per lane -- gives the oracle's results bit
    for bit, including step budgets resumed over several calls."""
    import ctypes as C
    import torch
    from dpa_b200 import _native as N
    n = 10000  # enough to be sorted into the processing order
    grid = fields.curl_noise(48, 3.0, 15)
    pos = _seeds_in_box(grid, n, 16)
    data = grid.data if storage != "f16" else grid.data.astype(np.float16).astype(np.float32)
    og = oracle.OracleGrid(data, grid.spacing, grid.offset)
    want = oracle.advect_round(og, integrator, 0.25, pos, np.full(n, 300, np.uint64))
    field = ctx.field(grid, storage)
    saved = N.Tuning()
    ctx.check(ctx._lib.dpa_context_get_tuning(ctx.handle, C.byref(saved)))
    try:
        for block, ppt, budget in ((256, 2, 0), (64, 2, 0), (128, 1, 0), (64, 2, 77), (96, 2, 0)):
            t = N.Tuning(16, 0, 64, 0.0, block, ppt)
            ctx.check(ctx._lib.dpa_context_set_tuning(ctx.handle, C.byref(t)))
            p = torch.from_numpy(pos).cuda()
            r = torch.full((n,), 300, dtype=torch.int64, device="cuda")
            term = torch.zeros(n, dtype=torch.uint8, device="cuda")
            opts = N.AdvectOptions(N.INTEGRATORS[integrator], 0.25, 0, 0, 0, 1, budget)
            for _ in range(300 // budget + 1 if budget else 1):
                ctx.check(ctx._lib.dpa_advect_device(ctx.handle, field.handle, C.byref(opts),
                                                     n, C.c_void_p(p.data_ptr()),
                                                     C.c_void_p(r.data_ptr()),
                                                     C.c_void_p(term.data_ptr()), None))
            ctx.synchronize()
            assert_same(p.cpu().numpy(), want.positions)
            assert_same(r.cpu().numpy().astype(np.uint64), want.remaining)
            assert_same(term.cpu().numpy(), want.termination)
    finally:
        ctx.check(ctx._lib.dpa_context_set_tuning(ctx.handle, C.byref(saved)))
        field.close()


def _signed_zero_field(n, spacing):
    """v = (-z, -y, -x) stored reversed: every component is -0.0 on its own
    face, so the sign of a zero weight decides the sign of a zero velocity
    and, through x + dt * v, of a zero coordinate."""
    data = np.zeros((n, n, n, 3), np.float32)
    c = np.arange(n, dtype=np.float32) * np.float32(spacing)
    data[..., 0] = -c[None, None, :]
    data[..., 1] = -c[None, :, None]
    data[..., 2] = -c[:, None, None]
    return dpa_b200.RegularGrid.from_data(data, (spacing,) * 3)


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


@pytest.mark.parametrize("spacing", [1.0, 0.7])
def test_signed_zeros_nan_field_values_and_huge_budgets(ctx, oracle, spacing):
    """Bit for bit, signs of zero included: starts at -0.0 on each axis
    (a zero weight keeps its sign as fmod's does), a NaN node in the field
    (the velocity turns NaN, the next step leaves the grid), infinite starts,
    and remaining counts above 2^32 that end out of bounds. Power-of-two and
    general spacings; end positions through the device entry point and
    recorded curves through rounds."""
    import ctypes as C
    import torch
    from dpa_b200 import _native as N
    grid = _signed_zero_field(8, spacing)
    grid.data[5, 5, 5] = np.nan
    h = np.float32(spacing)
    mid = np.float32(1.5) * h
    nan_cell = np.float32(4.5) * h
    pos = np.array([[-0.0, mid, mid], [mid, -0.0, mid], [mid, mid, -0.0], [-0.0, -0.0, -0.0],
                    [0.0, 0.0, 0.0], [nan_cell, nan_cell, nan_cell], [np.inf, mid, mid],
                    [mid, -np.inf, mid], [mid, mid, mid], [np.float32(6.5) * h, mid, mid]],
                   np.float32)
    rem = np.array([3, 3, 3, 3, 3, 5, 4, 4, 2 ** 33, 2 ** 40 + 7], np.uint64)
    og = oracle.OracleGrid.of(grid)
    # Curves only for the first eight: a curve's staging spans the round's
    # largest remaining count (particle_advector.cpp:311-316).
    rec = slice(0, 8)
    for integrator in ("euler", "runge_kutta_4"):
        want = oracle.advect_round(og, integrator, 0.25, pos, rem)
        assert np.isnan(want.positions[5]).all()  # the NaN node reached the particle
        want_rec = oracle.advect_round(og, integrator, 0.25, pos[rec], rem[rec], record=True)
        field = ctx.field(grid)
        n = pos.shape[0]
        p = torch.from_numpy(pos).cuda()
        r = torch.from_numpy(rem.astype(np.int64)).cuda()
        term = torch.zeros(n, dtype=torch.uint8, device="cuda")
        opts = N.AdvectOptions(N.INTEGRATORS[integrator], 0.25, 0, 0, 0, 0, 0)
        ctx.check(ctx._lib.dpa_advect_device(ctx.handle, field.handle, C.byref(opts), n,
                                             C.c_void_p(p.data_ptr()), C.c_void_p(r.data_ptr()),
                                             C.c_void_p(term.data_ptr()), None))
        ctx.synchronize()
        got = p.cpu().numpy()
        finite = ~np.isnan(want.positions)
        assert_same(np.isnan(got), ~finite)
        assert_same(_bits(got)[finite], _bits(want.positions)[finite])
        assert_same(r.cpu().numpy().astype(np.uint64), want.remaining)
        assert_same(term.cpu().numpy(), want.termination)
        adv = ParticleAdvector(ctx, n, "none", integrator, 0.25, False, True)
        out = adv.advect(field, Particles(pos[rec].copy(), rem[rec].copy(), pos[rec].copy()))
        field.close()
        curve = out.integral_curves[0]
        ok = ~np.isnan(want_rec.vertices)
        assert_same(np.isnan(curve.vertices), ~ok)
        assert_same(_bits(curve.vertices)[ok], _bits(want_rec.vertices)[ok])
        assert_same(curve.indices, want_rec.indices)
        assert_same(out.inactive_particles.termination, want_rec.termination)
        done = out.inactive_particles
        fin = ~np.isnan(want_rec.positions)
        assert_same(_bits(done.position)[fin], _bits(want_rec.positions)[fin])
