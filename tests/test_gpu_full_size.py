"""Parity at the configurations' full sizes.

Particles are independent given the field, so a seeded sample of a full-size
launch, re-run by the oracle at the full iteration count, checks that launch
particle by particle (bit-exact end states). Size-independent properties
complete it: the processing order and the batching do not change any result.

Configurations:
- throughput: 256^3 curl noise (sigma 4, seed 1, spacing 1), 1,048,576 seeds
  (seed 1) in [0, 255)^3, runge_kutta_4, step 0.25, 2000 iterations, end
  positions only, F32 / F16 / BF16 field storage;
- recording: 64^3 ABC on [0, 2 pi]^3, 4096 seeds (seed 0), runge_kutta_4, step
  0.01, 1000 iterations, curves with uint32 indices, compared in full;
- FTLE: 256^3 ABC + 5 % smoothed perturbation (sigma 3, seed 2), 128^3
  lattice, runge_kutta_4, step 0.02, 250 iterations, compared in full;
- batched: 512^3 curl noise (sigma 8, seed 3), 64 seed sets with log-uniform
  sizes and iterations uniform in [200, 4000], one persistent launch.
"""
import ctypes as C
import math

import numpy as np
import pytest

import dpa_b200
from dpa_b200 import ParticleAdvector, Particles, fields, seeds
from dpa_b200 import _native as N
from bitwise import assert_same

pytestmark = pytest.mark.gpu

COLOR_ATOL = 2e-6  # atan2f of CUDA and of the host libm may differ in the last bits
FTLE_RTOL = 1e-3


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _rounded(grid, storage):
    """The field values the device holds for a storage, widened to FP32."""
    if storage == "f16":
        return grid.data.astype(np.float16).astype(np.float32)
    if storage == "bf16":
        import torch
        return torch.from_numpy(grid.data).to(torch.bfloat16).float().numpy()
    return grid.data


def _device_advect(ctx, field, positions, remaining, integrator, step, morton=True,
                   batch_offsets=None):
    """One dpa_advect_device (or dpa_advect_batch_device) call on device copies."""
    import torch
    pos = torch.from_numpy(np.ascontiguousarray(positions, np.float32)).cuda()
    rem = torch.from_numpy(np.asarray(remaining).astype(np.int64)).cuda()
    term = torch.zeros(pos.shape[0], dtype=torch.uint8, device="cuda")
    opts = N.AdvectOptions(N.INTEGRATORS[integrator], float(np.float32(step)), 0, 0, 0,
                           int(morton), 0)
    if batch_offsets is None:
        ctx.check(ctx._lib.dpa_advect_device(ctx.handle, field.handle, C.byref(opts),
                                             pos.shape[0], _ptr(pos), _ptr(rem), _ptr(term),
                                             None))
    else:
        offsets = np.ascontiguousarray(batch_offsets, np.uint64)
        ctx.check(ctx._lib.dpa_advect_batch_device(
            ctx.handle, field.handle, C.byref(opts), len(offsets) - 1,
            offsets.ctypes.data_as(N._U64P), _ptr(pos), _ptr(rem), _ptr(term), None, None))
    ctx.synchronize()
    return pos.cpu().numpy(), rem.cpu().numpy().astype(np.uint64), term.cpu().numpy()


def _assert_sample_matches(oracle, data, grid, got, positions, remaining, sample, integrator,
                           step):
    og = oracle.OracleGrid(data, grid.spacing, grid.offset)
    want = oracle.advect_round(og, integrator, step, positions[sample],
                               np.asarray(remaining, np.uint64)[sample])
    assert_same(got[2][sample], want.termination)
    assert_same(got[1][sample], want.remaining)
    assert_same(got[0][sample], want.positions)
    return want


@pytest.fixture(scope="module")
def throughput_inputs():
    grid = fields.curl_noise(256, 4.0, 1, device="cuda")
    offset, size = seeds.seed_box(grid)
    pos = seeds.generate_random(offset, size, 1 << 20, 0, aabb=([0.0] * 3, [255.0] * 3),
                                seed=1).position
    return grid, pos


@pytest.mark.parametrize("storage", ["f32", "f16", "bf16", "f32_edges"])
def test_throughput_configuration_matches_the_oracle_on_a_sample(ctx, oracle, throughput_inputs,
                                                                 storage):
    grid, pos = throughput_inputs
    n = pos.shape[0]
    rem = np.full(n, 2000, np.uint64)
    field = ctx.field(grid, storage)
    try:
        got = _device_advect(ctx, field, pos, rem, "runge_kutta_4", 0.25)
    finally:
        field.close()
    sample = np.sort(np.random.default_rng(7).choice(n, 8192, replace=False))
    want = _assert_sample_matches(oracle, _rounded(grid, storage), grid, got, pos, rem, sample,
                                  "runge_kutta_4", 0.25)
    # The sample exercises both ends: particles that leave the grid and ones
    # that run all 2000 iterations.
    assert np.sum(want.termination == 1) > 1000
    assert np.sum(want.termination == 0) > 100
    steps = float(np.sum(2000 - got[1].astype(np.int64)))
    assert 0.3 * 2000 * n < steps < 2000 * n


def test_throughput_configuration_does_not_depend_on_the_order(ctx, throughput_inputs):
    grid, pos = throughput_inputs
    rem = np.full(pos.shape[0], 2000, np.uint64)
    field = ctx.field(grid)
    try:
        a = _device_advect(ctx, field, pos, rem, "runge_kutta_4", 0.25, morton=True)
        b = _device_advect(ctx, field, pos, rem, "runge_kutta_4", 0.25, morton=False)
    finally:
        field.close()
    for x, y in zip(a, b):
        assert_same(x, y)


def test_recording_configuration_in_full(ctx, oracle):
    grid = fields.abc(64)
    offset, size = seeds.seed_box(grid)
    parts = seeds.generate_random(offset, size, 4096, 1000, aabb=([0, 0, 0], [2 * math.pi] * 3),
                                  seed=0)
    field = ctx.field(grid)
    try:
        adv = ParticleAdvector(ctx, 4096, "none", "runge_kutta_4", 0.01, False, True)
        out = adv.advect(field, Particles.create(parts.position, 1000))
    finally:
        field.close()
    assert len(out.integral_curves) == 1
    curve = out.integral_curves[0]
    og = oracle.OracleGrid.of(grid)
    want = oracle.advect_round(og, "runge_kutta_4", 0.01, parts.position,
                               np.full(4096, 1000, np.uint64), record=True)
    assert_same(out.inactive_particles.termination, want.termination)
    assert_same(out.inactive_particles.position, want.positions)
    assert_same(curve.vertices, want.vertices)
    assert curve.indices.dtype == np.uint32  # 4096 * 1000 <= UINT32_MAX
    assert_same(curve.indices, want.indices)
    np.testing.assert_allclose(curve.colors, want.colors, rtol=0, atol=COLOR_ATOL)
    assert curve.vertices.shape[0] > 4096 * 100


def test_ftle_configuration_in_full(ctx, oracle):
    grid = fields.abc_perturbed(256, 0.05, 3.0, 2, device="cuda")
    offset, size = seeds.seed_box(grid)
    parts = seeds.generate(offset, size, (grid.spacing * np.float32(2)).astype(np.float32), 250)
    assert len(parts) == 128 ** 3
    field = ctx.field(grid)
    try:
        adv = ParticleAdvector(ctx, len(parts), "none", "runge_kutta_4", 0.02, False, False)
        out = adv.advect(field, parts).inactive_particles
        got = dpa_b200.estimate_ftle(ctx, field, 250, (2, 2, 2), 0.02, out)
    finally:
        field.close()
    og = oracle.OracleGrid.of(grid)
    ref = oracle.advect_round(og, "runge_kutta_4", 0.02, parts.position,
                              np.full(len(parts), 250, np.uint64))
    assert_same(out.termination, ref.termination)
    assert_same(out.position, ref.positions)
    want, _ = oracle.ftle(grid.shape, grid.offset, grid.spacing, (2, 2, 2), 250, 0.02,
                          out.original_position, ref.positions, 0)
    assert got.data.shape == want.shape == (128, 128, 128)
    finite = np.isfinite(want)
    assert_same(np.isfinite(got.data), finite)
    np.testing.assert_allclose(got.data[finite], want[finite], rtol=FTLE_RTOL, atol=1e-6)


def test_batched_configuration_matches_single_calls_and_the_oracle(ctx, oracle):
    grid = fields.curl_noise(512, 8.0, 3, device="cuda")
    rng = np.random.default_rng(3)
    sets = 64
    sizes = np.exp(rng.uniform(np.log(1e3), np.log(1e6), size=sets)).astype(np.int64)
    iters = rng.integers(200, 4001, size=sets)
    offset, size = seeds.seed_box(grid)
    total = int(sizes.sum())
    pos = seeds.generate_random(offset, size, total, 0, aabb=([0.0] * 3, [511.0] * 3),
                                seed=3).position
    rem = np.repeat(iters, sizes).astype(np.uint64)
    offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.uint64)
    field = ctx.field(grid, "f16")
    try:
        batched = _device_advect(ctx, field, pos, rem, "runge_kutta_4", 0.25,
                                 batch_offsets=offsets)
        single = _device_advect(ctx, field, pos, rem, "runge_kutta_4", 0.25)
    finally:
        field.close()
    for x, y in zip(batched, single):
        assert_same(x, y)
    sample = np.sort(rng.choice(total, 2048, replace=False))
    _assert_sample_matches(oracle, _rounded(grid, "f16"), grid, batched, pos, rem, sample,
                           "runge_kutta_4", 0.25)
