"""The CUDA path, through the C ABI, against the committed golden vectors
(tests/golden/*.npz): bit-exact end states, curves and indices; colors within
2e-6 rad; FTLE within 1e-3 relative."""
from pathlib import Path

import numpy as np
import pytest

import dpa_b200
from dpa_b200 import ParticleAdvector, Particles
from dpa_b200.advector import RegularGrid
from bitwise import assert_same

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
ADVECTION = sorted(p for p in GOLDEN.glob("*.npz") if "ftle" not in p.name)
FTLE = sorted(GOLDEN.glob("*ftle*.npz"))
COLOR_ATOL = 2e-6
FTLE_RTOL = 1e-3


def _grid(d):
    return RegularGrid.from_data(d["field"], d["spacing"], d["offset"])


@pytest.mark.parametrize("path", ADVECTION, ids=lambda p: p.stem)
def test_device_reproduces_the_fixture(ctx, path):
    d = np.load(path)
    record = bool(d["record"])
    field = ctx.field(_grid(d))
    try:
        adv = ParticleAdvector(ctx, len(d["seeds"]), "none", str(d["integrator"]),
                               float(d["step"]), False, record)
        out = adv.advect(field, Particles.create(d["seeds"], int(d["iterations"])))
    finally:
        field.close()
    got = out.inactive_particles
    assert_same(got.position, d["positions"])
    assert_same(got.remaining_iterations, d["remaining"])
    assert_same(got.termination, d["termination"])
    if record:
        curve = out.integral_curves[0]
        assert_same(curve.vertices, d["vertices"])
        assert curve.indices.dtype == d["indices"].dtype
        assert_same(curve.indices, d["indices"])
        np.testing.assert_allclose(curve.colors, d["colors"], rtol=0, atol=COLOR_ATOL)


def test_device_reproduces_the_ftle_fixture(ctx):
    d = np.load(FTLE[0])
    field = ctx.field(_grid(d))
    try:
        adv = ParticleAdvector(ctx, len(d["seeds"]), "none", "runge_kutta_4", float(d["step"]),
                               False, False)
        out = adv.advect(field, Particles.create(d["seeds"], int(d["iterations"])))
        assert_same(out.inactive_particles.position, d["positions"])
        got = dpa_b200.estimate_ftle(ctx, field, int(d["iterations"]), d["stride"],
                                     float(d["step"]), out.inactive_particles)
    finally:
        field.close()
    finite = np.isfinite(d["ftle"])
    assert_same(np.isfinite(got.data), finite)
    np.testing.assert_allclose(got.data[finite], d["ftle"][finite], rtol=FTLE_RTOL, atol=1e-6)
