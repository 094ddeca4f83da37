"""The committed golden vectors (tests/golden/*.npz, made by
tests/golden/make_golden.py) against the oracle and the independent numpy
restatement: both must still reproduce every fixture, so a change to either
shows up here."""
import importlib.util
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"
ADVECTION = sorted(p for p in GOLDEN.glob("*.npz") if "ftle" not in p.name)
FTLE = sorted(GOLDEN.glob("*ftle*.npz"))


def _restatement():
    spec = importlib.util.spec_from_file_location("make_golden", GOLDEN / "make_golden.py")
    module = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(module)
    return module


def test_fixtures_are_present():
    assert len(ADVECTION) >= 5 and len(FTLE) == 1
    kinds = np.concatenate([np.load(p)["termination"] for p in ADVECTION])
    # Completed, out-of-bounds and zero-velocity endings all occur.
    assert set(np.unique(kinds)) == {0, 1, 2}


@pytest.mark.parametrize("path", ADVECTION, ids=lambda p: p.stem)
def test_oracle_reproduces_the_fixture(oracle, path):
    d = np.load(path)
    record = bool(d["record"])
    og = oracle.OracleGrid(d["field"], d["spacing"], d["offset"])
    rem = np.full(len(d["seeds"]), int(d["iterations"]), np.uint64)
    got = oracle.advect_round(og, str(d["integrator"]), float(d["step"]), d["seeds"], rem,
                              record=record)
    np.testing.assert_array_equal(got.positions, d["positions"])
    np.testing.assert_array_equal(got.remaining, d["remaining"])
    np.testing.assert_array_equal(got.termination, d["termination"])
    if record:
        np.testing.assert_array_equal(got.vertices, d["vertices"])
        np.testing.assert_array_equal(got.indices, d["indices"])
        np.testing.assert_array_equal(got.colors, d["colors"])


@pytest.mark.parametrize("path", ADVECTION, ids=lambda p: p.stem)
def test_numpy_restatement_reproduces_the_fixture(path):
    m = _restatement()
    d = np.load(path)
    record = bool(d["record"])
    rem = np.full(len(d["seeds"]), int(d["iterations"]), np.uint64)
    want = m.advect_round(d["field"], d["offset"], d["spacing"], str(d["integrator"]),
                          np.float32(d["step"]), d["seeds"], rem, record)
    np.testing.assert_array_equal(want["positions"], d["positions"])
    np.testing.assert_array_equal(want["remaining"], d["remaining"])
    np.testing.assert_array_equal(want["termination"], d["termination"])
    if record:
        np.testing.assert_array_equal(want["vertices"], d["vertices"])
        np.testing.assert_array_equal(want["indices"], d["indices"])
        np.testing.assert_allclose(want["colors"], d["colors"], rtol=0, atol=2e-6)


def test_ftle_fixture(oracle):
    m = _restatement()
    d = np.load(FTLE[0])
    shape = d["field"].shape[:3]
    got, _ = oracle.ftle(shape, d["offset"], d["spacing"], d["stride"], int(d["iterations"]),
                         float(d["step"]), d["seeds"], d["positions"], 0)
    np.testing.assert_array_equal(got, d["ftle"])
    want = m.ftle(shape, d["offset"], d["spacing"], d["stride"], int(d["iterations"]),
                  float(d["step"]), d["seeds"], d["positions"])
    finite = np.isfinite(want)
    np.testing.assert_allclose(want[finite], d["ftle"][finite], rtol=1e-5, atol=1e-7)
