"""CPU tests of the host library: HDF5 reading and writing, configuration
errors, and the seed generators (no GPU needed)."""
import json
import math
from pathlib import Path

import numpy as np
import pytest

from dpa_b200 import fields, host, seeds

MATLAB_HDF5 = (Path(np.__file__).resolve().parent.parent / "scipy" / "io" / "matlab" / "tests" /
               "data" / "testhdf5_7.4_GLNX86.mat")


@pytest.mark.skipif(not MATLAB_HDF5.exists(), reason="scipy's MATLAB v7.3 test file is absent")
def test_reader_reads_a_file_written_by_the_hdf5_library():
    # A MATLAB v7.3 file: the HDF5 library's output with a 512-byte user block,
    # superblock v0, a symbol-table root group and a layout-v2 dataset.
    assert host.names(MATLAB_HDF5) == ["testdouble"]
    dims, cls, size = host.info(MATLAB_HDF5, "testdouble")
    assert dims == (9, 1) and cls == 1 and size == 8
    values = host.read(MATLAB_HDF5, "testdouble").ravel()
    np.testing.assert_allclose(values, np.arange(9) * math.pi / 4, rtol=0, atol=1e-15)


def test_writer_round_trip(tmp_path):
    path = tmp_path / "field.h5"
    grid = fields.abc(9)
    host.write_field(path, grid, "velocity", "spacing")
    assert host.names(path) == ["velocity"]
    assert host.info(path, "velocity") == ((9, 9, 9, 3), 1, 4)
    np.testing.assert_array_equal(host.read(path, "velocity"), grid.data)
    np.testing.assert_array_equal(host.attribute(path, "spacing").astype(np.float32), grid.spacing)


def test_many_datasets_in_one_group(tmp_path):
    # More members than a default-sized symbol table node (8) holds, with the
    # reference's per-round names and every element type it writes.
    rng = np.random.default_rng(0)
    data = {}
    for r in range(40):
        data[f"vertices_{r}"] = rng.random(3 * (r + 1)).astype(np.float32)
        data[f"colors_{r}"] = rng.random(r + 1).astype(np.float32)
        data[f"indices_{r}"] = (np.arange(2 * r, dtype=np.uint64) * (1 << 33)
                                if r % 2 else np.arange(2 * r, dtype=np.uint32))
    data["bytes"] = np.arange(7, dtype=np.uint8)
    data["empty"] = np.zeros(0, np.float32)
    path = tmp_path / "many.h5"
    host.write_datasets(path, data)
    assert host.names(path) == sorted(data)
    for name, want in data.items():
        got = host.read(path, name)
        assert got.shape == want.shape
        np.testing.assert_array_equal(got, want.astype(got.dtype))


def test_unknown_dataset_and_missing_file_raise(tmp_path):
    path = tmp_path / "f.h5"
    host.write_field(path, fields.abc(4), "data", "spacing")
    with pytest.raises(RuntimeError, match="no dataset"):
        host.read(path, "nope")
    with pytest.raises(RuntimeError, match="cannot open"):
        host.read(tmp_path / "missing.h5", "data")


def _config(tmp_path, **over):
    cfg = {
        "input_dataset_filepath": str(tmp_path / "in.h5"),
        "input_dataset_name": "data",
        "input_dataset_spacing_name": "spacing",
        "particle_advector_load_balancer": "none",
        "particle_advector_integrator": "runge_kutta_4",
        "particle_advector_step_size": 0.01,
        "particle_advector_gather_particles": True,
        "particle_advector_record": True,
        "estimate_ftle": False,
        "output_dataset_filepath": str(tmp_path / "out" / "result.h5"),
        "seed_generation_iterations": "10",
        "particle_advector_particles_per_round": "100",
        "seed_generation_count": "50",
    }
    cfg.update(over)
    p = tmp_path / "config.json"
    p.write_text(json.dumps(cfg))
    return p


def test_pipeline_rejects_bad_configurations(tmp_path):
    bad = tmp_path / "bad.json"
    bad.write_text("{ not json")
    r = host.run_pipeline(bad)
    assert r.returncode == 1 and "JSON" in r.stderr
    cfg = _config(tmp_path)
    d = json.loads(cfg.read_text())
    del d["particle_advector_step_size"]
    cfg.write_text(json.dumps(d))
    r = host.run_pipeline(cfg)
    assert r.returncode == 1 and "particle_advector_step_size" in r.stderr
    cfg = _config(tmp_path, seed_generation_iterations=10)  # must be a string
    r = host.run_pipeline(cfg)
    assert r.returncode == 1 and "not a string" in r.stderr
    cfg = _config(tmp_path, particle_advector_integrator="rk9")
    r = host.run_pipeline(cfg)
    assert r.returncode == 1 and "unknown integrator" in r.stderr
    cfg = _config(tmp_path)  # valid, but the input file does not exist
    r = host.run_pipeline(cfg)
    assert r.returncode == 1 and "cannot open" in r.stderr


def test_seed_generators_agree_across_python_and_host(oracle):
    o = np.zeros(3, np.float32)
    s = np.array([6.3, 4.0, 9.5], np.float32)
    np.testing.assert_array_equal(seeds.generate_random(o, s, 5000, 1, seed=3).position,
                                  host.random_seeds(o, s, 5000, 3))
    box = ([0.5, 0.5, 0.5], [2.0, 3.0, 4.0])
    np.testing.assert_array_equal(seeds.generate_random(o, s, 100, 1, aabb=box, seed=9).position,
                                  host.random_seeds(o, s, 100, 9, aabb=box))
    stride = np.float32([0.25, 0.5, 0.75])
    lat = host.lattice_seeds(o, s, stride)
    np.testing.assert_array_equal(lat, seeds.generate(o, s, stride, 1).position)
    np.testing.assert_array_equal(lat, oracle.lattice_seeds(o, s, stride)[0])
    for lo, hi, seed in [(1, 1, 0), (10, 20, 5), (0, 1000000, 77)]:
        n = host.random_count(lo, hi, seed)
        assert lo <= n <= hi and n == seeds.random_count(lo, hi, seed)
    u = seeds.random_unit(100000, 4)
    assert u.min() >= 0.0 and u.max() < 1.0 and abs(float(u.mean()) - 0.5) < 0.01


@pytest.mark.skipif(not Path("/dev/full").exists(), reason="no /dev/full")
def test_writer_reports_a_short_write():
    # A device whose every write fails with ENOSPC: the writer must raise,
    # not leave a silently truncated file behind.
    data = {"vertices_0": np.arange(3 * 100000, dtype=np.float32)}
    with pytest.raises(RuntimeError, match="short write|cannot close"):
        host.write_datasets("/dev/full", data)
