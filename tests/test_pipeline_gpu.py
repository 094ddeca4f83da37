"""End-to-end runs of `dpa_pipeline config.json` on the GPU: the per-round
HDF5/XDMF curves, the FTLE grid and the benchmark CSV, checked against the
oracle on the same seeds."""
import ctypes as C
import json
import math

import numpy as np
import pytest

import dpa_b200
from dpa_b200 import fields, host, seeds
from bitwise import assert_same

pytestmark = pytest.mark.gpu


def write_config(tmp_path, **fields_):
    cfg = {
        "input_dataset_filepath": str(tmp_path / "in.h5"),
        "input_dataset_name": "data",
        "input_dataset_spacing_name": "spacing",
        "particle_advector_load_balancer": "none",
        "particle_advector_integrator": "runge_kutta_4",
        "particle_advector_step_size": 0.02,
        "particle_advector_gather_particles": True,
        "particle_advector_record": True,
        "estimate_ftle": False,
        "output_dataset_filepath": str(tmp_path / "result.h5"),
        "seed_generation_iterations": "80",
        "particle_advector_particles_per_round": "250",
    }
    cfg.update(fields_)
    path = tmp_path / "config.json"
    path.write_text(json.dumps(cfg))
    return path


def test_pipeline_curves_match_the_oracle(tmp_path, oracle):
    grid = fields.abc(32)
    host.write_field(tmp_path / "in.h5", grid, "data", "spacing")
    box = {"minimum": [0.0, 0.0, 0.0], "maximum": [2 * math.pi] * 3}
    cfg = write_config(tmp_path, seed_generation_count="600", seed_generation_boundaries=box,
                       dpa_b200_seed="5")
    r = host.run_pipeline(cfg, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    for stage in ("domain_partitioning", "data_loading", "seed_generation", "particle_advection",
                  "save_integral_curves", "estimate_ftle"):
        assert stage in r.stdout

    offset, size = seeds.seed_box(grid)
    pos = host.random_seeds(offset, size, 600, 5, aabb=([0, 0, 0], [2 * math.pi] * 3))
    og = oracle.OracleGrid.of(grid)
    _, rounds = oracle.advect_rounds(og, "runge_kutta_4", 0.02, pos, np.full(600, 80, np.uint64),
                                     250, record=True, index64=False)
    out = tmp_path / "result.rank_0.h5"
    assert len(rounds) == 3
    assert sorted(host.names(out)) == sorted(f"{k}_{i}" for i in range(3)
                                             for k in ("vertices", "colors", "indices"))
    for i, want in enumerate(rounds):
        assert_same(host.read(out, f"vertices_{i}").reshape(-1, 3), want.vertices)
        idx = host.read(out, f"indices_{i}")
        assert host.info(out, f"indices_{i}")[2] == 4  # uint32 (pipeline.cpp:155)
        assert_same(idx, want.indices.astype(np.uint64))
        np.testing.assert_allclose(host.read(out, f"colors_{i}"), want.colors, rtol=0, atol=2e-6)

    xdmf = (tmp_path / "result.rank_0.h5.xdmf").read_text()
    assert xdmf.count('<Grid Name="grid_') == 3
    assert "result.rank_0.h5:/vertices_0" in xdmf and 'TopologyType="Polyline"' in xdmf
    v0 = rounds[0].vertices.shape[0]
    assert f'Dimensions="{3 * v0}"' in xdmf

    csv = (tmp_path / "result.h5.benchmark.csv").read_text().splitlines()
    assert csv[0] == "rank,name,iteration 0,"
    names = [line.split(",")[1] for line in csv[1:]]
    want_names = []
    for i in range(3):
        want_names += [f"round.{i}.load", f"round.{i}.load_balancing_time",
                       f"round.{i}.advection_time", f"round.{i}.communication_time",
                       f"round.{i}.time"]
    assert names == want_names + ["total_time"]
    loads = [float(line.split(",")[2]) for line in csv[1:] if ".load," in line]
    assert loads == [600.0, 350.0, 100.0]


def test_pipeline_ftle_matches_the_oracle(tmp_path, oracle):
    grid = fields.abc_perturbed(48, seed=2)
    host.write_field(tmp_path / "in.h5", grid, "data", "spacing")
    cfg = write_config(tmp_path, seed_generation_stride=[2.0, 2.0, 2.0], estimate_ftle=True,
                       particle_advector_record=False, seed_generation_iterations="40",
                       particle_advector_particles_per_round="100000")
    r = host.run_pipeline(cfg, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    offset, size = seeds.seed_box(grid)
    stride = (grid.spacing * np.float32(2)).astype(np.float32)
    pos = host.lattice_seeds(offset, size, stride)
    og = oracle.OracleGrid.of(grid)
    final, _ = oracle.advect_rounds(og, "runge_kutta_4", 0.02, pos, np.full(len(pos), 40, np.uint64),
                                    100000)
    want, _ = oracle.ftle(grid.shape, grid.offset, grid.spacing, (2, 2, 2), 40, 0.02, pos,
                          final.positions)
    path = tmp_path / "result.rank_0_grid.h5"
    got = host.read(path, "data")
    assert got.shape == want.shape == (24, 24, 24)
    finite = np.isfinite(want)
    assert_same(np.isfinite(got), finite)
    np.testing.assert_allclose(got[finite], want[finite], rtol=1e-3, atol=1e-6)
    xdmf = (tmp_path / "result.rank_0_grid.h5.xdmf").read_text()
    assert "3DCoRectMesh" in xdmf and 'NumberOfElements="24 24 24"' in xdmf
    assert not (tmp_path / "result.rank_0.h5").exists()  # recording off: no curve file


def test_device_seed_generators_match_the_host(ctx):
    import torch
    from dpa_b200 import _native as N
    lib = ctx._lib
    offset = np.zeros(3, np.float32)
    size = np.array([6.5, 3.25, 9.0], np.float32)
    out = torch.zeros((5000, 3), dtype=torch.float32, device="cuda")
    n = C.c_uint64()
    f3 = lambda a: (C.c_float * 3)(*a)
    ctx.check(lib.dpa_seed_random_device(ctx.handle, f3(offset), f3(size), 5000, 11, None,
                                         C.byref(n), C.c_void_p(out.data_ptr()), None))
    ctx.synchronize()
    assert n.value == 5000
    assert_same(out.cpu().numpy(), host.random_seeds(offset, size, 5000, 11))
    stride = np.float32([0.5, 0.25, 0.75])
    shape = (C.c_uint64 * 3)()
    ctx.check(lib.dpa_seed_lattice_device(ctx.handle, f3(offset), f3(size), f3(stride), None,
                                          C.byref(n), shape, None, None))
    lat = torch.zeros((n.value, 3), dtype=torch.float32, device="cuda")
    ctx.check(lib.dpa_seed_lattice_device(ctx.handle, f3(offset), f3(size), f3(stride), None,
                                          C.byref(n), shape, C.c_void_p(lat.data_ptr()), None))
    ctx.synchronize()
    assert_same(lat.cpu().numpy(), host.lattice_seeds(offset, size, stride))
