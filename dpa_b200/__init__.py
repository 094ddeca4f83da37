"""dpa_b200 -- B200 (sm_100a) advection stage of VRGroupRWTH/dpa.

The compute lives in libdpa_b200.so (C ABI: include/dpa_b200.h). This package
is the host-side mirror of the reference's stage interface over that ABI:

    from dpa_b200 import Context, ParticleAdvector, fields, seeds
    with Context(0) as ctx:
        grid = fields.abc(64)
        field = ctx.field(grid)
        offset, size = seeds.seed_box(grid)
        particles = seeds.generate_random(offset, size, 4096, 1000, seed=0)
        out = ParticleAdvector(ctx, 4096, "none", "runge_kutta_4", 0.01,
                               False, True).advect(field, particles)
"""
from ._native import DpaError, load as load_library
from .advector import (AdvectOutput, Context, Field, IntegralCurve, ParticleAdvector, Particles,
                       PathlineResult, RegularGrid, UnsteadyGrid, advect_pathlines, estimate_ftle)
from . import fields, seeds

__all__ = [
    "AdvectOutput", "Context", "DpaError", "Field", "IntegralCurve", "ParticleAdvector",
    "Particles", "PathlineResult", "RegularGrid", "UnsteadyGrid", "advect_pathlines",
    "estimate_ftle", "fields", "load_library", "seeds",
]
