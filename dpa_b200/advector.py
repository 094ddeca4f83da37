"""Host-side mirror of the reference's advection stage over the C ABI.

Class and argument names follow the reference so that a caller of
``dpa::particle_advector`` (include/dpa/stages/particle_advector.hpp:124-138),
``dpa::ftle_estimator`` (include/dpa/stages/ftle_estimator.hpp) and
``dpa::uniform_seed_generator`` finds the same operations here. All compute
goes through libdpa_b200.so; nothing here computes particles on the CPU.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field as dc_field

import numpy as np

from . import _native as N

UINT32_MAX = 0xFFFFFFFF


@dataclass
class RegularGrid:
    """regular_grid<T, 3> (include/dpa/types/regular_grid.hpp:17-152): C-order
    data [n0][n1][n2](...), world offset, size and cell spacing."""

    data: np.ndarray
    offset: np.ndarray
    size: np.ndarray
    spacing: np.ndarray

    @staticmethod
    def from_data(data: np.ndarray, spacing, offset=(0.0, 0.0, 0.0)) -> "RegularGrid":
        data = np.ascontiguousarray(data, dtype=np.float32)
        spacing = np.asarray(spacing, dtype=np.float32).reshape(3)
        offset = np.asarray(offset, dtype=np.float32).reshape(3)
        # regular_grid_loader.cpp:86-87: size = shape * spacing
        size = (np.asarray(data.shape[:3], dtype=np.float32) * spacing).astype(np.float32)
        return RegularGrid(data, offset, size, spacing)

    @property
    def shape(self) -> tuple[int, int, int]:
        return tuple(int(s) for s in self.data.shape[:3])


@dataclass
class UnsteadyGrid:
    """A time-varying field (no counterpart in the reference): `slices` grids
    of one shape, data [slices][n0][n1][n2][3], slice s at time
    time_origin + s * time_spacing."""

    data: np.ndarray
    offset: np.ndarray
    spacing: np.ndarray
    time_origin: float
    time_spacing: float

    @staticmethod
    def from_data(data: np.ndarray, spacing, time_spacing: float, offset=(0.0, 0.0, 0.0),
                  time_origin: float = 0.0) -> "UnsteadyGrid":
        data = np.ascontiguousarray(data, dtype=np.float32)
        if data.ndim != 5 or data.shape[-1] != 3 or data.shape[0] < 2:
            raise ValueError("expected data of shape [slices >= 2][n0][n1][n2][3]")
        return UnsteadyGrid(data, np.asarray(offset, np.float32).reshape(3),
                            np.asarray(spacing, np.float32).reshape(3),
                            float(np.float32(time_origin)), float(np.float32(time_spacing)))

    @property
    def shape(self) -> tuple[int, int, int]:
        return tuple(int(s) for s in self.data.shape[1:4])

    @property
    def slices(self) -> int:
        return int(self.data.shape[0])

    def slice(self, s: int) -> RegularGrid:
        return RegularGrid.from_data(self.data[s], self.spacing, self.offset)


@dataclass
class Particles:
    """Structure-of-arrays form of particle_3d (include/dpa/types/particle.hpp:12-77)."""

    position: np.ndarray                 # float32 [N, 3]
    remaining_iterations: np.ndarray     # uint64 [N]
    original_position: np.ndarray        # float32 [N, 3]
    termination: np.ndarray | None = None  # uint8 [N], set by advection

    @staticmethod
    def create(positions, iterations) -> "Particles":
        p = np.ascontiguousarray(positions, dtype=np.float32).reshape(-1, 3)
        rem = np.broadcast_to(np.asarray(iterations, dtype=np.uint64), (p.shape[0],)).copy()
        return Particles(p.copy(), rem, p.copy())

    def __len__(self) -> int:
        return int(self.position.shape[0])

    def copy(self) -> "Particles":
        return Particles(self.position.copy(), self.remaining_iterations.copy(),
                         self.original_position.copy(),
                         None if self.termination is None else self.termination.copy())


@dataclass
class IntegralCurve:
    """integral_curve (include/dpa/types/integral_curves.hpp:11-18) of one round."""

    vertices: np.ndarray   # float32 [V, 3]
    colors: np.ndarray     # float32 [V]
    indices: np.ndarray    # uint32 or uint64 [I]


@dataclass
class AdvectOutput:
    """particle_advector::output (particle_advector.hpp:85-89)."""

    inactive_particles: Particles
    integral_curves: list = dc_field(default_factory=list)
    rounds: int = 0


class Context:
    """A device context (dpa_context): one CUDA device, one stream."""

    def __init__(self, device: int = 0):
        self._lib = N.load()
        handle = C.c_void_p()
        st = self._lib.dpa_context_create(int(device), C.byref(handle))
        if st != N.DPA_OK:
            raise N.DpaError(st, f"cannot create a context on CUDA device {device}")
        self.handle = handle
        self.device = int(device)

    def close(self) -> None:
        if self.handle:
            self._lib.dpa_context_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def check(self, status: int) -> None:
        N.check(status, self.handle)

    @property
    def stream(self) -> int:
        return int(self._lib.dpa_context_stream(self.handle) or 0)

    def synchronize(self) -> None:
        self.check(self._lib.dpa_context_synchronize(self.handle))

    def set_staging_limit(self, nbytes: int) -> None:
        self.check(self._lib.dpa_context_set_staging_limit(self.handle, int(nbytes)))

    def field(self, grid: RegularGrid, storage: str = "f32") -> "Field":
        return Field(self, grid, storage)


def _f3(values) -> C.Array:
    return (C.c_float * 3)(*[float(v) for v in np.asarray(values, dtype=np.float32).reshape(3)])


def _u3(values) -> C.Array:
    return (C.c_uint64 * 3)(*[int(v) for v in values])


class Field:
    """A field resident on the device (dpa_field), repacked to `storage`."""

    def __init__(self, context: Context, grid: RegularGrid, storage: str = "f32",
                 device_pointer: int | None = None):
        self.context = context
        self.grid = grid
        self.storage = storage
        handle = C.c_void_p()
        lib = context._lib
        if isinstance(grid, UnsteadyGrid):
            if device_pointer is not None:
                raise ValueError("time-varying fields are uploaded from host memory")
            data = np.ascontiguousarray(grid.data, dtype=np.float32)
            st = lib.dpa_field_create_unsteady(context.handle, data.ctypes.data_as(C.c_void_p),
                                               _u3(grid.shape), grid.slices, _f3(grid.offset),
                                               _f3(grid.spacing), grid.time_origin,
                                               grid.time_spacing, N.STORAGE[storage],
                                               C.byref(handle))
        elif device_pointer is None:
            data = np.ascontiguousarray(grid.data, dtype=np.float32)
            st = lib.dpa_field_create(context.handle, data.ctypes.data_as(C.c_void_p),
                                      _u3(grid.shape), _f3(grid.offset), _f3(grid.spacing),
                                      N.STORAGE[storage], C.byref(handle))
        else:
            st = lib.dpa_field_create_device(context.handle, C.c_void_p(device_pointer),
                                             _u3(grid.shape), _f3(grid.offset),
                                             _f3(grid.spacing), N.STORAGE[storage],
                                             C.byref(handle))
        context.check(st)
        self.handle = handle

    def close(self) -> None:
        if self.handle and self.context.handle:
            self.context._lib.dpa_field_destroy(self.context.handle, self.handle)
        self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def device_bytes(self) -> int:
        b = C.c_uint64()
        N.check(self.context._lib.dpa_field_info(self.handle, None, None, None, None, C.byref(b)))
        return int(b.value)


class _CurveCollector:
    """Curve sink that concatenates a round's chunks into numpy arrays."""

    def __init__(self, index64: bool):
        self.index64 = index64
        self.vertices, self.colors, self.indices = [], [], []
        self.callback = N.CURVE_SINK(self._on_chunk)

    def _on_chunk(self, user, chunk_ptr) -> int:
        c = chunk_ptr.contents
        v = int(c.vertex_count)
        if v:
            self.vertices.append(np.ctypeslib.as_array(c.vertices, shape=(v * 3,)).reshape(v, 3).copy())
            if c.colors:
                self.colors.append(np.ctypeslib.as_array(c.colors, shape=(v,)).copy())
        i = int(c.index_count)
        if i:
            ctype = C.c_uint64 if self.index64 else C.c_uint32
            ptr = C.cast(c.indices, C.POINTER(ctype))
            self.indices.append(np.ctypeslib.as_array(ptr, shape=(i,)).copy())
        return 0

    def curve(self) -> IntegralCurve:
        itype = np.uint64 if self.index64 else np.uint32
        vert = np.concatenate(self.vertices) if self.vertices else np.zeros((0, 3), np.float32)
        col = np.concatenate(self.colors) if self.colors else np.zeros(0, np.float32)
        idx = np.concatenate(self.indices) if self.indices else np.zeros(0, itype)
        return IntegralCurve(vert, col, idx.astype(itype, copy=False))


LOAD_BALANCERS = ("none", "diffuse_constant", "diffuse_lesser_average",
                  "diffuse_greater_limited_lesser_average")


class ParticleAdvector:
    """particle_advector (particle_advector.hpp:124-131; particle_advector.cpp:17-55)
    at world size 1: rounds of at most particles_per_round particles taken
    from the tail of the active particles, every particle of a round
    finishing within it (no neighbour ranks exist to hand particles to)."""

    def __init__(self, context: Context, particles_per_round: int, load_balancer: str,
                 integrator: str, step_size: float, gather_particles: bool, record: bool,
                 use_64_bit_indices: bool | None = None, colors: bool = True,
                 morton_order: bool = True):
        if load_balancer not in LOAD_BALANCERS:
            load_balancer = "none"  # particle_advector.cpp:24-27 falls back silently
        if integrator not in N.INTEGRATORS:
            raise ValueError(f"unknown integrator {integrator!r}")
        if int(particles_per_round) <= 0:
            raise ValueError("particles_per_round must be positive")
        self.context = context
        self.particles_per_round = int(particles_per_round)
        self.load_balancer = load_balancer
        self.integrator = integrator
        self.step_size = float(np.float32(step_size))
        self.gather_particles = bool(gather_particles)
        self.record = bool(record)
        self.use_64_bit_indices = use_64_bit_indices
        self.colors = bool(colors)
        self.morton_order = bool(morton_order)

    def options(self, index64: bool) -> N.AdvectOptions:
        return N.AdvectOptions(N.INTEGRATORS[self.integrator], self.step_size,
                               int(self.record), int(index64), int(self.colors),
                               int(self.morton_order))

    def index64_for(self, iterations: int) -> bool:
        # pipeline.cpp:155: particles_per_round * iterations > UINT32_MAX
        if self.use_64_bit_indices is not None:
            return bool(self.use_64_bit_indices)
        return self.particles_per_round * int(iterations) > UINT32_MAX

    def advect_round(self, field: Field, positions: np.ndarray, remaining: np.ndarray,
                     index64: bool) -> tuple[np.ndarray, IntegralCurve | None]:
        """One round over contiguous arrays, updated in place. Returns the
        termination reasons and, when recording, the round's curve."""
        lib = self.context._lib
        n = int(positions.shape[0])
        term = np.zeros(n, dtype=np.uint8)
        opts = self.options(index64)
        collector = _CurveCollector(index64) if self.record else None
        sink = collector.callback if collector else N.CURVE_SINK()
        st = lib.dpa_advect_round(self.context.handle, field.handle, C.byref(opts), n,
                                  positions.ctypes.data_as(C.c_void_p),
                                  remaining.ctypes.data_as(C.c_void_p),
                                  term.ctypes.data_as(C.c_void_p), sink, None)
        self.context.check(st)
        return term, (collector.curve() if collector else None)

    def advect(self, field: Field, particles: Particles) -> AdvectOutput:
        """particle_advector::advect (particle_advector.cpp:39-55). The
        particles are consumed; the output holds every particle's final state
        in the original order, and one curve per round when recording."""
        total = len(particles)
        positions = np.ascontiguousarray(particles.position, dtype=np.float32).copy()
        remaining = np.ascontiguousarray(particles.remaining_iterations, dtype=np.uint64).copy()
        termination = np.zeros(total, dtype=np.uint8)
        iterations = int(remaining.max()) if total else 0
        index64 = self.index64_for(iterations)
        curves = []
        active = total
        rounds = 0
        while active > 0:  # check_completion at world size 1
            # compute_round_state (particle_advector.cpp:261-310): the tail.
            count = min(self.particles_per_round, active)
            lo, hi = active - count, active
            pos = np.ascontiguousarray(positions[lo:hi])
            rem = np.ascontiguousarray(remaining[lo:hi])
            term, curve = self.advect_round(field, pos, rem, index64)
            positions[lo:hi] = pos
            remaining[lo:hi] = rem
            termination[lo:hi] = term
            if curve is not None:
                curves.append(curve)
            active = lo
            rounds += 1
        out = Particles(positions, remaining, particles.original_position.copy(), termination)
        return AdvectOutput(out, curves, rounds)


def estimate_ftle(context: Context, field: Field, seed_maximum_iterations: int, seed_stride,
                  step_size: float, particles: Particles, mapping: str = "reference") -> RegularGrid:
    """ftle_estimator::estimate (ftle_estimator.cpp:7-65)."""
    lib = context._lib
    shape = (C.c_uint64 * 3)()
    stride = _f3(seed_stride)
    n = len(particles)
    orig = np.ascontiguousarray(particles.original_position, dtype=np.float32)
    final = np.ascontiguousarray(particles.position, dtype=np.float32)
    context.check(lib.dpa_ftle_estimate(context.handle, field.handle, stride,
                                        int(seed_maximum_iterations), float(step_size), n,
                                        orig.ctypes.data_as(C.c_void_p),
                                        final.ctypes.data_as(C.c_void_p),
                                        N.FTLE_MAPPING[mapping], None, shape))
    dims = tuple(int(s) for s in shape)
    out = np.zeros(dims, dtype=np.float32)
    context.check(lib.dpa_ftle_estimate(context.handle, field.handle, stride,
                                        int(seed_maximum_iterations), float(step_size), n,
                                        orig.ctypes.data_as(C.c_void_p),
                                        final.ctypes.data_as(C.c_void_p),
                                        N.FTLE_MAPPING[mapping],
                                        out.ctypes.data_as(C.c_void_p), shape))
    spacing = (field.grid.spacing * np.asarray(seed_stride, dtype=np.float32)).astype(np.float32)
    return RegularGrid(out, field.grid.offset.copy(), field.grid.size.copy(), spacing)


@dataclass
class PathlineResult:
    position: np.ndarray
    time: np.ndarray
    remaining_iterations: np.ndarray
    termination: np.ndarray


def advect_pathlines(context: Context, field: Field, positions, times, iterations,
                     integrator: str = "runge_kutta_4", step_size: float = 0.25,
                     max_steps: int = 0, morton_order: bool = True) -> PathlineResult:
    """Pathlines (end states) through a field, each particle starting at its
    own time, via dpa_advect_pathlines_device on device copies of the inputs."""
    import torch
    pos = torch.from_numpy(np.ascontiguousarray(positions, np.float32).reshape(-1, 3)).cuda()
    n = pos.shape[0]
    t = torch.from_numpy(np.broadcast_to(np.asarray(times, np.float32), (n,)).copy()).cuda()
    rem = torch.from_numpy(
        np.broadcast_to(np.asarray(iterations, np.uint64), (n,)).astype(np.int64)).cuda()
    term = torch.zeros(n, dtype=torch.uint8, device="cuda")
    opts = N.AdvectOptions(N.INTEGRATORS[integrator], float(np.float32(step_size)), 0, 0, 0,
                           int(morton_order), int(max_steps))
    ptr = lambda x: C.c_void_p(x.data_ptr())
    torch.cuda.synchronize()
    context.check(context._lib.dpa_advect_pathlines_device(
        context.handle, field.handle, C.byref(opts), n, ptr(pos), ptr(t), ptr(rem), ptr(term),
        None))
    context.synchronize()
    return PathlineResult(pos.cpu().numpy(), t.cpu().numpy(),
                          rem.cpu().numpy().astype(np.uint64), term.cpu().numpy())
