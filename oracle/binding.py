"""ctypes wrapper of the CPU oracle (oracle/liboracle.so) for tests and the
CPU baseline. Test infrastructure only: the oracle is the checker, never the
thing measured as the product."""
from __future__ import annotations

import ctypes as C
import subprocess
from dataclasses import dataclass
from pathlib import Path

import numpy as np

ORACLE_DIR = Path(__file__).resolve().parent
ORACLE_LIB = ORACLE_DIR / "liboracle.so"

EULER, RK4, RK4_TRUE = 0, 2, 100
# include/dpa/types/integrators.hpp:31-39 order; 100 has no reference counterpart.
INTEGRATOR_CODES = {"euler": EULER, "modified_midpoint": 1, "runge_kutta_4": RK4,
                    "runge_kutta_cash_karp_54": 3, "runge_kutta_dormand_prince_5": 4,
                    "runge_kutta_fehlberg_78": 5, "adams_bashforth_2": 6,
                    "adams_bashforth_moulton_2": 7, "runge_kutta_4_true": RK4_TRUE}


class Grid(C.Structure):
    _fields_ = [("data", C.c_void_p), ("shape", C.c_uint64 * 3), ("offset", C.c_float * 3),
                ("spacing", C.c_float * 3)]


class UnsteadyGridC(C.Structure):
    _fields_ = [("data", C.c_void_p), ("shape", C.c_uint64 * 3), ("slices", C.c_uint64),
                ("offset", C.c_float * 3), ("spacing", C.c_float * 3),
                ("time_origin", C.c_float), ("time_spacing", C.c_float)]


_lib = None


def build() -> Path:
    src = [ORACLE_DIR / "oracle.cpp", ORACLE_DIR / "oracle.h"]
    if not ORACLE_LIB.exists() or any(s.stat().st_mtime > ORACLE_LIB.stat().st_mtime for s in src):
        subprocess.run(["make", "-s", "-C", str(ORACLE_DIR)], check=True)
    return ORACLE_LIB


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(str(ORACLE_LIB))
        P = C.c_void_p
        L.oracle_set_threads.argtypes = [C.c_int]
        L.oracle_get_threads.restype = C.c_int
        L.oracle_contains.argtypes = [P, P]
        L.oracle_contains.restype = C.c_int
        L.oracle_interpolate.argtypes = [P, P, P]
        L.oracle_advect_round.argtypes = [P, C.c_int, C.c_float, C.c_uint64, P, P, P, P, C.c_int,
                                          C.c_uint64, P]
        L.oracle_advect_round.restype = C.c_int
        L.oracle_advect_pathlines.argtypes = [P, C.c_int, C.c_float, C.c_uint64, P, P, P, P, P]
        L.oracle_advect_pathlines.restype = C.c_int
        L.oracle_prune.argtypes = [P, C.c_uint64]
        L.oracle_prune.restype = C.c_uint64
        L.oracle_generate_indices.argtypes = [P, C.c_uint64, C.c_int, P]
        L.oracle_generate_indices.restype = C.c_uint64
        L.oracle_generate_colors.argtypes = [P, C.c_uint64, P]
        L.oracle_lattice_seeds.argtypes = [P, P, P, P, P, P]
        L.oracle_lattice_seeds.restype = C.c_uint64
        L.oracle_ftle.argtypes = [P, P, P, P, C.c_uint64, C.c_float, C.c_uint64, P, P, C.c_int,
                                  P, P, P, P, P]
        L.oracle_ftle.restype = C.c_int
        L.oracle64_advect.argtypes = [P, C.c_int, C.c_double, C.c_uint64, P, P, P, P]
        L.oracle64_advect.restype = C.c_int
        L.oracle64_advect_abc.argtypes = [C.c_double, C.c_double, C.c_double, P, P, C.c_double,
                                          C.c_uint64, P, P, P, P]
        L.oracle64_advect_abc.restype = C.c_int
        _lib = L
    return _lib


def _ptr(a: np.ndarray) -> C.c_void_p:
    return a.ctypes.data_as(C.c_void_p)


class OracleGrid:
    def __init__(self, data: np.ndarray, spacing, offset=(0, 0, 0)):
        self.data = np.ascontiguousarray(data, dtype=np.float32)
        self.g = Grid(self.data.ctypes.data, (C.c_uint64 * 3)(*self.data.shape[:3]),
                      (C.c_float * 3)(*np.asarray(offset, np.float32)),
                      (C.c_float * 3)(*np.asarray(spacing, np.float32)))

    @staticmethod
    def of(grid) -> "OracleGrid":
        return OracleGrid(grid.data, grid.spacing, grid.offset)

    @property
    def ref(self):
        return C.byref(self.g)


def set_threads(n: int) -> None:
    lib().oracle_set_threads(int(n))


def contains(grid: OracleGrid, p) -> bool:
    p = np.asarray(p, np.float32)
    return bool(lib().oracle_contains(grid.ref, _ptr(p)))


def interpolate(grid: OracleGrid, p) -> np.ndarray:
    p = np.asarray(p, np.float32)
    out = np.zeros(3, np.float32)
    lib().oracle_interpolate(grid.ref, _ptr(p), _ptr(out))
    return out


@dataclass
class RoundResult:
    positions: np.ndarray
    remaining: np.ndarray
    termination: np.ndarray
    steps: np.ndarray
    vertices: np.ndarray | None = None
    colors: np.ndarray | None = None
    indices: np.ndarray | None = None


def advect_round(grid: OracleGrid, integrator: str, step: float, positions, remaining,
                 record: bool = False, index64: bool = False) -> RoundResult:
    """allocate_integral_curves + advect + prune_integral_curves for one round,
    then (when recording) the index and color post-passes on its curve."""
    pos = np.ascontiguousarray(positions, np.float32).copy()
    rem = np.ascontiguousarray(remaining, np.uint64).copy()
    n = pos.shape[0]
    term = np.zeros(n, np.uint8)
    steps = np.zeros(n, np.uint64)
    stride = int(rem.max()) + 2 if (record and n) else 0
    raw = np.zeros(n * stride * 3 if record else 1, np.float32)
    st = lib().oracle_advect_round(grid.ref, INTEGRATOR_CODES[integrator], float(step), n,
                                   _ptr(pos), _ptr(rem), _ptr(term), _ptr(steps), int(record),
                                   stride, _ptr(raw))
    assert st == 0, st
    res = RoundResult(pos, rem, term, steps)
    if record:
        kept = lib().oracle_prune(_ptr(raw), n * stride)
        verts = raw[: kept * 3].reshape(kept, 3).copy()
        res.vertices = verts
        idx = np.zeros(2 * kept, np.uint64 if index64 else np.uint32)
        ni = lib().oracle_generate_indices(_ptr(verts), kept, int(index64), _ptr(idx))
        res.indices = idx[:ni].copy()
        col = np.zeros(kept, np.float32)
        lib().oracle_generate_colors(_ptr(verts), kept, _ptr(col))
        res.colors = col
    return res


def advect_rounds(grid: OracleGrid, integrator: str, step: float, positions, remaining,
                  particles_per_round: int, record: bool = False, index64: bool = False):
    """The world-size-1 round loop: each round takes the tail of the active
    particles (particle_advector.cpp:261-310). Returns final states in the
    original order and the per-round results."""
    pos = np.ascontiguousarray(positions, np.float32).copy()
    rem = np.ascontiguousarray(remaining, np.uint64).copy()
    term = np.zeros(pos.shape[0], np.uint8)
    steps = np.zeros(pos.shape[0], np.uint64)
    rounds = []
    active = pos.shape[0]
    while active > 0:
        count = min(particles_per_round, active)
        lo = active - count
        r = advect_round(grid, integrator, step, pos[lo:active], rem[lo:active], record, index64)
        pos[lo:active], rem[lo:active] = r.positions, r.remaining
        term[lo:active], steps[lo:active] = r.termination, r.steps
        rounds.append(r)
        active = lo
    return RoundResult(pos, rem, term, steps), rounds


def lattice_seeds(offset, size, stride, aabb=None):
    offset = np.asarray(offset, np.float32)
    size = np.asarray(size, np.float32)
    stride = np.asarray(stride, np.float32)
    box = None if aabb is None else np.concatenate([np.asarray(aabb[0], np.float32),
                                                    np.asarray(aabb[1], np.float32)])
    shape = np.zeros(3, np.uint64)
    n = lib().oracle_lattice_seeds(_ptr(offset), _ptr(size), _ptr(stride),
                                   None if box is None else _ptr(box), _ptr(shape), None)
    out = np.zeros((n, 3), np.float32)
    lib().oracle_lattice_seeds(_ptr(offset), _ptr(size), _ptr(stride),
                               None if box is None else _ptr(box), _ptr(shape), _ptr(out))
    return out, tuple(int(s) for s in shape)


def ftle(field_shape, offset, spacing, seed_stride, iterations, step, original, final,
         mapping: int = 0):
    fs = np.asarray(field_shape, np.uint64)
    off = np.asarray(offset, np.float32)
    sp = np.asarray(spacing, np.float32)
    st = np.asarray(seed_stride, np.float32)
    orig = np.ascontiguousarray(original, np.float32)
    fin = np.ascontiguousarray(final, np.float32)
    shape = np.zeros(3, np.uint64)
    cells = 1
    for i in range(3):
        cells *= int(np.float32(fs[i]) / st[i])
    out = np.zeros(cells, np.float32)
    coll = C.c_uint64()
    holes = C.c_uint64()
    outside = C.c_uint64()
    rc = lib().oracle_ftle(_ptr(fs), _ptr(off), _ptr(sp), _ptr(st), int(iterations), float(step),
                           orig.shape[0], _ptr(orig), _ptr(fin), int(mapping), _ptr(out),
                           _ptr(shape), C.byref(coll), C.byref(holes), C.byref(outside))
    assert rc == 0, rc
    dims = tuple(int(s) for s in shape)
    return out.reshape(dims), {"collisions": coll.value, "holes": holes.value,
                               "outside": outside.value}


def advect64(grid: OracleGrid, integrator: str, step: float, positions, remaining):
    pos = np.ascontiguousarray(positions, np.float64).copy()
    rem = np.ascontiguousarray(remaining, np.uint64).copy()
    n = pos.shape[0]
    term = np.zeros(n, np.uint8)
    steps = np.zeros(n, np.uint64)
    rc = lib().oracle64_advect(grid.ref, INTEGRATOR_CODES[integrator], float(step), n, _ptr(pos),
                               _ptr(rem), _ptr(term), _ptr(steps))
    assert rc == 0
    return RoundResult(pos, rem, term, steps)


def advect64_abc(A, B, Cc, lo, hi, step, positions, remaining):
    pos = np.ascontiguousarray(positions, np.float64).copy()
    rem = np.ascontiguousarray(remaining, np.uint64).copy()
    n = pos.shape[0]
    term = np.zeros(n, np.uint8)
    steps = np.zeros(n, np.uint64)
    lo = np.asarray(lo, np.float64)
    hi = np.asarray(hi, np.float64)
    rc = lib().oracle64_advect_abc(A, B, Cc, _ptr(lo), _ptr(hi), float(step), n, _ptr(pos),
                                   _ptr(rem), _ptr(term), _ptr(steps))
    assert rc == 0
    return RoundResult(pos, rem, term, steps)


def advect_pathlines(grid, integrator: str, step: float, positions, times, remaining) -> RoundResult:
    """Pathlines through a time-varying field (an object with data [S][n0][n1][n2][3],
    offset, spacing, time_origin, time_spacing). The result's `steps` holds the
    steps taken and its extra attribute `times` the final times."""
    data = np.ascontiguousarray(grid.data, np.float32)
    g = UnsteadyGridC(data.ctypes.data, (C.c_uint64 * 3)(*data.shape[1:4]), data.shape[0],
                      (C.c_float * 3)(*np.asarray(grid.offset, np.float32)),
                      (C.c_float * 3)(*np.asarray(grid.spacing, np.float32)),
                      float(np.float32(grid.time_origin)), float(np.float32(grid.time_spacing)))
    pos = np.ascontiguousarray(positions, np.float32).reshape(-1, 3).copy()
    n = pos.shape[0]
    t = np.broadcast_to(np.asarray(times, np.float32), (n,)).copy()
    rem = np.broadcast_to(np.asarray(remaining, np.uint64), (n,)).copy()
    term = np.zeros(n, np.uint8)
    steps = np.zeros(n, np.uint64)
    rc = lib().oracle_advect_pathlines(C.byref(g), INTEGRATOR_CODES[integrator], float(step), n,
                                       _ptr(pos), _ptr(t), _ptr(rem), _ptr(term), _ptr(steps))
    assert rc == 0, rc
    res = RoundResult(pos, rem, term, steps)
    res.times = t
    return res
