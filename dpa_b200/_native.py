"""ctypes binding of the C ABI declared in include/dpa_b200.h.

The shared library is built in-tree (``python -m dpa_b200.build``) and loaded
from ``dpa_b200/libdpa_b200.so``. There is no fallback: when the library is
missing every use of the package raises.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIBRARY_PATH = Path(__file__).resolve().parent / "libdpa_b200.so"

DPA_OK = 0
STATUS_NAMES = {
    0: "DPA_OK",
    1: "DPA_ERROR_INVALID_ARGUMENT",
    2: "DPA_ERROR_UNSUPPORTED",
    3: "DPA_ERROR_OUT_OF_MEMORY",
    4: "DPA_ERROR_CUDA",
    5: "DPA_ERROR_SINK",
    6: "DPA_ERROR_INTERNAL",
    7: "DPA_ERROR_TIMEOUT",
    8: "DPA_ERROR_CANCELLED",
}

STORAGE = {"f32": 0, "f16": 1, "bf16": 2, "f32_edges": 3}

INTEGRATORS = {
    "euler": 0,
    "modified_midpoint": 1,
    "runge_kutta_4": 2,
    "runge_kutta_cash_karp_54": 3,
    "runge_kutta_dormand_prince_5": 4,
    "runge_kutta_fehlberg_78": 5,
    "adams_bashforth_2": 6,
    "adams_bashforth_moulton_2": 7,
    "runge_kutta_4_true": 100,
}

TERMINATION = {0: "complete", 1: "out_of_bounds", 2: "zero_velocity", 3: "in_flight",
               4: "cancelled"}

FTLE_MAPPING = {"reference": 0, "lattice": 1}

NO_ALLOC_MAX_PARTICLES = 1 << 20


class AdvectOptions(C.Structure):
    _fields_ = [
        ("integrator", C.c_int32),
        ("step_size", C.c_float),
        ("record", C.c_int32),
        ("index64", C.c_int32),
        ("colors", C.c_int32),
        ("morton_order", C.c_int32),
        ("max_steps", C.c_uint64),
    ]


class CurveChunk(C.Structure):
    _fields_ = [
        ("vertex_offset", C.c_uint64),
        ("vertex_count", C.c_uint64),
        ("vertices", C.POINTER(C.c_float)),
        ("colors", C.POINTER(C.c_float)),
        ("index_offset", C.c_uint64),
        ("index_count", C.c_uint64),
        ("indices", C.c_void_p),
        ("last", C.c_int32),
    ]


class Tuning(C.Structure):
    _fields_ = [
        ("claim", C.c_uint32),
        ("blocks_per_sm", C.c_uint32),
        ("order", C.c_uint32),
        ("measured_ms", C.c_float),
        ("block_size", C.c_uint32),
        ("particles_per_thread", C.c_uint32),
    ]


class ServerOptions(C.Structure):
    _fields_ = [
        ("particle_capacity", C.c_uint64),
        ("vertex_capacity", C.c_uint64),
        ("steps_per_tick", C.c_uint32),
        ("max_requests", C.c_uint32),
        ("small_request_seeds", C.c_uint64),
        ("reserved_percent", C.c_uint32),
        ("max_bypass_ms", C.c_uint32),
        ("response_bytes", C.c_uint64),
    ]


class Request(C.Structure):
    _fields_ = [
        ("field", C.c_int32),
        ("integrator", C.c_int32),
        ("step_size", C.c_float),
        ("record", C.c_int32),
        ("index64", C.c_int32),
        ("ftle", C.c_int32),
        ("seed_stride", C.c_float * 3),
        ("count", C.c_uint64),
        ("positions", C.POINTER(C.c_float)),
        ("iterations", C.c_uint64),
        ("user", C.c_void_p),
        ("start_time", C.c_float),
        ("deadline_ms", C.c_uint32),
    ]


class Response(C.Structure):
    _fields_ = [
        ("id", C.c_uint64),
        ("user", C.c_void_p),
        ("status", C.c_int32),
        ("count", C.c_uint64),
        ("positions", C.POINTER(C.c_float)),
        ("remaining", C.POINTER(C.c_uint64)),
        ("termination", C.POINTER(C.c_uint8)),
        ("vertex_count", C.c_uint64),
        ("vertices", C.POINTER(C.c_float)),
        ("colors", C.POINTER(C.c_float)),
        ("index_count", C.c_uint64),
        ("indices", C.c_void_p),
        ("ftle_shape", C.c_uint64 * 3),
        ("ftle", C.POINTER(C.c_float)),
        ("particle_steps", C.c_uint64),
        ("queued_seconds", C.c_double),
        ("admitted_seconds", C.c_double),
        ("finished_seconds", C.c_double),
        ("times", C.POINTER(C.c_float)),
    ]


class ServerStats(C.Structure):
    _fields_ = [
        ("submitted", C.c_uint64),
        ("admitted", C.c_uint64),
        ("completed", C.c_uint64),
        ("ticks", C.c_uint64),
        ("launches", C.c_uint64),
        ("particle_steps", C.c_uint64),
        ("busy_seconds", C.c_double),
        ("queued", C.c_uint32),
        ("active", C.c_uint32),
        ("tick_device_seconds", C.c_double),
        ("peak_slots", C.c_uint64),
        ("peak_vertices", C.c_uint64),
        ("slot_refusals", C.c_uint64),
        ("vertex_refusals", C.c_uint64),
        ("overdue_scans", C.c_uint64),
        ("peak_finishing", C.c_uint32),
        ("reserved0", C.c_uint32),
        ("finish_seconds", C.c_double),
    ]


CURVE_SINK = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(CurveChunk))

_P = C.c_void_p
_U64P = C.POINTER(C.c_uint64)
_F32P = C.POINTER(C.c_float)

# name -> (restype, argtypes); every function the header declares.
SIGNATURES = {
    "dpa_version": (C.c_char_p, []),
    "dpa_device_count": (C.c_int, [C.POINTER(C.c_int)]),
    "dpa_context_create": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    "dpa_context_destroy": (C.c_int, [_P]),
    "dpa_last_error": (C.c_char_p, [_P]),
    "dpa_context_stream": (C.c_void_p, [_P]),
    "dpa_context_synchronize": (C.c_int, [_P]),
    "dpa_context_set_staging_limit": (C.c_int, [_P, C.c_uint64]),
    "dpa_context_set_host_chunk_limit": (C.c_int, [_P, C.c_uint64]),
    "dpa_context_set_profiling": (C.c_int, [_P, C.c_int32]),
    "dpa_context_last_timing": (C.c_int, [_P, _F32P, _F32P]),
    "dpa_context_last_emit_timing": (C.c_int, [_P, _F32P]),
    "dpa_context_launch_count": (C.c_int, [_P, _U64P]),
    "dpa_measure_gather_bandwidth": (C.c_int, [_P, C.c_uint64, C.c_int32,
                                               C.POINTER(C.c_double)]),
    "dpa_integrator_from_name": (C.c_int, [C.c_char_p, C.POINTER(C.c_int32)]),
    "dpa_field_create": (C.c_int, [_P, _P, _U64P, _F32P, _F32P, C.c_int32, C.POINTER(C.c_void_p)]),
    "dpa_field_create_device": (C.c_int, [_P, _P, _U64P, _F32P, _F32P, C.c_int32,
                                          C.POINTER(C.c_void_p)]),
    "dpa_field_destroy": (C.c_int, [_P, _P]),
    "dpa_field_info": (C.c_int, [_P, _U64P, _F32P, _F32P, C.POINTER(C.c_int32), _U64P]),
    "dpa_field_create_unsteady": (C.c_int, [_P, _P, _U64P, C.c_uint32, _F32P, _F32P, C.c_float,
                                            C.c_float, C.c_int32, C.POINTER(C.c_void_p)]),
    "dpa_field_time_info": (C.c_int, [_P, C.POINTER(C.c_uint32), _F32P, _F32P]),
    "dpa_field_locate_mode": (C.c_int, [_P, C.POINTER(C.c_int32)]),
    "dpa_context_set_ieee_division": (C.c_int, [_P, C.c_int32]),
    "dpa_advect_round": (C.c_int, [_P, _P, C.POINTER(AdvectOptions), C.c_uint64, _P, _P, _P,
                                   CURVE_SINK, _P]),
    "dpa_advect_device": (C.c_int, [_P, _P, C.POINTER(AdvectOptions), C.c_uint64, _P, _P, _P, _P]),
    "dpa_advect_pathlines_device": (C.c_int, [_P, _P, C.POINTER(AdvectOptions), C.c_uint64, _P, _P,
                                              _P, _P, _P]),
    "dpa_advect_batch_device": (C.c_int, [_P, _P, C.POINTER(AdvectOptions), C.c_uint64, _U64P,
                                          _P, _P, _P, _U64P, _P]),
    "dpa_graph_create_advect": (C.c_int, [_P, _P, C.POINTER(AdvectOptions), C.c_uint64, _P, _P,
                                          _P, C.POINTER(C.c_void_p)]),
    "dpa_graph_launch": (C.c_int, [_P, _P, _P]),
    "dpa_graph_destroy": (C.c_int, [_P, _P]),
    "dpa_context_set_tuning": (C.c_int, [_P, C.POINTER(Tuning)]),
    "dpa_context_get_tuning": (C.c_int, [_P, C.POINTER(Tuning)]),
    "dpa_autotune_advect": (C.c_int, [_P, _P, C.POINTER(AdvectOptions), C.c_uint64, _P, _P,
                                      C.c_uint64, C.POINTER(Tuning)]),
    "dpa_server_create": (C.c_int, [_P, C.POINTER(ServerOptions), C.POINTER(C.c_void_p)]),
    "dpa_server_add_field": (C.c_int, [_P, _P, C.POINTER(C.c_int32)]),
    "dpa_server_submit": (C.c_int, [_P, C.POINTER(Request), _U64P]),
    "dpa_server_poll": (C.c_int, [_P, C.c_int32, C.POINTER(Response), C.POINTER(C.c_int32)]),
    "dpa_server_release": (C.c_int, [_P, C.c_uint64]),
    "dpa_server_cancel": (C.c_int, [_P, C.c_uint64]),
    "dpa_server_get_stats": (C.c_int, [_P, C.POINTER(ServerStats)]),
    "dpa_server_destroy": (C.c_int, [_P]),
    "dpa_advect_device_no_alloc": (C.c_int, [_P, _P, C.POINTER(AdvectOptions), C.c_uint64, _P, _P,
                                             _P, _P]),
    "dpa_seed_lattice_device": (C.c_int, [_P, _F32P, _F32P, _F32P, _F32P, _U64P, _U64P, _P, _P]),
    "dpa_seed_random_device": (C.c_int, [_P, _F32P, _F32P, C.c_uint64, C.c_uint64, _F32P, _U64P,
                                         _P, _P]),
    "dpa_ftle_estimate": (C.c_int, [_P, _P, _F32P, C.c_uint64, C.c_float, C.c_uint64, _P, _P,
                                    C.c_int32, _P, _U64P]),
    "dpa_ftle_estimate_device": (C.c_int, [_P, _P, _F32P, C.c_uint64, C.c_float, C.c_uint64, _P,
                                           _P, C.c_int32, _P, _U64P, _P]),
}

_lib = None


def load() -> C.CDLL:
    """Loads libdpa_b200.so and declares its signatures; raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIBRARY_PATH.exists():
        raise ImportError(
            f"{LIBRARY_PATH} is missing: build it with `python -m dpa_b200.build` "
            "(nvcc, sm_100a). There is no CPU fallback.")
    lib = C.CDLL(str(LIBRARY_PATH))
    for name, (restype, argtypes) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = restype
        fn.argtypes = argtypes
    _lib = lib
    return lib


class DpaError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def check(status: int, ctx=None) -> None:
    if status != DPA_OK:
        lib = load()
        msg = lib.dpa_last_error(ctx).decode() if ctx else ""
        raise DpaError(status, msg)
