"""Host-side binding of the request server (dpa_server_* in include/dpa_b200.h)."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _native as N


@dataclass
class Result:
    """A finished request, copied out of the server."""

    id: int
    status: int
    positions: np.ndarray
    remaining: np.ndarray
    termination: np.ndarray
    vertices: np.ndarray | None
    colors: np.ndarray | None
    indices: np.ndarray | None
    ftle: np.ndarray | None
    particle_steps: int
    queued: float
    admitted: float
    finished: float
    times: np.ndarray | None = None  # each particle's time at its end

    @property
    def latency(self) -> float:
        return self.finished - self.queued


class Server:
    """Continuous-batching request server over resident fields."""

    def __init__(self, context, particle_capacity: int, vertex_capacity: int = 0,
                 steps_per_tick: int = 64, max_requests: int = 256, small_request_seeds: int = 0,
                 reserved_percent: int = 0, max_bypass_ms: int = 0, response_bytes: int = 0):
        self.context = context
        self._lib = context._lib
        opts = N.ServerOptions(int(particle_capacity), int(vertex_capacity), int(steps_per_tick),
                               int(max_requests), int(small_request_seeds), int(reserved_percent),
                               int(max_bypass_ms), int(response_bytes))
        handle = C.c_void_p()
        context.check(self._lib.dpa_server_create(context.handle, C.byref(opts), C.byref(handle)))
        self.handle = handle
        self._index64 = {}

    def add_field(self, field) -> int:
        fid = C.c_int32()
        N.check(self._lib.dpa_server_add_field(self.handle, field.handle, C.byref(fid)),
                self.context.handle)
        return fid.value

    def submit(self, field_id: int, positions, iterations: int, integrator: str = "runge_kutta_4",
               step_size: float = 0.25, record: bool = False, index64: bool = False,
               ftle: bool = False, seed_stride=(1.0, 1.0, 1.0), start_time: float = 0.0,
               deadline_ms: int = 0) -> int:
        pos = np.ascontiguousarray(positions, np.float32).reshape(-1, 3)
        req = N.Request(int(field_id), N.INTEGRATORS[integrator], float(np.float32(step_size)),
                        int(record), int(index64), int(ftle),
                        (C.c_float * 3)(*[float(v) for v in seed_stride]), pos.shape[0],
                        pos.ctypes.data_as(C.POINTER(C.c_float)), int(iterations), None,
                        float(np.float32(start_time)), int(deadline_ms))
        rid = C.c_uint64()
        status = self._lib.dpa_server_submit(self.handle, C.byref(req), C.byref(rid))
        if status != N.DPA_OK:
            raise N.DpaError(status, "request rejected")
        self._index64[rid.value] = bool(index64)
        return rid.value

    def cancel(self, request_id: int) -> bool:
        """Asks the server to drop a request; False when it is unknown or
        already returned."""
        return self._lib.dpa_server_cancel(self.handle, int(request_id)) == N.DPA_OK

    def poll(self, wait_ms: int = 0, copy_ids=None) -> Result | None:
        """Takes one finished request. Its arrays are copied out unless
        copy_ids is given and does not hold its id (then only its status,
        counts and times come back)."""
        r = N.Response()
        got = C.c_int32()
        N.check(self._lib.dpa_server_poll(self.handle, int(wait_ms), C.byref(r), C.byref(got)),
                self.context.handle)
        if not got.value:
            return None
        if copy_ids is not None and int(r.id) not in copy_ids:
            result = Result(int(r.id), int(r.status), None, None, None, None, None, None, None,
                            int(r.particle_steps), r.queued_seconds, r.admitted_seconds,
                            r.finished_seconds, None)
            self._lib.dpa_server_release(self.handle, r.id)
            self._index64.pop(r.id, None)
            return result
        # A request dropped before admission returns no arrays.
        n = int(r.count) if r.positions else 0
        arr = lambda p, shape: np.ctypeslib.as_array(p, shape=shape).copy() if n else np.zeros(shape)
        pos = arr(r.positions, (n * 3,)).reshape(n, 3).astype(np.float32) if n else np.zeros((0, 3), np.float32)
        rem = arr(r.remaining, (n,)).astype(np.uint64) if n else np.zeros(0, np.uint64)
        term = arr(r.termination, (n,)).astype(np.uint8) if n else np.zeros(0, np.uint8)
        vertices = colors = indices = ftle = None
        if r.vertices:
            v = int(r.vertex_count)
            vertices = np.ctypeslib.as_array(r.vertices, shape=(3 * v,)).reshape(v, 3).copy()
            colors = np.ctypeslib.as_array(r.colors, shape=(v,)).copy()
            ni = int(r.index_count)
            ctype = C.c_uint64 if self._index64.get(r.id) else C.c_uint32
            indices = (np.ctypeslib.as_array(C.cast(r.indices, C.POINTER(ctype)), shape=(ni,)).copy()
                       if ni else np.zeros(0, np.uint64 if ctype is C.c_uint64 else np.uint32))
        if r.ftle:
            shape = tuple(int(s) for s in r.ftle_shape)
            ftle = np.ctypeslib.as_array(r.ftle, shape=(int(np.prod(shape)),)).reshape(shape).copy()
        times = arr(r.times, (n,)).astype(np.float32) if (n and r.times) else np.zeros(0, np.float32)
        result = Result(int(r.id), int(r.status), pos, rem, term, vertices, colors, indices, ftle,
                        int(r.particle_steps), r.queued_seconds, r.admitted_seconds,
                        r.finished_seconds, times)
        self._lib.dpa_server_release(self.handle, r.id)
        self._index64.pop(r.id, None)
        return result

    def stats(self) -> dict:
        s = N.ServerStats()
        N.check(self._lib.dpa_server_get_stats(self.handle, C.byref(s)), self.context.handle)
        return {name: getattr(s, name) for name, _ in N.ServerStats._fields_}

    def close(self) -> None:
        if self.handle:
            self._lib.dpa_server_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
