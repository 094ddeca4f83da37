"""ctypes binding of the host library (dpa_b200/host/dpa_host.h): the pipeline
driver, its HDF5 reader/writer and its seed generators."""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

PACKAGE = Path(__file__).resolve().parent
HOST_LIBRARY = PACKAGE / "libdpa_host.so"
PIPELINE = PACKAGE / "bin" / "dpa_pipeline"

_lib = None


def load() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not HOST_LIBRARY.exists():
        raise ImportError(f"{HOST_LIBRARY} is missing: build it with `python -m dpa_b200.build`")
    L = C.CDLL(str(HOST_LIBRARY))
    P = C.c_void_p
    L.dpa_host_last_error.restype = C.c_char_p
    L.dpa_host_run_pipeline.argtypes = [C.c_char_p]
    L.dpa_host_h5_write_field.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p, P, P, P]
    L.dpa_host_h5_write_datasets.argtypes = [C.c_char_p, C.c_uint64, P, P, P, P]
    L.dpa_host_h5_names.argtypes = [C.c_char_p, C.c_char_p, C.c_uint64]
    L.dpa_host_h5_info.argtypes = [C.c_char_p, C.c_char_p, P, P, P, P]
    L.dpa_host_h5_read.argtypes = [C.c_char_p, C.c_char_p, C.c_int32, P, C.c_uint64]
    L.dpa_host_h5_attribute.argtypes = [C.c_char_p, C.c_char_p, P, C.c_uint64, P]
    L.dpa_host_lattice_seeds.argtypes = [P, P, P, P, P, C.c_uint64]
    L.dpa_host_lattice_seeds.restype = C.c_uint64
    L.dpa_host_random_seeds.argtypes = [P, P, C.c_uint64, C.c_uint64, P, P]
    L.dpa_host_random_seeds.restype = C.c_uint64
    L.dpa_host_random_count.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64]
    L.dpa_host_random_count.restype = C.c_uint64
    _lib = L
    return L


def _check(rc: int) -> None:
    if rc != 0:
        raise RuntimeError(load().dpa_host_last_error().decode())


def _p(a: np.ndarray) -> C.c_void_p:
    return a.ctypes.data_as(C.c_void_p)


def write_field(path, grid, dataset: str = "data", spacing_attribute: str = "spacing") -> None:
    """Writes an XYZV field file of the layout the reference's loader reads."""
    data = np.ascontiguousarray(grid.data, np.float32)
    shape = np.asarray(data.shape[:3], np.uint64)
    spacing = np.asarray(grid.spacing, np.float32)
    _check(load().dpa_host_h5_write_field(str(path).encode(), dataset.encode(),
                                          spacing_attribute.encode(), _p(data), _p(shape),
                                          _p(spacing)))


_KINDS = {np.dtype(np.float32): 0, np.dtype(np.uint8): 1, np.dtype(np.uint32): 2,
          np.dtype(np.uint64): 3}


def write_datasets(path, datasets: dict) -> None:
    """Writes one-dimensional arrays (float32, uint8, uint32, uint64) as
    datasets of the root group of a new file."""
    items = [(k, np.ascontiguousarray(v).ravel()) for k, v in datasets.items()]
    n = len(items)
    names_c = (C.c_char_p * n)(*[k.encode() for k, _ in items])
    kinds = np.array([_KINDS[a.dtype] for _, a in items], np.int32)
    lengths = np.array([a.size for _, a in items], np.uint64)
    ptrs = (C.c_void_p * n)(*[a.ctypes.data for _, a in items])
    _check(load().dpa_host_h5_write_datasets(str(path).encode(), n, names_c, _p(kinds),
                                             _p(lengths), ptrs))


def names(path) -> list[str]:
    buf = C.create_string_buffer(1 << 20)
    _check(load().dpa_host_h5_names(str(path).encode(), buf, len(buf)))
    return [n for n in buf.value.decode().split("\n") if n]


def info(path, dataset: str) -> tuple[tuple[int, ...], int, int]:
    dims = np.zeros(8, np.uint64)
    rank, cls, size = C.c_int32(), C.c_int32(), C.c_int32()
    _check(load().dpa_host_h5_info(str(path).encode(), dataset.encode(), _p(dims), C.byref(rank),
                                   C.byref(cls), C.byref(size)))
    return tuple(int(d) for d in dims[: rank.value]), cls.value, size.value


def read(path, dataset: str) -> np.ndarray:
    """A dataset as float32/float64 (floats) or uint64 (integers)."""
    dims, cls, size = info(path, dataset)
    n = int(np.prod(dims)) if dims else 1
    if cls == 1:
        kind, dtype = (1, np.float32) if size == 4 else (0, np.float64)
    else:
        kind, dtype = 2, np.uint64
    out = np.zeros(n, dtype)
    _check(load().dpa_host_h5_read(str(path).encode(), dataset.encode(), kind, _p(out), n))
    return out.reshape(dims)


def attribute(path, name: str) -> np.ndarray:
    out = np.zeros(64, np.float64)
    count = C.c_uint64()
    _check(load().dpa_host_h5_attribute(str(path).encode(), name.encode(), _p(out), 64,
                                        C.byref(count)))
    return out[: count.value].copy()


def lattice_seeds(offset, size, stride, aabb=None) -> np.ndarray:
    o, s, t = (np.asarray(v, np.float32) for v in (offset, size, stride))
    box = None if aabb is None else np.concatenate([np.asarray(aabb[0], np.float32),
                                                    np.asarray(aabb[1], np.float32)])
    L = load()
    n = L.dpa_host_lattice_seeds(_p(o), _p(s), _p(t), None if box is None else _p(box), None, 0)
    out = np.zeros((n, 3), np.float32)
    L.dpa_host_lattice_seeds(_p(o), _p(s), _p(t), None if box is None else _p(box), _p(out), n)
    return out


def random_seeds(offset, size, count: int, seed: int, aabb=None) -> np.ndarray:
    o, s = (np.asarray(v, np.float32) for v in (offset, size))
    box = None if aabb is None else np.concatenate([np.asarray(aabb[0], np.float32),
                                                    np.asarray(aabb[1], np.float32)])
    out = np.zeros((int(count), 3), np.float32)
    n = load().dpa_host_random_seeds(_p(o), _p(s), int(count), int(seed),
                                     None if box is None else _p(box), _p(out))
    return out[:n]


def random_count(lo: int, hi: int, seed: int) -> int:
    return int(load().dpa_host_random_count(int(lo), int(hi), int(seed)))


def run_pipeline(config_path, timeout: float | None = None) -> subprocess.CompletedProcess:
    """Runs `dpa_pipeline config.json` as a child process."""
    if not PIPELINE.exists():
        raise ImportError(f"{PIPELINE} is missing: build it with `python -m dpa_b200.build`")
    return subprocess.run([str(PIPELINE), str(config_path)], capture_output=True, text=True,
                          timeout=timeout)
