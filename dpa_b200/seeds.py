"""Seed generation: uniform_seed_generator (source/stages/uniform_seed_generator.cpp).

The lattice generator reproduces the reference's float arithmetic exactly.
The reference's random generator draws from a thread_local mt19937 seeded by
std::random_device (uniform_seed_generator.cpp:70-72), so its seeds can never
be reproduced. ``generate_random`` here takes an explicit seed and uses the
counter-based stream of dpa_seed_random_device and of the C++ host pipeline:
seed i, axis a is offset[a] + size[a] * u with
u = (splitmix64(splitmix64(seed) ^ (3 i + a)) >> 40) * 2^-24, so Python, the
host pipeline and the device produce the same seeds.
"""
from __future__ import annotations

import numpy as np

from .advector import Particles


def seed_box(grid) -> tuple[np.ndarray, np.ndarray]:
    """The seed box of pipeline.cpp:59-60 at world size 1: offset =
    spacing * 0, size = spacing * block size (the whole grid shape)."""
    spacing = np.asarray(grid.spacing, dtype=np.float32)
    offset = (spacing * np.zeros(3, dtype=np.float32)).astype(np.float32)
    size = (spacing * np.asarray(grid.shape, dtype=np.float32)).astype(np.float32)
    return offset, size


def _clip(offset, size, aabb):
    if aabb is None:
        return offset, size, False
    lo = np.maximum(np.asarray(aabb[0], np.float32), offset).astype(np.float32)
    hi = np.minimum(np.asarray(aabb[1], np.float32), (offset + size).astype(np.float32)).astype(np.float32)
    if np.any(lo > hi):  # Eigen AlignedBox::isEmpty
        return offset, size, True
    return lo, (hi - lo).astype(np.float32), False


def lattice_shape(offset, size, stride, aabb=None) -> tuple[int, int, int]:
    offset = np.asarray(offset, np.float32)
    size = np.asarray(size, np.float32)
    offset, size, empty = _clip(offset, size, aabb)
    if empty:
        return (0, 0, 0)
    q = (size / np.asarray(stride, np.float32)).astype(np.float32)
    return tuple(int(v) if v > 0 else 0 for v in q)


def generate(offset, size, stride, iterations: int, process_index: int = 0,
             aabb=None) -> Particles:
    """uniform_seed_generator::generate (uniform_seed_generator.cpp:16-45):
    seeds offset + stride * (i, j, k), last axis fastest (indexing.hpp:11-20)."""
    offset = np.asarray(offset, np.float32)
    size = np.asarray(size, np.float32)
    stride = np.asarray(stride, np.float32)
    offset, size, empty = _clip(offset, size, aabb)
    if empty:
        return Particles.create(np.zeros((0, 3), np.float32), iterations)
    shape = [int(v) for v in (size / stride).astype(np.float32)]
    grids = np.meshgrid(*[np.arange(s, dtype=np.float32) for s in shape], indexing="ij")
    sub = np.stack([g.reshape(-1) for g in grids], axis=1).astype(np.float32)
    pos = (offset[None, :] + (stride[None, :] * sub).astype(np.float32)).astype(np.float32)
    return Particles.create(pos, iterations)


def splitmix64(x: np.ndarray) -> np.ndarray:
    """splitmix64 (Steele, Lea and Flood 2014) on uint64 arrays, wrapping."""
    x = np.asarray(x, np.uint64)
    with np.errstate(over="ignore"):
        x = x + np.uint64(0x9E3779B97F4A7C15)
        x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return x ^ (x >> np.uint64(31))


def random_unit(count: int, seed: int) -> np.ndarray:
    """The [0, 1) float32 draws behind generate_random, shape (count, 3)."""
    key = splitmix64(np.array([seed], np.uint64))[0]
    idx = np.arange(3 * int(count), dtype=np.uint64)
    r = splitmix64(key ^ idx)
    return ((r >> np.uint64(40)).astype(np.float32) * np.float32(2.0 ** -24)).reshape(-1, 3)


def random_count(lo: int, hi: int, seed: int) -> int:
    """Seed count drawn for seed_generation_range [lo, hi]."""
    lo, hi = min(lo, hi), max(lo, hi)
    r = int(splitmix64(splitmix64(np.array([seed], np.uint64)) ^ np.uint64(0x72616E6765))[0])
    return lo + r % (hi - lo + 1)


def generate_random(offset, size, count: int, iterations: int, process_index: int = 0,
                    aabb=None, seed: int = 0) -> Particles:
    """uniform_seed_generator::generate_random (uniform_seed_generator.cpp:46-81)
    with an explicit seed: per axis offset + size * u, u in [0, 1)."""
    offset = np.asarray(offset, np.float32)
    size = np.asarray(size, np.float32)
    offset, size, empty = _clip(offset, size, aabb)
    if empty:
        return Particles.create(np.zeros((0, 3), np.float32), iterations)
    u = random_unit(count, seed)
    pos = (offset[None, :] + (size[None, :] * u).astype(np.float32)).astype(np.float32)
    return Particles.create(pos, iterations)
