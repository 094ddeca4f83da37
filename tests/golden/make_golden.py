"""Golden vectors of the advection path: small seeded cases and their
expected outputs, written to tests/golden/*.npz.

    python tests/golden/make_golden.py

The reference cannot be built or run here (its Boost / Eigen / TBB / HDF5 /
MPI dependencies are absent), and it ships no golden vectors of its own. Two
restatements of its algorithm written independently of each other must
therefore agree before a fixture is written: the C++ oracle
(oracle/oracle.cpp) and the numpy float32 restatement below, which follows the
reference's source text function by function (file:line per function). Every
output is checked bit for bit between the two, except colors (atan2f of two
math libraries, 2e-6 rad) and FTLE (the oracle solves the eigenvalue problem
by Jacobi in double, numpy by LAPACK in double; 1e-5 relative). The fixtures
then pin the CUDA path and any later change of the oracle.
"""
from __future__ import annotations

import math
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

f32 = np.float32
TERMINAL = f32(-2.0)  # basic_types.hpp:51-60
INVALID = f32(-1.0)
ZERO_PRECISION = f32(1e-5)  # Eigen NumTraits<float>::dummy_precision()


# ---- numpy restatement -------------------------------------------------------

def contains(data, offset, spacing, p) -> bool:
    """regular_grid::contains, regular_grid.hpp:41-50."""
    for i in range(3):
        q = (p[i] - offset[i]) / spacing[i]
        if not (q == q):  # NaN: the int64 cast yields INT64_MIN on x86-64
            return False
        s = math.floor(float(q))
        if s < 0 or s >= data.shape[i] - 1:
            return False
    return True


def interpolate(data, offset, spacing, p):
    """regular_grid::interpolate, regular_grid.hpp:52-75, corners in the
    permute_for order of permute_for.hpp:12-34 (axis 0 outermost)."""
    w = [f32(0)] * 3
    s = [0] * 3
    for i in range(3):
        a = f32(p[i] - offset[i])
        w[i] = f32(np.fmod(a, spacing[i]) / spacing[i])
        s[i] = int(math.floor(float(a / spacing[i])))
    corners = []
    for dx in (0, 1):
        for dy in (0, 1):
            for dz in (0, 1):
                corners.append(data[s[0] + dx, s[1] + dy, s[2] + dz].astype(np.float32))
    for i in (2, 1, 0):
        one_minus = f32(1) - w[i]
        corners = [(one_minus * corners[2 * j]).astype(np.float32) +
                   (w[i] * corners[2 * j + 1]).astype(np.float32)
                   for j in range(len(corners) // 2)]
        corners = [c.astype(np.float32) for c in corners]
    return corners[0]


def rk4_coefficients(dt):
    """odeint runge_kutta4's b = {1/6, 1/3, 1/3, 1/6} formed in float, times dt."""
    return f32(f32(1) / f32(6)) * dt, f32(f32(1) / f32(3)) * dt


def advect_particle(data, offset, spacing, integrator, dt, p, remaining):
    """The per-particle loop of particle_advector::advect,
    particle_advector.cpp:325-396, for euler and runge_kutta_4 (the system
    functor returns the iteration's sample, :369, so every RK4 stage sees the
    same derivative). Returns position, remaining, reason, curve."""
    p = np.array(p, np.float32)
    dt = f32(dt)
    c0, c1 = rk4_coefficients(dt)
    curve = [p.copy()]
    reason = 0
    while remaining > 0:
        if not contains(data, offset, spacing, p):
            reason = 1
            break
        v = interpolate(data, offset, spacing, p)
        if np.all(np.abs(v) <= ZERO_PRECISION):
            reason = 2
            break
        d = np.array([v[2], v[1], v[0]], np.float32)
        if integrator == "euler":
            p = (f32(1) * p + dt * d).astype(np.float32)
        else:
            x = f32(1) * p
            for c in (c0, c1, c1, c0):
                x = (x + (c * d).astype(np.float32)).astype(np.float32)
            p = x
        curve.append(p.copy())
        remaining -= 1
    curve.append(np.full(3, TERMINAL, np.float32))
    return p, remaining, reason, curve


def indices_of(vertices, index64):
    """index_generator::generate, index_generator.cpp:10-39."""
    dtype = np.uint64 if index64 else np.uint32
    out = []
    for i in range(len(vertices) - 1):
        if not np.all(vertices[i] == TERMINAL) and not np.all(vertices[i + 1] == TERMINAL):
            out += [i, i + 1]
    return np.array(out, dtype)


def colors_of(vertices):
    """color_generator::generate_from_angular_velocities,
    color_generator.cpp:37-58: Eigen normalized() (unchanged when the squared
    norm is 0), cross, dot and norm with fixed-size reductions c0 + (c1 + c2)."""
    def sq(a, b):
        return f32(a[0] * b[0]) + f32(f32(a[1] * b[1]) + f32(a[2] * b[2]))

    def normalized(v):
        z = sq(v, v)
        return (v / np.sqrt(z)).astype(np.float32) if z > 0 else v

    out = np.zeros(len(vertices), np.float32)
    for i, v in enumerate(vertices):
        if np.all(v == TERMINAL):
            continue
        prev = np.zeros(3, np.float32)
        nxt = np.zeros(3, np.float32)
        if i > 1 and not np.all(vertices[i - 1] == TERMINAL):
            prev = normalized((v - vertices[i - 1]).astype(np.float32))
        if i + 1 < len(vertices) and not np.all(vertices[i + 1] == TERMINAL):
            nxt = normalized((vertices[i + 1] - v).astype(np.float32))
        cross = np.array([f32(prev[1] * nxt[2]) - f32(prev[2] * nxt[1]),
                          f32(prev[2] * nxt[0]) - f32(prev[0] * nxt[2]),
                          f32(prev[0] * nxt[1]) - f32(prev[1] * nxt[0])], np.float32)
        out[i] = np.arctan2(np.sqrt(sq(cross, cross)), sq(prev, nxt)).astype(np.float32)
    return out


def advect_round(data, offset, spacing, integrator, dt, positions, remaining, record):
    """One round: allocate / advect / prune (particle_advector.cpp:311-316,
    402-408) and the index and color post-passes on its curve."""
    pos = np.zeros_like(positions)
    rem = np.zeros(len(positions), np.uint64)
    term = np.zeros(len(positions), np.uint8)
    curves = []
    for k in range(len(positions)):
        p, r, reason, curve = advect_particle(data, offset, spacing, integrator, dt,
                                              positions[k], int(remaining[k]))
        pos[k], rem[k], term[k] = p, r, reason
        curves.append(curve)
    out = {"positions": pos, "remaining": rem, "termination": term}
    if record:
        verts = [v for c in curves for v in c if not np.all(v == INVALID)]
        verts = np.array(verts, np.float32).reshape(-1, 3)
        out["vertices"] = verts
        out["indices"] = indices_of(verts, False)
        out["colors"] = colors_of(verts)
    return out


def ftle(shape, offset, spacing, stride, iterations, dt, original, final):
    """ftle_estimator::estimate, ftle_estimator.cpp:7-65, with
    regular_grid::cell (:28-40) and gradient (:87-108)."""
    dims = [int(f32(shape[i]) / f32(stride[i])) for i in range(3)]
    h = (spacing * stride).astype(np.float32)
    flow = np.zeros(dims + [3], np.float32)
    for o, p in zip(original, final):
        idx = [int(math.floor(float(f32(o[i] - offset[i]) / h[i]))) for i in range(3)]
        if all(0 <= idx[i] < dims[i] for i in range(3)):
            flow[tuple(idx)] = p
    two_h = (f32(2) * h).astype(np.float32)
    out = np.zeros(dims, np.float32)
    for i in range(dims[0]):
        for j in range(dims[1]):
            for k in range(dims[2]):
                J = np.zeros((3, 3), np.float32)
                for d in range(3):
                    nxt = [i, j, k]
                    prv = [i, j, k]
                    if prv[d] > 0:
                        prv[d] -= 1
                    if nxt[d] < dims[d] - 1:
                        nxt[d] += 1
                    J[:, d] = (flow[tuple(nxt)] - flow[tuple(prv)]) / two_h[d]
                C = J.T.astype(np.float64) @ J.astype(np.float64)
                lam = np.linalg.eigvalsh(C).max()
                out[i, j, k] = np.log(np.sqrt(lam)) / abs(float(f32(dt) * f32(iterations)))
    return out


# ---- cases -------------------------------------------------------------------

def cases():
    from dpa_b200 import fields, seeds
    box = ([0.0, 0.0, 0.0], [2 * math.pi] * 3)
    out = []
    g = fields.abc(16)
    off, size = seeds.seed_box(g)
    out.append(("abc16_rk4_recording", g, "runge_kutta_4", 0.05, 60, True,
                seeds.generate_random(off, size, 48, 0, aabb=box, seed=0).position))
    out.append(("abc16_default_seed_box_recording", g, "runge_kutta_4", 0.08, 30, True,
                seeds.generate_random(off, size, 48, 0, seed=7).position))
    g = fields.curl_noise(16, 2.0, 3)
    off, size = seeds.seed_box(g)
    out.append(("curl16_euler_unit_spacing", g, "euler", 0.3, 80, False,
                seeds.generate_random(off, size, 64, 0, aabb=([0.0] * 3, [15.0] * 3),
                                      seed=4).position))
    from dpa_b200.advector import RegularGrid
    g7 = RegularGrid.from_data(fields.curl_noise(16, 2.0, 5).data, (0.7, 0.7, 0.7),
                               (-1.5, 0.25, 2.0))
    off, size = seeds.seed_box(g7)
    out.append(("curl16_rk4_spacing_0.7_offset", g7, "runge_kutta_4", 0.2, 50, True,
                seeds.generate_random(off, size, 40, 0, seed=6).position))
    # A contracting linear field (its stored components reversed, so the
    # derivative is -0.5 (x - m)): particles creep towards m until the sample
    # is zero within Eigen's isZero precision.
    m = np.array([7.3, 7.6, 7.1])
    grad = np.zeros((3, 3))
    grad[2, 0] = grad[1, 1] = grad[0, 2] = -0.5
    gl = fields.linear(16, grad, 0.5 * m[::-1])
    off, size = seeds.seed_box(gl)
    out.append(("linear16_contracting_euler_zero_velocity", gl, "euler", 0.5, 100, True,
                seeds.generate_random(off, size, 24, 0, aabb=([2.0] * 3, [13.0] * 3),
                                      seed=8).position))
    return out


def ftle_case():
    from dpa_b200 import fields, seeds
    g = fields.abc_perturbed(16, 0.05, 1.5, 2)
    off, size = seeds.seed_box(g)
    lat = seeds.generate(off, size, (g.spacing * f32(2)).astype(np.float32), 0).position
    return g, lat, 20, 0.05


def main():
    from oracle import binding as ob
    ob.build()
    ob.set_threads(1)
    written = []
    for name, g, integrator, dt, iterations, record, pos in cases():
        rem = np.full(len(pos), iterations, np.uint64)
        want = advect_round(g.data, g.offset, g.spacing, integrator, f32(dt), pos, rem, record)
        got = ob.advect_round(ob.OracleGrid.of(g), integrator, dt, pos, rem, record=record)
        np.testing.assert_array_equal(got.positions, want["positions"])
        np.testing.assert_array_equal(got.remaining, want["remaining"])
        np.testing.assert_array_equal(got.termination, want["termination"])
        arrays = dict(field=g.data, offset=g.offset, spacing=g.spacing, seeds=pos,
                      iterations=np.uint64(iterations), step=f32(dt),
                      integrator=np.array(integrator), record=np.array(record),
                      positions=got.positions, remaining=got.remaining,
                      termination=got.termination)
        if record:
            np.testing.assert_array_equal(got.vertices, want["vertices"])
            np.testing.assert_array_equal(got.indices, want["indices"])
            np.testing.assert_allclose(got.colors, want["colors"], rtol=0, atol=2e-6)
            arrays.update(vertices=got.vertices, indices=got.indices, colors=got.colors)
        np.savez_compressed(HERE / f"{name}.npz", **arrays)
        written.append(name)
    g, lat, iterations, dt = ftle_case()
    rem = np.full(len(lat), iterations, np.uint64)
    adv = ob.advect_round(ob.OracleGrid.of(g), "runge_kutta_4", dt, lat, rem)
    mine = advect_round(g.data, g.offset, g.spacing, "runge_kutta_4", f32(dt), lat, rem, False)
    np.testing.assert_array_equal(adv.positions, mine["positions"])
    got, _ = ob.ftle(g.shape, g.offset, g.spacing, (2, 2, 2), iterations, dt, lat, adv.positions)
    want = ftle(g.shape, g.offset, g.spacing, np.array([2, 2, 2], np.float32), iterations, dt,
                lat, adv.positions)
    finite = np.isfinite(want)
    np.testing.assert_array_equal(np.isfinite(got), finite)
    np.testing.assert_allclose(got[finite], want[finite], rtol=1e-5, atol=1e-7)
    np.savez_compressed(HERE / "abc16_perturbed_ftle_lattice8.npz", field=g.data, offset=g.offset,
                        spacing=g.spacing, seeds=lat, iterations=np.uint64(iterations),
                        step=f32(dt), stride=np.array([2, 2, 2], np.float32),
                        positions=adv.positions, remaining=adv.remaining,
                        termination=adv.termination, ftle=got)
    written.append("abc16_perturbed_ftle_lattice8")
    print("wrote", ", ".join(written))


if __name__ == "__main__":
    main()
