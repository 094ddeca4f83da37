"""The reference's other odeint steppers in the oracle (integrators.hpp:13-28),
checked against an independent numpy float32 restatement step by step.

The reference's system functor ignores its state argument and returns the
iteration's field sample (particle_advector.cpp:376), so every stage of one
do_step sees the same derivative; each stepper reduces to its final
expression. The steppers with memory are pinned separately:
runge_kutta_dopri5 reuses the derivative the previous step ended with
(first-same-as-last), adams_bashforth<2> keeps the previous derivative and
both Adams methods start with their initialising extrapolation stepper."""
import numpy as np
import pytest

from dpa_b200 import fields

f32 = np.float32


def q(a, b):
    return f32(a) / f32(b)


def modified_midpoint(x, d, dt, steps):
    h = f32(dt) / f32(steps)
    h2 = f32(2) * h
    x1 = f32(1) * x + h * d
    x0 = x
    for _ in range(steps - 1):
        x1, x0 = f32(1) * x0 + h2 * d, x1
    return f32(0.5) * x0 + f32(0.5) * x1 + (f32(0.5) * h) * d


def extrapolation4(x, d, dt):
    r = f32(4) / f32(2)
    c = f32(1) / (r * r - f32(1))
    return (f32(1) + c) * modified_midpoint(x, d, dt, 4) + (-c) * modified_midpoint(x, d, dt, 2)


def weighted(x, d, dt, b, dt_first=False):
    out = f32(1) * x
    for bi in b:
        out = out + ((f32(dt) * bi) if dt_first else (bi * f32(dt))) * d
    return out


def numpy_step(name, x, d, dt, state):
    """One do_step of the named stepper; `state` is the per-particle copy of
    the integrator (particle_advector.cpp:335)."""
    dt = f32(dt)
    first = not state.get("started")
    if name == "euler":
        out = f32(1) * x + dt * d
    elif name == "modified_midpoint":
        out = modified_midpoint(x, d, dt, 2)
    elif name == "runge_kutta_4":
        out = weighted(x, d, dt, [q(1, 6), q(1, 3), q(1, 3), q(1, 6)])
    elif name == "runge_kutta_cash_karp_54":
        out = weighted(x, d, dt, [q(37, 378), f32(0), q(250, 621), q(125, 594), f32(0),
                                  q(512, 1771)])
    elif name == "runge_kutta_fehlberg_78":
        b = [f32(0)] * 5 + [q(34, 105), q(9, 35), q(9, 35), q(9, 280), q(9, 280), f32(0),
                            q(41, 840), q(41, 840)]
        out = weighted(x, d, dt, b)
    elif name == "runge_kutta_dormand_prince_5":
        fsal = d if first else state["fsal"]
        c = [q(35, 384), q(500, 1113), q(125, 192), q(-2187, 6784), q(11, 84)]
        out = f32(1) * x + (dt * c[0]) * fsal
        for ci in c[1:]:
            out = out + (dt * ci) * d
        state["fsal"] = d
    elif name == "adams_bashforth_2":
        if first:
            out = extrapolation4(x, d, dt)
        else:
            out = f32(1) * x + (dt * q(3, 2)) * d + (dt * -q(1, 2)) * state["prev"]
        state["prev"] = d
    elif name == "adams_bashforth_moulton_2":
        if first:
            out = extrapolation4(x, d, dt)
        else:
            out = f32(1) * x + (dt * q(1, 2)) * d + (dt * q(1, 2)) * d
    else:
        raise KeyError(name)
    state["started"] = True
    return out.astype(np.float32)


NAMES = ["euler", "modified_midpoint", "runge_kutta_4", "runge_kutta_cash_karp_54",
         "runge_kutta_dormand_prince_5", "runge_kutta_fehlberg_78", "adams_bashforth_2",
         "adams_bashforth_moulton_2"]


@pytest.fixture(scope="module")
def swirl(oracle):
    # A linear field (trilinear sampling is exact up to rounding) whose
    # derivative changes from step to step, so the steppers with memory
    # differ visibly from the memoryless ones.
    grad = np.array([[0.0, -0.6, 0.1], [0.6, 0.0, -0.2], [-0.1, 0.2, 0.05]])
    grid = fields.linear(17, grad, np.array([0.3, -0.2, 0.4]), spacing=(0.5, 0.5, 0.5))
    return grid, oracle.OracleGrid.of(grid)


@pytest.mark.parametrize("name", NAMES)
def test_oracle_steps_match_the_numpy_restatement(oracle, swirl, name):
    grid, g = swirl
    rng = np.random.default_rng(9)
    starts = (f32(3.0) + rng.random((40, 3)) * f32(2.0)).astype(np.float32)
    dt, steps = 0.02, 25
    got = oracle.advect_round(g, name, dt, starts, np.full(len(starts), steps, np.uint64))
    assert np.all(got.termination == 0) and np.all(got.remaining == 0)
    for i, x0 in enumerate(starts):
        x, state = x0.copy(), {}
        for _ in range(steps):
            v = oracle.interpolate(g, x)
            d = np.array([v[2], v[1], v[0]], np.float32)  # particle_advector.cpp:376
            x = numpy_step(name, x, d, dt, state)
        np.testing.assert_array_equal(got.positions[i], x)


def test_steppers_agree_in_exact_arithmetic_and_memory_shows(oracle, swirl):
    # Every stepper's weights sum to 1, so the memoryless ones stay within a
    # few ulps of Euler; dopri5 and adams_bashforth_2 weight the previous
    # step's derivative and move measurably away.
    grid, g = swirl
    starts = np.array([[4.0, 4.0, 4.0], [3.0, 5.0, 2.5]], np.float32)
    rem = np.full(2, 40, np.uint64)
    euler = oracle.advect_round(g, "euler", 0.02, starts, rem).positions
    for name in NAMES:
        out = oracle.advect_round(g, name, 0.02, starts, rem)
        assert np.all(out.termination == 0)
        pos = out.positions
        err = np.abs(pos - euler).max()
        if name in ("runge_kutta_dormand_prince_5", "adams_bashforth_2"):
            assert err > 1e-4, name
        else:
            assert err < 1e-4, name


def test_fp64_oracle_refuses_the_general_steppers(oracle, swirl):
    grid, g = swirl
    with pytest.raises(AssertionError):
        oracle.advect64(g, "modified_midpoint", 0.05, np.zeros((1, 3)), np.ones(1, np.uint64))
