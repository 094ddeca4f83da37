// oracle.cpp -- CPU restatement of the dpa advection path.
//
// TEST INFRASTRUCTURE ONLY: the checker for the CUDA path and the timed CPU
// baseline. Nothing in the product library links or calls this file.
//
// PARITY UNPINNED: the reference (VRGroupRWTH/dpa) has no tests or golden
// vectors and cannot be built here (Boost, Eigen, TBB, HDF5, MPI absent).
// Every function below cites the reference file:line it restates. Where the
// arithmetic lives in a third-party header that the reference does not vendor,
// the restated algorithm is named:
//   * Boost.Odeint (vcpkg "boost-odeint", version not pinned): euler and the
//     generic explicit Runge-Kutta stepper `runge_kutta4` with
//     vector_space_algebra. The final stage is one scale_sum5 expression
//     x_out = 1*x + (b0*dt)*k1 + (b1*dt)*k2 + (b2*dt)*k3 + (b3*dt)*k4,
//     evaluated left to right per component, with b = {1/6, 1/3, 1/3, 1/6}
//     computed in float. The other steppers of integrators.hpp:13-28 follow
//     odeint's published algorithms as of Boost 1.6x-1.8x (odeint_step
//     below): modified_midpoint with its default 2 sub-steps, the
//     runge_kutta_cash_karp54 / runge_kutta_fehlberg78 high-order weights,
//     runge_kutta_dopri5 with its first-same-as-last derivative, and
//     adams_bashforth<2> / adams_bashforth_moulton<2>, whose first step is
//     their default initialising stepper, extrapolation_stepper<4>.
//   * Eigen >= 3.3 (version not pinned): isZero() with the float dummy
//     precision 1e-5; fixed-size 3-element reductions (squaredNorm, dot,
//     lazy 3x3 product coefficients) unrolled as c0 + (c1 + c2);
//     normalized() returns the input unchanged when its squared norm is 0;
//     cross() as (a1 b2 - a2 b1, a2 b0 - a0 b2, a0 b1 - a1 b0).
//   * Eigen SelfAdjointEigenSolver<Matrix3f>: restated as a cyclic Jacobi
//     solve in double of the float matrix C = J^T J (the reference solves in
//     float; both return the largest eigenvalue of the same C to well below
//     the 1e-3 relative FTLE tolerance).
//
// The reference is compiled for baseline x86-64 (SSE, no FMA). This file is
// built with -ffp-contract=off so every float operation rounds on its own,
// exactly as there.
//
// The reference's per-call structure (heap-allocated corner list, recursive
// std::function corner traversal, a TBB parallel_for with grain 1 over the
// round's particles) is kept on purpose: this file is also the CPU baseline
// whose speed is reported, so it must cost what the reference costs.

#include "oracle.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <limits>
#include <vector>

#include <omp.h>

namespace {

using index3 = std::array<std::uint64_t, 3>;

// include/dpa/types/basic_types.hpp:51-60: invalid_value = -1 * Ones,
// terminal_value = -2 * Ones.
constexpr float kInvalid  = -1.0f;
constexpr float kTerminal = -2.0f;

// Eigen::NumTraits<float>::dummy_precision(), the default of isZero()
// (particle_advector.cpp:363).
constexpr float kZeroPrecision = 1e-5f;

int g_threads = 0;

inline bool equals_sentinel(const float* v, float s) {
  return v[0] == s && v[1] == s && v[2] == s;
}

// ---------------------------------------------------------------------------
// regular_grid<vector3, 3>
// ---------------------------------------------------------------------------

// regular_grid.hpp:41-50. Valid iff 0 <= floor((p - o) / h) < n - 1 on
// every axis (so an axis of one node holds no valid position). The reference
// converts the float subscript to int64 for the lower test and to size_t for
// the upper one, compared with shape - 1; on x86-64 both conversions reject
// NaN and out-of-range values, which the float comparisons below reproduce
// without the undefined conversions.
bool grid_contains(const oracle_grid& g, const float* p) {
  for (int i = 0; i < 3; ++i) {
    const float subscript = std::floor((p[i] - g.offset[i]) / g.spacing[i]);
    if (!(subscript >= 0.0f)) return false;
    if (!(subscript < static_cast<float>(g.shape[i] - 1))) return false;
  }
  return true;
}

inline const float* node(const oracle_grid& g, const index3& i) {
  return g.data + ((i[0] * g.shape[1] + i[1]) * g.shape[2] + i[2]) * 3;
}

// Corner traversal of permute_for.hpp:12-34: a recursive visit with axis 0
// outermost, each axis running from start to start + 2.
void visit_corners(const std::function<void(const index3&)>& leaf, const index3& start) {
  std::function<void(index3, int)> walk = [&](index3 at, int depth) {
    if (depth < 3) {
      for (std::uint64_t i = start[depth]; i < start[depth] + 2; ++i) {
        at[depth] = i;
        walk(at, depth + 1);
      }
    } else {
      leaf(at);
    }
  };
  walk(index3{}, 0);
}

// regular_grid.hpp:52-75. Weights from fmod, start cell from floor of the
// rounded quotient, corners gathered in traversal order, then reduced axis 2,
// then 1, then 0 with c[j] = (1 - w) * c[2j] + w * c[2j+1].
void grid_interpolate(const oracle_grid& g, const float* p, float* out) {
  float weights[3];
  index3 start;
  for (int i = 0; i < 3; ++i) {
    weights[i] = std::fmod(p[i] - g.offset[i], g.spacing[i]) / g.spacing[i];
    start[i]   = static_cast<std::uint64_t>(std::floor((p[i] - g.offset[i]) / g.spacing[i]));
  }
  std::vector<std::array<float, 3>> corners;
  corners.reserve(8);
  visit_corners([&](const index3& at) {
    const float* v = node(g, at);
    corners.push_back({v[0], v[1], v[2]});
  }, start);
  for (int axis = 2; axis >= 0; --axis) {
    const float w = weights[axis];
    for (int j = 0; j < (1 << axis); ++j)
      for (int c = 0; c < 3; ++c)
        corners[j][c] = (1.0f - w) * corners[2 * j][c] + w * corners[2 * j + 1][c];
  }
  out[0] = corners[0][0];
  out[1] = corners[0][1];
  out[2] = corners[0][2];
}

inline bool is_zero(const float* v) {
  return std::fabs(v[0]) <= kZeroPrecision && std::fabs(v[1]) <= kZeroPrecision &&
         std::fabs(v[2]) <= kZeroPrecision;
}

// The system functor of particle_advector.cpp:369 returns the sample with its
// components reversed (the "data-specific" axis swap).
inline void derivative_of(const float* v, float* d) {
  d[0] = v[2];
  d[1] = v[1];
  d[2] = v[0];
}

struct step_coefficients {
  float dt;
  float c0;   // (1/6) * dt
  float c1;   // (1/3) * dt
  float half; // (1/2) * dt
};

step_coefficients make_coefficients(float dt) {
  const float b0 = 1.0f / 6.0f;
  const float b1 = 1.0f / 3.0f;
  const float a  = 1.0f / 2.0f;
  return {dt, b0 * dt, b1 * dt, a * dt};
}

// ---------------------------------------------------------------------------
// The other odeint steppers (integrators.hpp:13-28) as the reference calls
// them: integrator.do_step(system, position, t, dt) once per iteration with a
// system that ignores its state and time arguments and returns this
// iteration's sample d (particle_advector.cpp:376-393). Every stage
// derivative inside one do_step is therefore d, and the stage states odeint
// forms are never read; what remains is each stepper's final expression,
// evaluated per component left to right in float. Tableau entries are
// quotients of floats (odeint's static_cast<value_type>(p) / q).
// ---------------------------------------------------------------------------
inline float fq(float p, float q) { return p / q; }

struct odeint_state {
  bool  started = false;  // the per-particle integrator copy has stepped
  float fsal[3] = {0, 0, 0};   // dopri5: derivative left by the last step
  float history[3] = {0, 0, 0};  // adams_bashforth: d of the previous step
};

// modified_midpoint::do_step_impl with `steps` sub-steps and constant d:
// h = dt / steps, h2 = 2 h; x1 = 1*x + h*d; x0 = x; (steps - 1) times
// scale_sum_swap2: (x1, x0) = (1*x0 + h2*d, x1); out = 0.5*x0 + 0.5*x1 + (0.5*h)*d.
float odeint_modified_midpoint(float x, float d, float dt, unsigned steps) {
  const float h = dt / static_cast<float>(steps);
  const float h2 = 2.0f * h;
  float x1 = 1.0f * x + h * d;
  float x0 = x;
  for (unsigned i = 1; i != steps; ++i) {
    const float tmp = x1;
    x1 = 1.0f * x0 + h2 * d;
    x0 = tmp;
  }
  return 0.5f * x0 + 0.5f * x1 + (0.5f * h) * d;
}

// extrapolation_stepper<4>::do_step_impl: interval sequence {2, 4}; out =
// midpoint(2); table[0] = midpoint(4); extrapolate(k = 1):
// out = (1 + c) * table[0] + (-c) * out with c = 1 / ((4/2)^2 - 1).
float odeint_extrapolation4(float x, float d, float dt) {
  const float r = static_cast<float>(4) / static_cast<float>(2);
  const float c = static_cast<float>(1) / (r * r - static_cast<float>(1));
  const float m2 = odeint_modified_midpoint(x, d, dt, 2);
  const float m4 = odeint_modified_midpoint(x, d, dt, 4);
  return (static_cast<float>(1) + c) * m4 + (-c) * m2;
}

void odeint_step(int integrator, float dt, const float* d, odeint_state& st, float* x) {
  switch (integrator) {
    case ORACLE_MODIFIED_MIDPOINT:
      for (int c = 0; c < 3; ++c) x[c] = odeint_modified_midpoint(x[c], d[c], dt, 2);
      break;
    case ORACLE_RUNGE_KUTTA_CASH_KARP_54: {
      // explicit_error_generic_rk<6,5,5,4>::do_step without error: final
      // scale_sum7(1, b0*dt, ..., b5*dt) with the 5th-order weights.
      const float b[6] = {fq(37, 378), 0.0f, fq(250, 621), fq(125, 594), 0.0f, fq(512, 1771)};
      for (int c = 0; c < 3; ++c) {
        float v = 1.0f * x[c];
        for (int i = 0; i < 6; ++i) v = v + (b[i] * dt) * d[c];
        x[c] = v;
      }
      break;
    }
    case ORACLE_RUNGE_KUTTA_DORMAND_PRINCE_5: {
      // explicit_error_stepper_fsal_base::do_step: on the first call
      // initialize() evaluates dxdt = system(x); afterwards dxdt is the
      // derivative the previous do_step_impl ended with (system(out), i.e.
      // that step's sample). x_out = 1*x + dt*c1*dxdt + dt*c3*k3 + dt*c4*k4 +
      // dt*c5*k5 + dt*c6*k6, then the new dxdt = system(x_out) = d.
      const float c1 = fq(35, 384), c3 = fq(500, 1113), c4 = fq(125, 192),
                  c5 = fq(-2187, 6784), c6 = fq(11, 84);
      if (!st.started) std::memcpy(st.fsal, d, sizeof st.fsal);
      for (int c = 0; c < 3; ++c)
        x[c] = 1.0f * x[c] + (dt * c1) * st.fsal[c] + (dt * c3) * d[c] + (dt * c4) * d[c] +
               (dt * c5) * d[c] + (dt * c6) * d[c];
      std::memcpy(st.fsal, d, sizeof st.fsal);
      break;
    }
    case ORACLE_RUNGE_KUTTA_FEHLBERG_78: {
      // explicit_error_generic_rk<13,8,8,7>: final scale_sum14 with the
      // 8th-order weights.
      const float b[13] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, fq(34, 105), fq(9, 35), fq(9, 35),
                           fq(9, 280), fq(9, 280), 0.0f, fq(41, 840), fq(41, 840)};
      for (int c = 0; c < 3; ++c) {
        float v = 1.0f * x[c];
        for (int i = 0; i < 13; ++i) v = v + (b[i] * dt) * d[c];
        x[c] = v;
      }
      break;
    }
    case ORACLE_ADAMS_BASHFORTH_2:
    case ORACLE_ADAMS_BASHFORTH_MOULTON_2: {
      if (!st.started) {
        // adams_bashforth::do_step_impl before 1 step is stored: the
        // initialising stepper advances, the step storage keeps d.
        for (int c = 0; c < 3; ++c) x[c] = odeint_extrapolation4(x[c], d[c], dt);
      } else if (integrator == ORACLE_ADAMS_BASHFORTH_2) {
        // rotate, store d; scale_sum3(1, dt*(3/2), dt*(-1/2)) of (x, d_n, d_n-1).
        const float a0 = fq(3, 2), a1 = -fq(1, 2);
        for (int c = 0; c < 3; ++c)
          x[c] = 1.0f * x[c] + (dt * a0) * d[c] + (dt * a1) * st.history[c];
      } else {
        // adams_bashforth_moulton: the AB2 predictor only feeds the system,
        // which ignores it; the AM2 corrector is scale_sum3(1, dt*(1/2),
        // dt*(1/2)) of (x, system(predicted), d_n).
        const float m0 = fq(1, 2), m1 = fq(1, 2);
        for (int c = 0; c < 3; ++c) x[c] = 1.0f * x[c] + (dt * m0) * d[c] + (dt * m1) * d[c];
      }
      std::memcpy(st.history, d, sizeof st.history);
      break;
    }
    default:
      break;
  }
  st.started = true;
}

// ---------------------------------------------------------------------------
// The field a particle loop samples: the reference's steady regular_grid, or
// a time-varying field (pathlines; no counterpart in the reference).
// ---------------------------------------------------------------------------
struct steady_field {
  const oracle_grid& g;
  bool contains(const float* p, float) const { return grid_contains(g, p); }
  void interpolate(const float* p, float, float* out) const { grid_interpolate(g, p, out); }
};

// Slices of one grid at times t0 + s * dt. The time axis follows the spatial
// rule of regular_grid.hpp:41-75: slice floor((t - t0) / dt) must lie in
// [0, slices - 2], weight fmod(t - t0, dt) / dt, and the two slices' samples
// blend as (1 - w) * a + w * b.
struct unsteady_field {
  const oracle_unsteady_grid& u;
  oracle_grid slice(std::uint64_t s) const {
    oracle_grid g;
    g.data = u.data + s * u.shape[0] * u.shape[1] * u.shape[2] * 3;
    for (int i = 0; i < 3; ++i) {
      g.shape[i] = u.shape[i];
      g.offset[i] = u.offset[i];
      g.spacing[i] = u.spacing[i];
    }
    return g;
  }
  bool contains(const float* p, float t) const {
    const float subscript = std::floor((t - u.time_origin) / u.time_spacing);
    if (!(subscript >= 0.0f) || !(subscript < static_cast<float>(u.slices - 1))) return false;
    return grid_contains(slice(0), p);
  }
  void interpolate(const float* p, float t, float* out) const {
    const float w = std::fmod(t - u.time_origin, u.time_spacing) / u.time_spacing;
    const auto s = static_cast<std::uint64_t>(std::floor((t - u.time_origin) / u.time_spacing));
    float a[3], b[3];
    grid_interpolate(slice(s), p, a);
    grid_interpolate(slice(s + 1), p, b);
    for (int c = 0; c < 3; ++c) out[c] = (1.0f - w) * a[c] + w * b[c];
  }
};

// ---------------------------------------------------------------------------
// particle_advector::advect, one particle (particle_advector.cpp:325-396)
// ---------------------------------------------------------------------------
// t (may be null: the time is then not tracked) is the particle's time, which
// advances by dt with every step taken.
template <class Field>
std::uint8_t advect_one(const Field& g, int integrator, const step_coefficients& k,
                        float* pos, std::uint64_t* remaining, std::uint64_t* steps_out,
                        float* curve /* null or curve_stride * 3 floats */,
                        float* time = nullptr) {
  float t = time ? *time : 0.0f;
  std::uint64_t iteration = 0;
  std::uint8_t reason = ORACLE_COMPLETE;
  odeint_state state;  // `auto integrator = integrator_;` per particle (:335)
  if (curve) std::memcpy(curve, pos, 3 * sizeof(float));
  for (; *remaining > 0; ++iteration, --*remaining) {
    if (!g.contains(pos, t)) { reason = ORACLE_OUT_OF_BOUNDS; break; }
    float v[3];
    g.interpolate(pos, t, v);
    if (is_zero(v)) { reason = ORACLE_ZERO_VELOCITY; break; }
    float d[3];
    derivative_of(v, d);
    if (integrator == ORACLE_EULER) {
      // odeint euler: x = 1*x + dt*dxdt
      for (int c = 0; c < 3; ++c) pos[c] = 1.0f * pos[c] + k.dt * d[c];
    } else if (integrator == ORACLE_RUNGE_KUTTA_4) {
      // odeint runge_kutta4 with a state-independent system: every stage
      // derivative equals d, so only the final scale_sum5 remains.
      for (int c = 0; c < 3; ++c)
        pos[c] = 1.0f * pos[c] + k.c0 * d[c] + k.c1 * d[c] + k.c1 * d[c] + k.c0 * d[c];
    } else if (integrator != ORACLE_RUNGE_KUTTA_4_TRUE) {
      odeint_step(integrator, k.dt, d, state, pos);
    } else {
      // Four-sample RK4 (not part of the reference): stages at x,
      // x + dt/2 k1, x + dt/2 k2, x + dt k3; a stage outside the grid ends
      // the particle as out of bounds without taking the step.
      // Stage times t + dt/2, t + dt/2 and t + dt.
      float k2[3], k3[3], k4[3], x[3], w[3];
      const float t_half = t + k.half, t_end = t + k.dt;
      for (int c = 0; c < 3; ++c) x[c] = pos[c] + k.half * d[c];
      if (!g.contains(x, t_half)) { reason = ORACLE_OUT_OF_BOUNDS; break; }
      g.interpolate(x, t_half, w); derivative_of(w, k2);
      for (int c = 0; c < 3; ++c) x[c] = pos[c] + k.half * k2[c];
      if (!g.contains(x, t_half)) { reason = ORACLE_OUT_OF_BOUNDS; break; }
      g.interpolate(x, t_half, w); derivative_of(w, k3);
      for (int c = 0; c < 3; ++c) x[c] = pos[c] + k.dt * k3[c];
      if (!g.contains(x, t_end)) { reason = ORACLE_OUT_OF_BOUNDS; break; }
      g.interpolate(x, t_end, w); derivative_of(w, k4);
      for (int c = 0; c < 3; ++c)
        pos[c] = pos[c] + k.c0 * d[c] + k.c1 * k2[c] + k.c1 * k3[c] + k.c0 * k4[c];
    }
    t = t + k.dt;
    if (curve) std::memcpy(curve + 3 * (iteration + 1), pos, 3 * sizeof(float));
  }
  if (time) *time = t;
  if (curve) {
    float* t = curve + 3 * (iteration + 1);
    t[0] = t[1] = t[2] = kTerminal;
  }
  if (steps_out) *steps_out = iteration;
  return reason;
}

// ---------------------------------------------------------------------------
// Symmetric 3x3 largest eigenvalue, cyclic Jacobi in double.
// ---------------------------------------------------------------------------
double symmetric3_max_eigenvalue(const double in[3][3]) {
  double a[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) a[i][j] = in[i][j];
  for (int sweep = 0; sweep < 32; ++sweep) {
    const double off = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2];
    const double diag = a[0][0] * a[0][0] + a[1][1] * a[1][1] + a[2][2] * a[2][2];
    if (off == 0.0 || off <= 1e-32 * diag) break;
    for (int p = 0; p < 2; ++p) {
      for (int q = p + 1; q < 3; ++q) {
        const double apq = a[p][q];
        if (apq == 0.0) continue;
        const double theta = (a[q][q] - a[p][p]) / (2.0 * apq);
        const double t = (theta >= 0.0 ? 1.0 : -1.0) /
                         (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0);
        const double s = t * c;
        for (int r = 0; r < 3; ++r) {
          const double arp = a[r][p], arq = a[r][q];
          a[r][p] = c * arp - s * arq;
          a[r][q] = s * arp + c * arq;
        }
        for (int r = 0; r < 3; ++r) {
          const double apr = a[p][r], aqr = a[q][r];
          a[p][r] = c * apr - s * aqr;
          a[q][r] = s * apr + c * aqr;
        }
      }
    }
  }
  return std::max(a[0][0], std::max(a[1][1], a[2][2]));
}

// ---------------------------------------------------------------------------
// FP64 oracle: double-precision grid and steps.
// ---------------------------------------------------------------------------
bool grid_contains64(const oracle_grid& g, const double* p) {
  for (int i = 0; i < 3; ++i) {
    const double s = std::floor((p[i] - double(g.offset[i])) / double(g.spacing[i]));
    if (!(s >= 0.0)) return false;
    if (!(s < double(g.shape[i] - 1))) return false;
  }
  return true;
}

void grid_interpolate64(const oracle_grid& g, const double* p, double* out) {
  double w[3];
  index3 s;
  for (int i = 0; i < 3; ++i) {
    const double a = p[i] - double(g.offset[i]);
    const double q = a / double(g.spacing[i]);
    const double f = std::floor(q);
    s[i] = static_cast<std::uint64_t>(f);
    w[i] = q - f;
  }
  double c[8][3];
  for (int dx = 0; dx < 2; ++dx)
    for (int dy = 0; dy < 2; ++dy)
      for (int dz = 0; dz < 2; ++dz) {
        const float* v = node(g, index3{s[0] + dx, s[1] + dy, s[2] + dz});
        for (int k = 0; k < 3; ++k) c[dx * 4 + dy * 2 + dz][k] = v[k];
      }
  for (int axis = 2; axis >= 0; --axis)
    for (int j = 0; j < (1 << axis); ++j)
      for (int k = 0; k < 3; ++k)
        c[j][k] = (1.0 - w[axis]) * c[2 * j][k] + w[axis] * c[2 * j + 1][k];
  out[0] = c[0][2];  // axis swap of particle_advector.cpp:369
  out[1] = c[0][1];
  out[2] = c[0][0];
}

inline bool is_zero64(const double* d) {
  return std::fabs(d[0]) <= kZeroPrecision && std::fabs(d[1]) <= kZeroPrecision &&
         std::fabs(d[2]) <= kZeroPrecision;
}

template <class Contains, class Derivative>
std::uint8_t advect_one64(int integrator, double dt, double* pos, std::uint64_t* remaining,
                          std::uint64_t* steps_out, Contains contains, Derivative derivative) {
  std::uint64_t iteration = 0;
  std::uint8_t reason = ORACLE_COMPLETE;
  for (; *remaining > 0; ++iteration, --*remaining) {
    if (!contains(pos)) { reason = ORACLE_OUT_OF_BOUNDS; break; }
    double k1[3];
    derivative(pos, k1);
    if (is_zero64(k1)) { reason = ORACLE_ZERO_VELOCITY; break; }
    if (integrator == ORACLE_EULER) {
      for (int c = 0; c < 3; ++c) pos[c] += dt * k1[c];
    } else if (integrator == ORACLE_RUNGE_KUTTA_4) {
      for (int c = 0; c < 3; ++c) pos[c] += dt * k1[c];
    } else {
      double x[3], k2[3], k3[3], k4[3];
      for (int c = 0; c < 3; ++c) x[c] = pos[c] + 0.5 * dt * k1[c];
      if (!contains(x)) { reason = ORACLE_OUT_OF_BOUNDS; break; }
      derivative(x, k2);
      for (int c = 0; c < 3; ++c) x[c] = pos[c] + 0.5 * dt * k2[c];
      if (!contains(x)) { reason = ORACLE_OUT_OF_BOUNDS; break; }
      derivative(x, k3);
      for (int c = 0; c < 3; ++c) x[c] = pos[c] + dt * k3[c];
      if (!contains(x)) { reason = ORACLE_OUT_OF_BOUNDS; break; }
      derivative(x, k4);
      for (int c = 0; c < 3; ++c)
        pos[c] += dt / 6.0 * (k1[c] + 2.0 * k2[c] + 2.0 * k3[c] + k4[c]);
    }
  }
  if (steps_out) *steps_out = iteration;
  return reason;
}

}  // namespace

extern "C" {

void oracle_set_threads(int threads) { g_threads = threads; }
int oracle_get_threads(void) { return g_threads > 0 ? g_threads : omp_get_max_threads(); }

int oracle_contains(const oracle_grid* grid, const float position[3]) {
  return grid_contains(*grid, position) ? 1 : 0;
}

void oracle_interpolate(const oracle_grid* grid, const float position[3], float out[3]) {
  grid_interpolate(*grid, position, out);
}

// particle_advector.cpp:311-316 (allocate: fill with the invalid sentinel)
// and :317-401 (advect). The parallel loop stands in for the reference's
// tbb::parallel_for with grain 1.
int oracle_advect_round(const oracle_grid* grid, int integrator, float step_size,
                        uint64_t count, float* positions, uint64_t* remaining,
                        uint8_t* termination, uint64_t* steps,
                        int record, uint64_t curve_stride, float* raw_vertices) {
  if (!grid || (count && (!positions || !remaining))) return 1;
  if (!((integrator >= ORACLE_EULER && integrator <= ORACLE_ADAMS_BASHFORTH_MOULTON_2) ||
        integrator == ORACLE_RUNGE_KUTTA_4_TRUE))
    return 2;
  if (record) {
    if (!raw_vertices) return 1;
    for (uint64_t i = 0; i < count; ++i)
      if (remaining[i] + 2 > curve_stride) return 1;
    std::fill(raw_vertices, raw_vertices + count * curve_stride * 3, kInvalid);
  }
  const step_coefficients k = make_coefficients(step_size);
  const int threads = oracle_get_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads)
  for (long long i = 0; i < static_cast<long long>(count); ++i) {
    float* curve = record ? raw_vertices + static_cast<uint64_t>(i) * curve_stride * 3 : nullptr;
    uint64_t taken = 0;
    const uint8_t reason = advect_one(steady_field{*grid}, integrator, k, positions + 3 * i,
                                      remaining + i, &taken, curve);
    if (termination) termination[i] = reason;
    if (steps) steps[i] = taken;
  }
  return 0;
}

int oracle_advect_pathlines(const oracle_unsteady_grid* grid, int integrator, float step_size,
                            uint64_t count, float* positions, float* times, uint64_t* remaining,
                            uint8_t* termination, uint64_t* steps) {
  if (!grid || grid->slices < 2 || (count && (!positions || !times || !remaining))) return 1;
  if (!((integrator >= ORACLE_EULER && integrator <= ORACLE_ADAMS_BASHFORTH_MOULTON_2) ||
        integrator == ORACLE_RUNGE_KUTTA_4_TRUE))
    return 2;
  const step_coefficients k = make_coefficients(step_size);
  const unsteady_field field{*grid};
  const int threads = oracle_get_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads)
  for (long long i = 0; i < static_cast<long long>(count); ++i) {
    uint64_t taken = 0;
    const uint8_t reason = advect_one(field, integrator, k, positions + 3 * i, remaining + i,
                                      &taken, nullptr, times + i);
    if (termination) termination[i] = reason;
    if (steps) steps[i] = taken;
  }
  return 0;
}

uint64_t oracle_prune(float* vertices, uint64_t vertex_count) {
  uint64_t kept = 0;
  for (uint64_t i = 0; i < vertex_count; ++i) {
    const float* v = vertices + 3 * i;
    if (equals_sentinel(v, kInvalid)) continue;
    if (kept != i) std::memmove(vertices + 3 * kept, v, 3 * sizeof(float));
    ++kept;
  }
  return kept;
}

// index_generator.cpp:10-39: 2V slots preset to the type's maximum, pairs
// (i, i+1) set where neither vertex is the terminal sentinel, then every
// maximum removed.
uint64_t oracle_generate_indices(const float* vertices, uint64_t vertex_count, int index64,
                                 void* indices) {
  if (vertex_count == 0) return 0;
  auto run = [&](auto* out) -> uint64_t {
    using T = std::remove_pointer_t<decltype(out)>;
    std::vector<T> slots(2 * vertex_count, std::numeric_limits<T>::max());
    for (uint64_t i = 0; i + 1 < vertex_count; ++i) {
      if (!equals_sentinel(vertices + 3 * i, kTerminal) &&
          !equals_sentinel(vertices + 3 * (i + 1), kTerminal)) {
        slots[2 * i]     = static_cast<T>(i);
        slots[2 * i + 1] = static_cast<T>(i + 1);
      }
    }
    uint64_t kept = 0;
    for (const T s : slots)
      if (s != std::numeric_limits<T>::max()) out[kept++] = s;
    return kept;
  };
  return index64 ? run(static_cast<uint64_t*>(indices)) : run(static_cast<uint32_t*>(indices));
}

// color_generator.cpp:37-58 (generate_from_angular_velocities).
void oracle_generate_colors(const float* vertices, uint64_t vertex_count, float* colors) {
  auto normalized = [](float* v) {
    const float z = v[0] * v[0] + (v[1] * v[1] + v[2] * v[2]);
    if (z > 0.0f) {
      const float n = std::sqrt(z);
      v[0] = v[0] / n; v[1] = v[1] / n; v[2] = v[2] / n;
    }
  };
  for (uint64_t i = 0; i < vertex_count; ++i) {
    colors[i] = 0.0f;
    const float* v = vertices + 3 * i;
    if (equals_sentinel(v, kTerminal)) continue;
    float prev[3] = {0.0f, 0.0f, 0.0f}, next[3] = {0.0f, 0.0f, 0.0f};
    if (i > 1 && !equals_sentinel(v - 3, kTerminal)) {
      for (int c = 0; c < 3; ++c) prev[c] = v[c] - v[c - 3];
      normalized(prev);
    }
    if (i + 1 < vertex_count && !equals_sentinel(v + 3, kTerminal)) {
      for (int c = 0; c < 3; ++c) next[c] = v[c + 3] - v[c];
      normalized(next);
    }
    const float cross[3] = {prev[1] * next[2] - prev[2] * next[1],
                            prev[2] * next[0] - prev[0] * next[2],
                            prev[0] * next[1] - prev[1] * next[0]};
    const float norm = std::sqrt(cross[0] * cross[0] + (cross[1] * cross[1] + cross[2] * cross[2]));
    const float dot = prev[0] * next[0] + (prev[1] * next[1] + prev[2] * next[2]);
    colors[i] = std::atan2(norm, dot);
  }
}

// uniform_seed_generator.cpp:16-45 with unravel_index of indexing.hpp:11-20
// (last axis fastest).
uint64_t oracle_lattice_seeds(const float offset_in[3], const float size_in[3],
                              const float stride[3], const float* aabb,
                              uint64_t shape_out[3], float* out) {
  float offset[3] = {offset_in[0], offset_in[1], offset_in[2]};
  float size[3] = {size_in[0], size_in[1], size_in[2]};
  if (aabb) {
    float lo[3], hi[3];
    bool empty = false;
    for (int i = 0; i < 3; ++i) {
      lo[i] = std::max(aabb[i], offset[i]);
      hi[i] = std::min(aabb[3 + i], offset[i] + size[i]);
      if (lo[i] > hi[i]) empty = true;
    }
    if (empty) {
      if (shape_out) shape_out[0] = shape_out[1] = shape_out[2] = 0;
      return 0;
    }
    for (int i = 0; i < 3; ++i) { offset[i] = lo[i]; size[i] = hi[i] - lo[i]; }
  }
  uint64_t shape[3];
  for (int i = 0; i < 3; ++i) shape[i] = static_cast<uint64_t>(size[i] / stride[i]);
  if (shape_out) for (int i = 0; i < 3; ++i) shape_out[i] = shape[i];
  const uint64_t count = shape[0] * shape[1] * shape[2];
  if (out) {
    for (uint64_t index = 0; index < count; ++index) {
      uint64_t rest = index, sub[3];
      for (int i = 2; i >= 0; --i) { sub[i] = rest % shape[i]; rest /= shape[i]; }
      for (int i = 0; i < 3; ++i)
        out[3 * index + i] = offset[i] + stride[i] * static_cast<float>(sub[i]);
    }
  }
  return count;
}

// ftle_estimator.cpp:7-65 with the gradient of regular_grid.hpp:87-108.
int oracle_ftle(const uint64_t field_shape[3], const float offset[3], const float spacing[3],
                const float seed_stride[3], uint64_t iterations, float step_size,
                uint64_t count, const float* original_positions, const float* final_positions,
                int mapping, float* ftle, uint64_t shape_out[3],
                uint64_t* collisions, uint64_t* holes, uint64_t* outside) {
  uint64_t shape[3];
  float sp[3], two_sp[3];
  for (int i = 0; i < 3; ++i) {
    shape[i] = static_cast<uint64_t>(static_cast<float>(field_shape[i]) / seed_stride[i]);
    sp[i] = spacing[i] * seed_stride[i];
    two_sp[i] = 2.0f * sp[i];
  }
  if (shape_out) for (int i = 0; i < 3; ++i) shape_out[i] = shape[i];
  const uint64_t cells = shape[0] * shape[1] * shape[2];
  if (mapping == 1 && count != cells) return 1;
  std::vector<float> flow(cells * 3, 0.0f);
  std::vector<uint32_t> writes(cells, 0);
  uint64_t out_of_range = 0;
  // Scatter in particle order: on a collision the larger particle index wins.
  for (uint64_t p = 0; p < count; ++p) {
    uint64_t cell;
    if (mapping == 1) {
      cell = p;
    } else {
      uint64_t sub[3];
      bool inside = true;
      for (int i = 0; i < 3; ++i) {
        const float s = std::floor((original_positions[3 * p + i] - offset[i]) / sp[i]);
        if (!(s >= 0.0f) || !(s < static_cast<float>(shape[i]))) { inside = false; break; }
        sub[i] = static_cast<uint64_t>(s);
      }
      if (!inside) { ++out_of_range; continue; }
      cell = (sub[0] * shape[1] + sub[1]) * shape[2] + sub[2];
    }
    std::memcpy(&flow[3 * cell], final_positions + 3 * p, 3 * sizeof(float));
    ++writes[cell];
  }
  if (collisions || holes) {
    uint64_t c = 0, h = 0;
    for (const uint32_t w : writes) { c += (w > 1); h += (w == 0); }
    if (collisions) *collisions = c;
    if (holes) *holes = h;
  }
  if (outside) *outside = out_of_range;
  const float horizon = std::fabs(step_size * static_cast<float>(iterations));
  const int threads = oracle_get_threads();
#pragma omp parallel for schedule(static) num_threads(threads)
  for (long long flat = 0; flat < static_cast<long long>(cells); ++flat) {
    uint64_t sub[3];
    uint64_t rest = static_cast<uint64_t>(flat);
    for (int i = 2; i >= 0; --i) { sub[i] = rest % shape[i]; rest /= shape[i]; }
    float J[3][3];  // J[r][d] = d flow_r / d x_d
    for (int d = 0; d < 3; ++d) {
      uint64_t prev[3] = {sub[0], sub[1], sub[2]}, next[3] = {sub[0], sub[1], sub[2]};
      if (sub[d] > 0) prev[d] -= 1;
      if (sub[d] < shape[d] - 1) next[d] += 1;
      const float* a = &flow[3 * ((next[0] * shape[1] + next[1]) * shape[2] + next[2])];
      const float* b = &flow[3 * ((prev[0] * shape[1] + prev[1]) * shape[2] + prev[2])];
      for (int r = 0; r < 3; ++r) J[r][d] = (a[r] - b[r]) / two_sp[d];
    }
    double C[3][3];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j)
        C[i][j] = static_cast<double>(J[0][i] * J[0][j] + (J[1][i] * J[1][j] + J[2][i] * J[2][j]));
    const double lambda = symmetric3_max_eigenvalue(C);
    ftle[flat] = static_cast<float>(std::log(std::sqrt(lambda)) / static_cast<double>(horizon));
  }
  return 0;
}

int oracle64_advect(const oracle_grid* grid, int integrator, double step_size,
                    uint64_t count, double* positions, uint64_t* remaining,
                    uint8_t* termination, uint64_t* steps) {
  if (!grid) return 1;
  if (integrator != ORACLE_EULER && integrator != ORACLE_RUNGE_KUTTA_4 &&
      integrator != ORACLE_RUNGE_KUTTA_4_TRUE)
    return 2;
  const oracle_grid& g = *grid;
  const int threads = oracle_get_threads();
#pragma omp parallel for schedule(dynamic, 64) num_threads(threads)
  for (long long i = 0; i < static_cast<long long>(count); ++i) {
    uint64_t taken = 0;
    const uint8_t reason = advect_one64(
        integrator, step_size, positions + 3 * i, remaining + i, &taken,
        [&](const double* p) { return grid_contains64(g, p); },
        [&](const double* p, double* d) { grid_interpolate64(g, p, d); });
    if (termination) termination[i] = reason;
    if (steps) steps[i] = taken;
  }
  return 0;
}

int oracle64_advect_abc(double A, double B, double C, const double lo[3], const double hi[3],
                        double step_size, uint64_t count, double* positions,
                        uint64_t* remaining, uint8_t* termination, uint64_t* steps) {
  const int threads = oracle_get_threads();
#pragma omp parallel for schedule(dynamic, 64) num_threads(threads)
  for (long long i = 0; i < static_cast<long long>(count); ++i) {
    uint64_t taken = 0;
    const uint8_t reason = advect_one64(
        ORACLE_RUNGE_KUTTA_4_TRUE, step_size, positions + 3 * i, remaining + i, &taken,
        [&](const double* p) {
          for (int k = 0; k < 3; ++k)
            if (!(p[k] >= lo[k] && p[k] < hi[k])) return false;
          return true;
        },
        [&](const double* p, double* d) {
          d[0] = A * std::sin(p[2]) + C * std::cos(p[1]);
          d[1] = B * std::sin(p[0]) + A * std::cos(p[2]);
          d[2] = C * std::sin(p[1]) + B * std::cos(p[0]);
        });
    if (termination) termination[i] = reason;
    if (steps) steps[i] = taken;
  }
  return 0;
}

}  // extern "C"
