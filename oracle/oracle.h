/*
 * oracle.h -- C interface of the CPU oracle for the dpa advection path.
 *
 * TEST INFRASTRUCTURE ONLY. The oracle is a CPU restatement of the reference
 * algorithm (VRGroupRWTH/dpa, files cited per function in oracle.cpp). It is
 * the checker for the CUDA path and the timed CPU baseline. Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline / reference arm may load
 * it. The product library (dpa_b200/libdpa_b200.so) never links or calls it.
 *
 * PARITY UNPINNED: the reference ships no tests, fixtures or golden vectors
 * (tests/catch/main.cpp only defines a Catch2 main) and cannot be compiled in
 * this environment (Boost.Odeint, Eigen, TBB, HDF5 and MPI are absent). The
 * restatement is anchored on the reference source text, on the published
 * algorithms of its two third-party arithmetic dependencies (Boost.Odeint
 * generic explicit Runge-Kutta, Eigen 3.3 fixed-size reductions; neither
 * version is pinned by the reference, which installs them through vcpkg) and
 * on analytic known answers checked in tests/.
 *
 * Array conventions (all C-order, little endian):
 *   field      float [nx][ny][nz][3]   (the reference's XYZV dataset layout)
 *   positions  float [count][3]
 *   remaining  uint64 [count]          (particle_3d::remaining_iterations)
 */
#ifndef DPA_ORACLE_H
#define DPA_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_grid {
  const float* data;      /* [n0][n1][n2][3] */
  uint64_t     shape[3];
  float        offset[3];
  float        spacing[3];
} oracle_grid;

/* Integrator codes follow the order of the reference's integrator variant
 * (include/dpa/types/integrators.hpp:31-39); 100 is the four-sample
 * Runge-Kutta 4 (no counterpart in the reference). The FP64 oracle takes
 * euler, runge_kutta_4 and 100 only. */
enum {
  ORACLE_EULER = 0,
  ORACLE_MODIFIED_MIDPOINT = 1,
  ORACLE_RUNGE_KUTTA_4 = 2,
  ORACLE_RUNGE_KUTTA_CASH_KARP_54 = 3,
  ORACLE_RUNGE_KUTTA_DORMAND_PRINCE_5 = 4,
  ORACLE_RUNGE_KUTTA_FEHLBERG_78 = 5,
  ORACLE_ADAMS_BASHFORTH_2 = 6,
  ORACLE_ADAMS_BASHFORTH_MOULTON_2 = 7,
  ORACLE_RUNGE_KUTTA_4_TRUE = 100
};

/* Termination reasons recorded per particle. */
enum { ORACLE_COMPLETE = 0, ORACLE_OUT_OF_BOUNDS = 1, ORACLE_ZERO_VELOCITY = 2 };

void oracle_set_threads(int threads);
int  oracle_get_threads(void);

int  oracle_contains(const oracle_grid* grid, const float position[3]);
void oracle_interpolate(const oracle_grid* grid, const float position[3], float out[3]);

/* One advection round of `count` particles (particle_advector.cpp:311-401).
 * positions / remaining are updated in place. termination and steps (may be
 * NULL) receive the exit reason and the number of steps taken. If record is
 * non-zero, raw_vertices must hold count*curve_stride*3 floats; it is filled
 * with the invalid sentinel and then written exactly like the reference's
 * unpruned curve buffer. Returns 0 on success. */
int oracle_advect_round(const oracle_grid* grid, int integrator, float step_size,
                        uint64_t count, float* positions, uint64_t* remaining,
                        uint8_t* termination, uint64_t* steps,
                        int record, uint64_t curve_stride, float* raw_vertices);

/* A time-varying field: `slices` grids of one shape, slice s at time
 * time_origin + s * time_spacing. Not part of the reference, which advects
 * steady fields; the pathline rules restate the library's documented ones. */
typedef struct oracle_unsteady_grid {
  const float* data;      /* [slices][n0][n1][n2][3] */
  uint64_t     shape[3];
  uint64_t     slices;
  float        offset[3];
  float        spacing[3];
  float        time_origin;
  float        time_spacing;
} oracle_unsteady_grid;

/* Pathlines: oracle_advect_round's particle loop (no recording) with a time
 * per particle, advanced by step_size per step; a particle whose time leaves
 * the slices' span ends out of bounds. */
int oracle_advect_pathlines(const oracle_unsteady_grid* grid, int integrator, float step_size,
                            uint64_t count, float* positions, float* times, uint64_t* remaining,
                            uint8_t* termination, uint64_t* steps);

/* Removes invalid-sentinel vertices in place; returns the kept count
 * (particle_advector.cpp:402-408). */
uint64_t oracle_prune(float* vertices, uint64_t vertex_count);

/* Index generation (index_generator.cpp:10-39). indices must hold
 * 2*vertex_count entries of uint32 (index64 == 0) or uint64. Returns the
 * number of indices kept. */
uint64_t oracle_generate_indices(const float* vertices, uint64_t vertex_count,
                                 int index64, void* indices);

/* Angular-velocity colors (color_generator.cpp:37-58). */
void oracle_generate_colors(const float* vertices, uint64_t vertex_count, float* colors);

/* Lattice seeds (uniform_seed_generator.cpp:16-45, indexing.hpp:11-20).
 * aabb may be NULL or {min0,min1,min2,max0,max1,max2}. Returns the particle
 * count; writes positions if out is not NULL. shape_out receives the per-axis
 * counts. */
uint64_t oracle_lattice_seeds(const float offset[3], const float size[3],
                              const float stride[3], const float* aabb,
                              uint64_t shape_out[3], float* out);

/* FTLE (ftle_estimator.cpp:7-65, regular_grid.hpp:28-34,87-108).
 * mapping 0 scatters each final position into the flow-map cell of its
 * original position, as the reference does; on a collision the particle with
 * the larger index wins. mapping 1 scatters by lattice id (particle i goes to
 * flat cell i), which requires count == product(shape). ftle receives
 * product(shape) floats, shape = floor(field shape / seed stride).
 * collisions / holes (may be NULL) receive the count of cells written more
 * than once and never. Returns 0 on success. */
int oracle_ftle(const uint64_t field_shape[3], const float offset[3], const float spacing[3],
                const float seed_stride[3], uint64_t iterations, float step_size,
                uint64_t count, const float* original_positions, const float* final_positions,
                int mapping, float* ftle, uint64_t shape_out[3],
                uint64_t* collisions, uint64_t* holes, uint64_t* outside);

/* FP64 oracle: the same per-particle loop in double precision on the same
 * float field samples. integrator 0 / 2 / 100. */
int oracle64_advect(const oracle_grid* grid, int integrator, double step_size,
                    uint64_t count, double* positions, uint64_t* remaining,
                    uint8_t* termination, uint64_t* steps);

/* FP64 oracle on the analytic ABC flow u = (A sin z + C cos y, B sin x + A cos z,
 * C sin y + B cos x), four-sample RK4, domain box [lo, hi) per axis. */
int oracle64_advect_abc(double A, double B, double C, const double lo[3], const double hi[3],
                        double step_size, uint64_t count, double* positions,
                        uint64_t* remaining, uint8_t* termination, uint64_t* steps);

#ifdef __cplusplus
}
#endif

#endif
