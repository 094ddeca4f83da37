/*
 * dpa_b200.h -- C ABI of the B200 (sm_100a) advection library.
 *
 * This library replaces the advection stage of VRGroupRWTH/dpa: the per-round
 * particle integration of particle_advector (source/stages/particle_advector.cpp),
 * its curve pruning, the index and color post-passes and the FTLE estimator.
 * Plain pointers and sizes only; every entry point returns a dpa_status and
 * nothing throws across this boundary. A context is bound to one device and is
 * not re-entrant: use one context per host thread.
 *
 * Array conventions (C-order, little endian):
 *   field       float [n0][n1][n2][3]   the reference's XYZV dataset
 *               (regular_grid_loader.cpp:65-88 reads it into boost::multi_array)
 *   positions   float [count][3]        particle_3d::position (particle.hpp:70)
 *   remaining   uint64 [count]          particle_3d::remaining_iterations
 *   termination uint8 [count]           dpa_termination per particle
 */
#ifndef DPA_B200_H
#define DPA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct dpa_context dpa_context;
typedef struct dpa_field dpa_field;
typedef struct dpa_graph dpa_graph;
typedef struct dpa_server dpa_server;

typedef enum dpa_status {
  DPA_OK = 0,
  DPA_ERROR_INVALID_ARGUMENT = 1,
  DPA_ERROR_UNSUPPORTED = 2,
  DPA_ERROR_OUT_OF_MEMORY = 3,
  DPA_ERROR_CUDA = 4,
  DPA_ERROR_SINK = 5,
  DPA_ERROR_INTERNAL = 6,
  DPA_ERROR_TIMEOUT = 7,   /* a served request passed its deadline and was dropped */
  DPA_ERROR_CANCELLED = 8  /* a served request was cancelled (dpa_server_cancel) */
} dpa_status;

/* Device storage of a field. F32 keeps the reference's values exactly; F16 and
 * BF16 halve the gather bytes and interpolate in FP32. F32_EDGES keeps the
 * F32 values (results identical to F32) as one 32-byte record per cell edge
 * along axis 2, twice F32's memory: a cell's corners are four loads instead
 * of eight, which pays where particles change cells almost every step (dense
 * FTLE lattices) and costs a little on sparse seeds in large fields. */
typedef enum dpa_storage {
  DPA_STORAGE_F32 = 0,
  DPA_STORAGE_F16 = 1,
  DPA_STORAGE_BF16 = 2,
  DPA_STORAGE_F32_EDGES = 3
} dpa_storage;

/* Integrators. Codes 0-7 follow the alternatives of the reference's
 * variant_integrator (include/dpa/types/integrators.hpp:31-39) and the names
 * of particle_advector.cpp:29-36, with the reference's semantics: its system
 * functor (particle_advector.cpp:376) samples the field once per step, so
 * every stage of a step sees the same derivative and each odeint stepper
 * reduces to its final combination. runge_kutta_dormand_prince_5 (its
 * first-same-as-last derivative is the previous step's sample),
 * adams_bashforth_2 (derivative history) and adams_bashforth_moulton_2
 * (extrapolated first step) depend on a particle's earlier steps: calls with
 * max_steps and the request server refuse them (DPA_ERROR_UNSUPPORTED).
 * DPA_INTEGRATOR_RUNGE_KUTTA_4_TRUE samples at all four stages (no
 * counterpart in the reference). */
typedef enum dpa_integrator {
  DPA_INTEGRATOR_EULER = 0,
  DPA_INTEGRATOR_MODIFIED_MIDPOINT = 1,
  DPA_INTEGRATOR_RUNGE_KUTTA_4 = 2,
  DPA_INTEGRATOR_RUNGE_KUTTA_CASH_KARP_54 = 3,
  DPA_INTEGRATOR_RUNGE_KUTTA_DORMAND_PRINCE_5 = 4,
  DPA_INTEGRATOR_RUNGE_KUTTA_FEHLBERG_78 = 5,
  DPA_INTEGRATOR_ADAMS_BASHFORTH_2 = 6,
  DPA_INTEGRATOR_ADAMS_BASHFORTH_MOULTON_2 = 7,
  DPA_INTEGRATOR_RUNGE_KUTTA_4_TRUE = 100
} dpa_integrator;

/* Why a particle stopped (particle_advector.cpp:336-395). */
typedef enum dpa_termination {
  DPA_TERMINATION_COMPLETE = 0,      /* remaining_iterations reached 0 */
  DPA_TERMINATION_OUT_OF_BOUNDS = 1, /* regular_grid::contains failed */
  DPA_TERMINATION_ZERO_VELOCITY = 2, /* interpolated vector isZero() */
  DPA_TERMINATION_IN_FLIGHT = 3,     /* stopped by dpa_advect_options.max_steps; resumable */
  DPA_TERMINATION_CANCELLED = 4      /* served request dropped (deadline or cancel) while the
                                        particle was still in flight */
} dpa_termination;

/* FTLE scatter rule. REFERENCE puts each final position into the flow-map
 * cell of floor((original_position - offset) / (spacing * stride)) exactly as
 * ftle_estimator.cpp:39-43 does (rounding can map two seeds to one cell; the
 * larger particle index then wins, and unmapped cells stay zero). LATTICE puts
 * particle i into flat cell i (count must equal the lattice size). */
typedef enum dpa_ftle_mapping {
  DPA_FTLE_MAPPING_REFERENCE = 0,
  DPA_FTLE_MAPPING_LATTICE = 1
} dpa_ftle_mapping;

typedef struct dpa_advect_options {
  int32_t integrator;   /* dpa_integrator */
  float   step_size;    /* particle_advector_step_size */
  int32_t record;       /* particle_advector_record: emit the round's curve */
  int32_t index64;      /* 64-bit indices (pipeline.cpp:155 decides) */
  int32_t colors;       /* emit angular-velocity colors with the curve */
  int32_t morton_order; /* process particles in Morton order of their start cell */
  uint64_t max_steps;   /* 0: no limit. Otherwise a particle takes at most this
                           many steps per call and, if it could go on, ends the
                           call as DPA_TERMINATION_IN_FLIGHT with its position
                           and remaining count updated, ready to resume (device
                           calls without recording only) */
} dpa_advect_options;

/* One chunk of a round's curve, delivered in order (a round arrives in one or
 * more chunks; vertex and index ranges each continue where the previous chunk
 * ended). The round's curve is the
 * reference's integral_curve after advect, prune_integral_curves,
 * index_generator::generate and color_generator::generate_from_angular_velocities
 * (particle_advector.cpp:402-408, index_generator.cpp:10-39,
 * color_generator.cpp:37-58). Index values are positions in the round's whole
 * vertex array. Pointers are host memory owned by the library and valid only
 * during the callback. */
typedef struct dpa_curve_chunk {
  uint64_t     vertex_offset; /* first vertex of this chunk within the round */
  uint64_t     vertex_count;
  const float* vertices;      /* vertex_count * 3 */
  const float* colors;        /* vertex_count, or NULL when colors are off */
  uint64_t     index_offset;  /* first index of this chunk within the round */
  uint64_t     index_count;
  const void*  indices;       /* uint32 or uint64 per dpa_advect_options.index64 */
  int32_t      last;          /* non-zero on the round's final chunk */
} dpa_curve_chunk;

/* Returns 0 to continue; any other value aborts the round with DPA_ERROR_SINK. */
typedef int (*dpa_curve_sink)(void* user, const dpa_curve_chunk* chunk);

/* ---- library and context ------------------------------------------------ */

const char* dpa_version(void);

/* Number of visible CUDA devices (0 when none or when the driver is absent). */
int dpa_device_count(int* count);

int dpa_context_create(int device, dpa_context** out);
int dpa_context_destroy(dpa_context* ctx);

/* Message of the last failed call on this context (never NULL). */
const char* dpa_last_error(const dpa_context* ctx);

/* The context's CUDA stream (a cudaStream_t) for callers that order their own
 * work against the library's. */
void* dpa_context_stream(dpa_context* ctx);

int dpa_context_synchronize(dpa_context* ctx);

/* Upper bound on the device bytes a recording round may stage at once; larger
 * rounds are processed in pieces (default 1 GiB). */
int dpa_context_set_staging_limit(dpa_context* ctx, uint64_t bytes);

/* Upper bound on the curve bytes one sink chunk carries (default 256 MiB of
 * vertices and colors, and as many bytes of indices). A piece's curve crosses
 * to the host through two pinned buffers of this size, the next chunk copying
 * while the sink takes the current one. */
int dpa_context_set_host_chunk_limit(dpa_context* ctx, uint64_t bytes);

/* Instrumentation, the counterpart of the reference's per-round timers
 * (pipeline.cpp:98-145, benchmark.hpp:152-158). With profiling on, every
 * advection records CUDA events on its stream around the ordering kernels
 * and the advection kernel (and, in a recording round, around each piece's
 * emission: curve offsets and emit kernel); dpa_context_last_timing waits for
 * the last call's events and returns both durations in milliseconds (summed
 * over the pieces of a recording round), dpa_context_last_emit_timing the
 * emission time of the last recording round. */
int dpa_context_set_profiling(dpa_context* ctx, int32_t enabled);
int dpa_context_last_timing(dpa_context* ctx, float* order_ms, float* advect_ms);
int dpa_context_last_emit_timing(dpa_context* ctx, float* emit_ms);

/* The device's load bandwidth for the advection kernels' gather pattern:
 * lanes load the eight 16-byte nodes of one cell (four edges of two
 * consecutive nodes) per iteration from a table of at most table_bytes.
 * pattern 0: the lanes of a warp read consecutive cells (the data path's
 * ceiling); 1: every lane reads a random cell. A table that fits each SM's
 * L1 (tens of KiB) measures the L1 data path, one that fits L2 (tens of MiB)
 * the L2 path. Returns node bytes delivered per second, in GB/s. No
 * counterpart in the reference; it gives the gather roofline its peak. */
int dpa_measure_gather_bandwidth(dpa_context* ctx, uint64_t table_bytes, int32_t pattern,
                                 double* gigabytes_per_second);

/* Number of kernels this context has launched on the advection path. */
int dpa_context_launch_count(const dpa_context* ctx, uint64_t* launches);

/* ---- integrator names ----------------------------------------------------- */

/* Maps the reference's config strings (particle_advector.cpp:29-36) and
 * "runge_kutta_4_true" to a dpa_integrator. Unknown names are an error (the
 * reference silently keeps euler). */
int dpa_integrator_from_name(const char* name, int32_t* integrator);

/* ---- fields ---------------------------------------------------------------- */

/* Replaces regular_grid_loader::load_vector_field (regular_grid_loader.cpp:65-88):
 * uploads a host XYZV field and repacks it for the device in the given storage.
 * offset/spacing are the grid's world offset and cell spacing. Each axis holds
 * 1 to 2^23 nodes, and a slice fewer than 2^32 (DPA_ERROR_INVALID_ARGUMENT
 * otherwise). */
int dpa_field_create(dpa_context* ctx, const float* xyzv, const uint64_t shape[3],
                     const float offset[3], const float spacing[3], int32_t storage,
                     dpa_field** out);

/* Same, from a device pointer already in this context's device memory. */
int dpa_field_create_device(dpa_context* ctx, const float* device_xyzv, const uint64_t shape[3],
                            const float offset[3], const float spacing[3], int32_t storage,
                            dpa_field** out);

/* Waits for the context's stream, then frees the field. Graphs captured on a
 * field and servers it was added to keep its device address: destroy them
 * first. */
int dpa_field_destroy(dpa_context* ctx, dpa_field* field);

int dpa_field_info(const dpa_field* field, uint64_t shape[3], float offset[3], float spacing[3],
                   int32_t* storage, uint64_t* device_bytes);

/* A time-varying field (no counterpart in the reference, which advects
 * steady fields): `slices` (>= 2) samples of one grid, slice s holding the
 * field at time time_origin + s * time_spacing, in host memory as
 * [slices][n0][n1][n2][3]. The velocity at (p, t) blends the trilinear samples
 * of slices s and s + 1 at p as (1 - w) a + w b, where s = floor((t - t0) /
 * dt) and w = fmod(t - t0, dt) / dt (the spatial rule on the time axis); a
 * particle whose time leaves [t0, t0 + (slices - 1) dt) ends out of bounds.
 * Advect it with dpa_advect_pathlines_device or the request server; the
 * other advection calls refuse it. */
int dpa_field_create_unsteady(dpa_context* ctx, const float* xyzv, const uint64_t shape[3],
                              uint32_t slices, const float offset[3], const float spacing[3],
                              float time_origin, float time_spacing, int32_t storage,
                              dpa_field** out);

/* How the field's kernels divide a position by the spacing: 2 = power-of-two
 * spacings (one FMA of exact scaled values), 1 = division by the reciprocal
 * split into two floats (one multiply and one FMA), used only for spacings
 * for which it was checked on the device, at field creation, to give IEEE
 * division's bits for every float dividend, 0 = IEEE division. All three give
 * the reference's rounded quotient. */
int dpa_field_locate_mode(const dpa_field* field, int32_t* mode);

/* Fields created on this context from now on use IEEE division (mode 0)
 * whatever their spacing, when enabled (for comparison; off by default). */
int dpa_context_set_ieee_division(dpa_context* ctx, int32_t enabled);

/* slices = 1 (and zero times) for a steady field. */
int dpa_field_time_info(const dpa_field* field, uint32_t* slices, float* time_origin,
                        float* time_spacing);

/* ---- advection --------------------------------------------------------------- */

/* One advection round over host arrays: replaces particle_advector::
 * allocate_integral_curves + advect + prune_integral_curves
 * (particle_advector.cpp:311-408, called from pipeline.cpp:115-127) and, when
 * recording, the index and color post-passes for that round. positions and
 * remaining are updated in place; termination (may be NULL) receives the exit
 * reason. With options->record, the round's curve goes to sink in order. */
int dpa_advect_round(dpa_context* ctx, const dpa_field* field, const dpa_advect_options* options,
                     uint64_t count, float* positions, uint64_t* remaining,
                     uint8_t* termination, dpa_curve_sink sink, void* sink_user);

/* The same round over device arrays on the given stream (NULL: the context's
 * stream), without recording. Asynchronous: returns after enqueueing. */
int dpa_advect_device(dpa_context* ctx, const dpa_field* field, const dpa_advect_options* options,
                      uint64_t count, float* device_positions, uint64_t* device_remaining,
                      uint8_t* device_termination, void* stream);

/* dpa_advect_device with a time per particle (device_times, float[count]),
 * advanced by step_size for every step taken and updated in place: pathlines
 * through a time-varying field (dpa_field_create_unsteady), or streamlines
 * through a steady one with their times tracked. Four-sample RK4 samples its
 * stages at t, t + dt/2 and t + dt; the other integrators sample at t. With
 * max_steps a particle resumes at its stored time in a later call. */
int dpa_advect_pathlines_device(dpa_context* ctx, const dpa_field* field,
                                const dpa_advect_options* options, uint64_t count,
                                float* device_positions, float* device_times,
                                uint64_t* device_remaining, uint8_t* device_termination,
                                void* stream);

/* ---- batching, graphs and tuning (no counterpart in the reference) -------- */

/* Many seed sets in one persistent launch: set s is particles
 * [set_offsets[s], set_offsets[s+1]) of the device arrays (set_offsets is a
 * host array of set_count + 1 entries starting at 0). Every particle carries
 * its own remaining count, so sets of any size and iteration count share the
 * launch. set_steps (host, may be NULL) receives the particle-steps each set
 * took; asking for it makes the call wait for the launch. No recording. */
int dpa_advect_batch_device(dpa_context* ctx, const dpa_field* field,
                            const dpa_advect_options* options, uint64_t set_count,
                            const uint64_t* set_offsets, float* device_positions,
                            uint64_t* device_remaining, uint8_t* device_termination,
                            uint64_t* set_steps, void* stream);

/* The launch sequence of dpa_advect_device (processing order + advection) for
 * fixed device arrays, captured once into a CUDA graph; each
 * dpa_graph_launch replays it on a stream (NULL: the context's). The graph
 * owns its scratch (8 bytes per particle and about 1 MB), so the context's
 * other calls may run between replays; replays of one graph must not
 * overlap. dpa_graph_destroy waits for the device. */
int dpa_graph_create_advect(dpa_context* ctx, const dpa_field* field,
                            const dpa_advect_options* options, uint64_t count,
                            float* device_positions, uint64_t* device_remaining,
                            uint8_t* device_termination, dpa_graph** out);
int dpa_graph_launch(dpa_context* ctx, dpa_graph* graph, void* stream);
int dpa_graph_destroy(dpa_context* ctx, dpa_graph* graph);

/* Launch parameters of a context's advection kernels. */
typedef struct dpa_tuning {
  uint32_t claim;          /* processing-order entries a warp takes per atomic claim */
  uint32_t blocks_per_sm;  /* persistent grid blocks per SM; 0 = as many as fit */
  uint32_t order;          /* processing order: Morton buckets of a order^3 coarsening
                              of the grid (1..64), 0 = input order */
  float    measured_ms;    /* dpa_autotune_advect: time of the chosen setting */
  uint32_t block_size;     /* threads per block, a multiple of 32 up to 256; 0 = 256,
                              or fewer when a launch's particles would not reach
                              every SM */
  uint32_t particles_per_thread; /* 1 or 2 particles stepped together by each lane
                              (2 applies to steady fields without recording) */
} dpa_tuning;

int dpa_context_set_tuning(dpa_context* ctx, const dpa_tuning* tuning);
int dpa_context_get_tuning(const dpa_context* ctx, dpa_tuning* tuning);

/* Times candidate settings on copies of the first min(count, 4,194,304) of
 * the given device particles, each advanced at most sample_steps steps (0: its
 * whole remaining budget, capped by options->max_steps), keeps the fastest in
 * the context and returns it in best (may be NULL). The search goes one knob
 * group at a time from the defaults, keeping the best so far: processing order
 * (64 / 16 / off), then launch shape (256, 128 or 64 threads per block, one or
 * two particles per lane), then claim size (16 or 32) with blocks per SM (all
 * that fit, 3, 2). A setting tried later replaces the best so far only when
 * it is at least 3 % faster. The processing order pays off with particle
 * density and run length, so a sample as dense and as long as the real run
 * picks the setting that run wants. */
int dpa_autotune_advect(dpa_context* ctx, const dpa_field* field, const dpa_advect_options* options,
                        uint64_t count, const float* device_positions,
                        const uint64_t* device_remaining, uint64_t sample_steps,
                        dpa_tuning* best);

/* ---- serving (no counterpart in the reference) ------------------------------ */

/* A request server: fields stay resident, and requests are admitted when the
 * device arenas have room for them (count particle slots; for recording
 * requests also count * (iterations + 2) curve-staging vertices, their output
 * buffer). Admission scans the waiting requests oldest first and admits every
 * one that fits, so a small request does not wait behind a large one that has
 * no room yet; reserved_percent of the slots are kept for small requests (at
 * most small_request_seeds seeds), and once the oldest waiting request has
 * waited max_bypass_ms nothing behind it is admitted before it. Admitted
 * requests advance together in ticks of steps_per_tick steps: one persistent
 * launch per group of requests sharing a field, integrator, step size and
 * recording switch. Requests that arrive while others run join at the next
 * tick. A worker thread owns the ticks; a second thread, on its own stream,
 * copies out, emits and returns the requests that have finished while the
 * ticks go on. A request of 4096 seeds or more is swept in the Morton order
 * of its seeds' start cells. The launches use the context's tuning
 * (dpa_context_set_tuning) as it was when the server was created; an order of
 * 0 there sweeps requests in submission order. submit, poll, cancel and stats
 * may be called from any thread. The context is used for its device, its
 * fields and that tuning only.
 *
 * Failure handling is on the host: a request with a deadline that has not
 * finished deadline_ms after its submission, or one cancelled with
 * dpa_server_cancel, is dropped between ticks (the ticks never wait on the
 * host inside a kernel) and returned with status DPA_ERROR_TIMEOUT or
 * DPA_ERROR_CANCELLED: a request dropped while waiting carries no arrays; one
 * dropped while running carries its particles as they stood (those still in
 * flight marked DPA_TERMINATION_CANCELLED) and no curve or FTLE. The other
 * requests are not affected. */
typedef struct dpa_server_options {
  uint64_t particle_capacity;  /* particle slots of the arena (62 bytes each) */
  uint64_t vertex_capacity;    /* curve-staging vertices of the arena (12 bytes each) */
  uint32_t steps_per_tick;     /* step budget of a tick while requests wait for
                                  admission (0: 64); four times as many while
                                  none waits */
  uint32_t max_requests;       /* requests admitted at once */
  uint64_t small_request_seeds; /* requests of at most this many seeds may use the
                                  reserved slots (0: 65536) */
  uint32_t reserved_percent;   /* share of the slots kept for small requests (0-90) */
  uint32_t max_bypass_ms;      /* how long the oldest waiting request may be passed
                                  by younger ones that fit (0: 250 ms); after that
                                  no large request passes it, and small ones only
                                  within the reserved share */
  uint64_t response_bytes;     /* pinned host memory for returned arrays (0: 256 MiB);
                                  a response that does not fit it is returned from
                                  pageable memory */
} dpa_server_options;

typedef struct dpa_request {
  int32_t     field;           /* from dpa_server_add_field */
  int32_t     integrator;      /* dpa_integrator */
  float       step_size;
  int32_t     record;          /* return the curve (pruned, indexed, colored) */
  int32_t     index64;
  int32_t     ftle;            /* also return the lattice FTLE of the final positions */
  float       seed_stride[3];  /* FTLE: the seeds' lattice stride in cells */
  uint64_t    count;
  const float* positions;      /* host, count * 3; copied by dpa_server_submit */
  uint64_t    iterations;      /* per seed */
  void*       user;
  float       start_time;      /* the seeds' time: pathlines through a time-varying
                                  field start there (steady fields: tracked only) */
  uint32_t    deadline_ms;     /* drop the request if it has not finished this long
                                  after submission (0: no deadline) */
} dpa_request;

/* A finished request. Arrays are host memory owned by the server until
 * dpa_server_release(id) (pinned when the response arena has room; release
 * promptly, a held response keeps its share of the arena). Times are seconds
 * since the server started. */
typedef struct dpa_response {
  uint64_t       id;
  void*          user;
  int32_t        status;        /* DPA_OK, DPA_ERROR_TIMEOUT or DPA_ERROR_CANCELLED */
  uint64_t       count;
  const float*   positions;
  const uint64_t* remaining;
  const uint8_t* termination;
  uint64_t       vertex_count;
  const float*   vertices;
  const float*   colors;
  uint64_t       index_count;
  const void*    indices;       /* uint32 or uint64 per the request's index64 */
  uint64_t       ftle_shape[3];
  const float*   ftle;
  uint64_t       particle_steps;
  double         queued_seconds;
  double         admitted_seconds;
  double         finished_seconds;
  const float*   times;         /* count: each particle's time at its end */
} dpa_response;

typedef struct dpa_server_stats {
  uint64_t submitted;
  uint64_t admitted;
  uint64_t completed;
  uint64_t ticks;
  uint64_t launches;
  uint64_t particle_steps;
  double   busy_seconds;         /* worker time spent on ticks (host side) */
  uint32_t queued;
  uint32_t active;
  double   tick_device_seconds;  /* device time of the ticks (their launches, in
                                    stream order; overlapping finishing work on
                                    the finisher's stream is not counted) */
  /* Where admission waited (for tuning arena sizes and admission options): */
  uint64_t peak_slots;           /* most particle slots in use at once */
  uint64_t peak_vertices;        /* most curve-staging vertices in use at once */
  uint64_t slot_refusals;        /* admission attempts the slot arena had no room for */
  uint64_t vertex_refusals;      /* ... the curve-staging arena had no room for */
  uint64_t overdue_scans;        /* admission scans that ended with the oldest request
                                    past max_bypass_ms still waiting (no large
                                    request passed it) */
  uint32_t peak_finishing;       /* most finished requests waiting for the finisher */
  uint32_t reserved0;
  double   finish_seconds;       /* finisher time spent returning requests */
} dpa_server_stats;

int dpa_server_create(dpa_context* ctx, const dpa_server_options* options, dpa_server** out);
/* Makes a field of the server's context resident for requests (at most 256
 * fields); it must outlive the server. */
int dpa_server_add_field(dpa_server* server, const dpa_field* field, int32_t* field_id);
/* Queues a request; DPA_ERROR_OUT_OF_MEMORY when it could never fit the arenas. */
int dpa_server_submit(dpa_server* server, const dpa_request* request, uint64_t* id);
/* Asks the server to drop a queued or running request; it comes back through
 * dpa_server_poll with status DPA_ERROR_CANCELLED (or its normal result if it
 * finished first). DPA_ERROR_INVALID_ARGUMENT for an unknown or returned id. */
int dpa_server_cancel(dpa_server* server, uint64_t id);
/* Takes one finished request (*got = 1), waiting up to wait_ms for one. */
int dpa_server_poll(dpa_server* server, int32_t wait_ms, dpa_response* out, int32_t* got);
int dpa_server_release(dpa_server* server, uint64_t id);
int dpa_server_get_stats(dpa_server* server, dpa_server_stats* out);
/* Finishes the admitted and queued requests, then stops the worker. */
int dpa_server_destroy(dpa_server* server);

/* ---- allocation-free advection ----------------------------------------------- */

/* No counterpart in the reference. dpa_advect_device for callers that must not
 * allocate device memory while running: programs whose device memory is
 * reserved up front by another owner (a framework's caching allocator, a
 * service with a fixed HBM budget), and latency-bound loops, since cudaMalloc
 * and cudaFree may synchronize the whole device and stall other streams.
 * Same inputs, outputs and results as dpa_advect_device (recording is not
 * offered); the ordering scratch comes from a fixed device array inside the
 * library (about 9 MiB, held by every GPU on which the library's code is
 * loaded until the process exits) instead of cudaMalloc. It checks its
 * arguments as dpa_advect_device does and applies the context's tuning
 * (dpa_context_set_tuning) the same way, so both give the same launches. At most
 * DPA_NO_ALLOC_MAX_PARTICLES particles per call; more is rejected with
 * DPA_ERROR_INVALID_ARGUMENT. The first call on a device resolves the array's
 * device address (and may load the library's code on that device), so make
 * it during set-up, before any stream capture. Every call shares the one
 * array: calls whose work overlaps on the GPU (two streams, or two contexts
 * on one device) race; order them on one stream or synchronize between
 * them. Asynchronous like dpa_advect_device. */
#define DPA_NO_ALLOC_MAX_PARTICLES 1048576u

int dpa_advect_device_no_alloc(dpa_context* ctx, const dpa_field* field,
                               const dpa_advect_options* options, uint64_t count,
                               float* device_positions, uint64_t* device_remaining,
                               uint8_t* device_termination, void* stream);

/* ---- seeds ------------------------------------------------------------------- */

/* Lattice seeds on the device: uniform_seed_generator::generate
 * (uniform_seed_generator.cpp:16-45, unravel order of indexing.hpp:11-20).
 * aabb is NULL or {min0,min1,min2,max0,max1,max2}. Writes count*3 floats to
 * device_positions when it is not NULL; *count and shape_out receive the
 * lattice size either way. */
int dpa_seed_lattice_device(dpa_context* ctx, const float offset[3], const float size[3],
                            const float stride[3], const float* aabb, uint64_t* count,
                            uint64_t shape_out[3], float* device_positions, void* stream);

/* Uniform random seeds on the device, for uniform_seed_generator::generate_random
 * (uniform_seed_generator.cpp:46-81). The reference draws from a thread_local
 * std::mt19937 seeded by std::random_device and can never repeat a seed set;
 * here seed i, axis a is offset[a] + size[a] * u with
 * u = (splitmix64(splitmix64(seed) ^ (3 i + a)) >> 40) * 2^-24 in [0, 1), so a
 * (seed, count) pair always gives the same seeds, on any device or host.
 * aabb clips the box as for the lattice; *count_out receives the count
 * (0 when the clipped box is empty). */
int dpa_seed_random_device(dpa_context* ctx, const float offset[3], const float size[3],
                           uint64_t count, uint64_t seed, const float* aabb, uint64_t* count_out,
                           float* device_positions, void* stream);

/* ---- FTLE --------------------------------------------------------------------- */

/* Replaces ftle_estimator::estimate (ftle_estimator.cpp:7-65): flow map of
 * shape floor(field shape / seed_stride) with spacing field spacing *
 * seed_stride, central-difference Jacobian with the clamped border rule of
 * regular_grid::gradient (regular_grid.hpp:87-108), C = J^T J, FP64 largest
 * eigenvalue and ln(sqrt(lambda)) / |step_size * iterations|. Host arrays;
 * ftle receives product(shape_out) floats (pass NULL to query shape_out). */
int dpa_ftle_estimate(dpa_context* ctx, const dpa_field* field, const float seed_stride[3],
                      uint64_t iterations, float step_size, uint64_t count,
                      const float* original_positions, const float* final_positions,
                      int32_t mapping, float* ftle, uint64_t shape_out[3]);

/* Device-array variant on the given stream (NULL: the context's stream). */
int dpa_ftle_estimate_device(dpa_context* ctx, const dpa_field* field, const float seed_stride[3],
                             uint64_t iterations, float step_size, uint64_t count,
                             const float* device_original_positions,
                             const float* device_final_positions, int32_t mapping,
                             float* device_ftle, uint64_t shape_out[3], void* stream);

#ifdef __cplusplus
}
#endif

#endif
