/*
 * dpa_host.h -- C entry points of the host library (libdpa_host.so): the
 * pipeline driver and its HDF5, seeding and configuration pieces, for
 * bindings and tests. The GPU compute lives behind include/dpa_b200.h.
 * Every function returns 0 on success; dpa_host_last_error() describes a
 * failure of the calling thread's last call.
 */
#ifndef DPA_HOST_H
#define DPA_HOST_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

const char* dpa_host_last_error(void);

/* Runs the whole pipeline on a JSON configuration (dpa_pipeline config.json). */
int dpa_host_run_pipeline(const char* config_path);

/* Writes an XYZV input field: dataset `dataset` float [n0][n1][n2][3] and a
 * root attribute `spacing_attribute` float[3], as the reference's loader
 * expects (regular_grid_loader.cpp:34-88). */
int dpa_host_h5_write_field(const char* path, const char* dataset, const char* spacing_attribute,
                            const float* xyzv, const uint64_t shape[3], const float spacing[3]);

/* Writes `count` one-dimensional datasets into a new file: names[i] with
 * lengths[i] elements of kinds[i] (0 float32, 1 uint8, 2 uint32, 3 uint64). */
int dpa_host_h5_write_datasets(const char* path, uint64_t count, const char* const* names,
                               const int32_t* kinds, const uint64_t* lengths,
                               const void* const* data);

/* Root group member names, '\n'-separated, into buffer (truncated to size). */
int dpa_host_h5_names(const char* path, char* buffer, uint64_t size);

/* Shape (rank <= 8), class (0 integer, 1 float) and element size. */
int dpa_host_h5_info(const char* path, const char* dataset, uint64_t dims[8], int32_t* rank,
                     int32_t* type_class, int32_t* type_size);

/* Reads a dataset converted to double (kind 0), float (kind 1) or uint64 (kind 2). */
int dpa_host_h5_read(const char* path, const char* dataset, int32_t kind, void* out,
                     uint64_t elements);

/* Reads a root attribute as doubles; *count receives its element count. */
int dpa_host_h5_attribute(const char* path, const char* name, double* out, uint64_t capacity,
                          uint64_t* count);

/* Seeds of the host pipeline (see pipeline.hpp); aabb is NULL or min xyz, max xyz. */
uint64_t dpa_host_lattice_seeds(const float offset[3], const float size[3], const float stride[3],
                                const float* aabb, float* out, uint64_t capacity);
uint64_t dpa_host_random_seeds(const float offset[3], const float size[3], uint64_t count,
                               uint64_t seed, const float* aabb, float* out);
uint64_t dpa_host_random_count(uint64_t lo, uint64_t hi, uint64_t seed);

#ifdef __cplusplus
}
#endif

#endif
