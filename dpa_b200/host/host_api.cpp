// host_api.cpp -- the C entry points of dpa_host.h.
#include <cstring>
#include <string>

#include "dpa_host.h"
#include "hdf5.hpp"
#include "pipeline.hpp"

namespace {

thread_local std::string g_error;

template <class F>
int guarded(F&& body) {
  try {
    g_error.clear();
    body();
    return 0;
  } catch (const std::exception& e) {
    g_error = e.what();
    return 1;
  } catch (...) {
    g_error = "unknown error";
    return 1;
  }
}

std::optional<std::array<float, 6>> box(const float* aabb) {
  if (!aabb) return std::nullopt;
  std::array<float, 6> b;
  std::memcpy(b.data(), aabb, sizeof(b));
  return b;
}

}  // namespace

extern "C" {

const char* dpa_host_last_error(void) { return g_error.c_str(); }

int dpa_host_run_pipeline(const char* config_path) {
  if (!config_path) return 1;
  return dpa_host::run(config_path);
}

int dpa_host_h5_write_field(const char* path, const char* dataset, const char* spacing_attribute,
                            const float* xyzv, const uint64_t shape[3], const float spacing[3]) {
  return guarded([&] {
    dpa_host::h5::writer w(path);
    w.add_dataset(dataset, dpa_host::h5::element::f32, {shape[0], shape[1], shape[2], 3}, xyzv);
    w.add_root_attribute(spacing_attribute, dpa_host::h5::element::f32, {3}, spacing);
    w.close();
  });
}

int dpa_host_h5_write_datasets(const char* path, uint64_t count, const char* const* names,
                               const int32_t* kinds, const uint64_t* lengths,
                               const void* const* data) {
  return guarded([&] {
    dpa_host::h5::writer w(path);
    for (uint64_t i = 0; i < count; ++i) {
      dpa_host::h5::element e = dpa_host::h5::element::f32;
      switch (kinds[i]) {
        case 0: e = dpa_host::h5::element::f32; break;
        case 1: e = dpa_host::h5::element::u8; break;
        case 2: e = dpa_host::h5::element::u32; break;
        case 3: e = dpa_host::h5::element::u64; break;
        default: throw std::runtime_error("unknown element kind");
      }
      w.add_dataset(names[i], e, {lengths[i]}, data[i]);
    }
    w.close();
  });
}

int dpa_host_h5_names(const char* path, char* buffer, uint64_t size) {
  return guarded([&] {
    dpa_host::h5::reader r(path);
    std::string all;
    for (const auto& n : r.names()) all += n + "\n";
    if (buffer && size) {
      const size_t n = std::min<size_t>(all.size(), size_t(size - 1));
      std::memcpy(buffer, all.data(), n);
      buffer[n] = 0;
    }
  });
}

int dpa_host_h5_info(const char* path, const char* dataset, uint64_t dims[8], int32_t* rank,
                     int32_t* type_class, int32_t* type_size) {
  return guarded([&] {
    dpa_host::h5::reader r(path);
    const auto d = r.info(dataset);
    if (d.dims.size() > 8) throw std::runtime_error("rank above 8");
    for (size_t i = 0; i < d.dims.size(); ++i) dims[i] = d.dims[i];
    *rank = int32_t(d.dims.size());
    *type_class = d.type_class;
    *type_size = int32_t(d.type_size);
  });
}

int dpa_host_h5_read(const char* path, const char* dataset, int32_t kind, void* out,
                     uint64_t elements) {
  return guarded([&] {
    dpa_host::h5::reader r(path);
    const auto e = kind == 0   ? dpa_host::h5::element::f64
                   : kind == 1 ? dpa_host::h5::element::f32
                               : dpa_host::h5::element::u64;
    r.read(dataset, e, out, elements);
  });
}

int dpa_host_h5_attribute(const char* path, const char* name, double* out, uint64_t capacity,
                          uint64_t* count) {
  return guarded([&] {
    dpa_host::h5::reader r(path);
    const auto v = r.root_attribute(name);
    *count = v.size();
    for (size_t i = 0; i < v.size() && i < capacity; ++i) out[i] = v[i];
  });
}

uint64_t dpa_host_lattice_seeds(const float offset[3], const float size[3], const float stride[3],
                                const float* aabb, float* out, uint64_t capacity) {
  const auto s = dpa_host::lattice_seeds({offset[0], offset[1], offset[2]},
                                         {size[0], size[1], size[2]},
                                         {stride[0], stride[1], stride[2]}, box(aabb), nullptr);
  const uint64_t n = s.size() / 3;
  if (out) std::memcpy(out, s.data(), sizeof(float) * 3 * std::min(n, capacity));
  return n;
}

uint64_t dpa_host_random_seeds(const float offset[3], const float size[3], uint64_t count,
                               uint64_t seed, const float* aabb, float* out) {
  const auto s = dpa_host::random_seeds({offset[0], offset[1], offset[2]},
                                        {size[0], size[1], size[2]}, count, seed, box(aabb));
  if (out && !s.empty()) std::memcpy(out, s.data(), sizeof(float) * s.size());
  return s.size() / 3;
}

uint64_t dpa_host_random_count(uint64_t lo, uint64_t hi, uint64_t seed) {
  return dpa_host::random_count(lo, hi, seed);
}

}  // extern "C"
