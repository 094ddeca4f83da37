// pipeline.cpp -- see pipeline.hpp.
#include "pipeline.hpp"

#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <filesystem>
#include <fstream>
#include <functional>
#include <iostream>
#include <limits>
#include <memory>
#include <mutex>
#include <sstream>
#include <stdexcept>
#include <thread>

#include "dpa_b200.h"
#include "hdf5.hpp"

namespace dpa_host {

namespace {

std::array<float, 3> float3(const json::value& v) {
  return {v[0].as_float(), v[1].as_float(), v[2].as_float()};
}

// "Due to limitations of JSON, 64 bit integers are stored as strings"
// (argument_parser.cpp:27): boost::lexical_cast<std::size_t> of the string.
uint64_t u64_string(const json::value& v, const char* key) {
  const std::string& s = v.as_string();
  if (s.empty() || s.find_first_not_of("0123456789") != std::string::npos)
    throw std::runtime_error(std::string("config: ") + key + " is not an unsigned integer string");
  errno = 0;
  char* end = nullptr;
  const unsigned long long r = std::strtoull(s.c_str(), &end, 10);
  if (errno == ERANGE) throw std::runtime_error(std::string("config: ") + key + " out of range");
  return uint64_t(r);
}

uint64_t splitmix64(uint64_t x) {
  x += 0x9e3779b97f4a7c15ull;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
  return x ^ (x >> 31);
}

// Clips [offset, offset + size] to the box as Eigen::AlignedBox::intersection
// does (uniform_seed_generator.cpp:18-27); false when the result is empty.
bool clip(std::array<float, 3>& offset, std::array<float, 3>& size,
          const std::optional<std::array<float, 6>>& aabb) {
  if (!aabb) return true;
  std::array<float, 3> lo, hi;
  for (int i = 0; i < 3; ++i) {
    lo[i] = std::max((*aabb)[i], offset[i]);
    hi[i] = std::min((*aabb)[3 + i], offset[i] + size[i]);
    if (lo[i] > hi[i]) return false;
  }
  for (int i = 0; i < 3; ++i) {
    offset[i] = lo[i];
    size[i] = hi[i] - lo[i];
  }
  return true;
}

// session_recorder / mpi_session (include/dpa/benchmark/benchmark.hpp:19-200):
// named float millisecond values in order of first use, one iteration.
class recorder {
 public:
  void set(const std::string& name, float value) {
    for (auto& r : records_)
      if (r.first == name) {
        r.second = value;
        return;
      }
    records_.push_back({name, value});
  }
  void record(const std::string& name, const std::function<void()>& body) {
    const auto start = std::chrono::high_resolution_clock::now();
    body();
    const auto end = std::chrono::high_resolution_clock::now();
    set(name, std::chrono::duration<float, std::milli>(end - start).count());
  }
  void to_csv(const std::string& path) const {
    std::ofstream out(path);
    if (!out) throw std::runtime_error("cannot write " + path);
    out.precision(std::numeric_limits<float>::max_digits10);
    out << "rank,name,iteration 0,\n";
    for (const auto& r : records_) out << 0 << "," << r.first << "," << r.second << ",\n";
  }

 private:
  std::vector<std::pair<std::string, float>> records_;
};

// XDMF bodies with the structure of include/dpa/utility/xdmf.hpp.
const char* kXdmfHeader =
    "<?xml version =\"1.0\" ?>\n<!DOCTYPE xdmf SYSTEM \"Xdmf.dtd\" []>\n<Xdmf Version=\"2.0\">\n"
    "  <Domain>\n";
const char* kXdmfFooter = "\n  </Domain>\n</Xdmf>\n";

std::string xdmf_polyline(const std::string& file, uint64_t round, uint64_t vertices,
                          uint64_t indices, bool index64) {
  std::ostringstream s;
  s << "\n    <Grid Name=\"grid_" << round << "\">\n\n"
    << "      <Topology TopologyType=\"Polyline\" NodesPerElement=\"2\" NumberOfElements=\""
    << indices / 2 << "\">\n"
    << "        <DataItem Dimensions=\"" << indices << "\" NumberType=\"UInt\" Precision=\""
    << (index64 ? 8 : 4) << "\" Format=\"HDF\">\n"
    << "          " << file << ":/indices_" << round << "\n"
    << "        </DataItem>\n      </Topology>\n\n"
    << "      <Geometry GeometryType=\"XYZ\">\n"
    << "        <DataItem Dimensions=\"" << 3 * vertices
    << "\" NumberType=\"Float\" Precision=\"4\" Format=\"HDF\">\n"
    << "          " << file << ":/vertices_" << round << "\n"
    << "        </DataItem>\n      </Geometry>\n\n"
    << "      <Attribute Name=\"Colors\" AttributeType=\"Scalar\" Center=\"Node\">\n"
    << "        <DataItem Dimensions=\"" << vertices
    << "\" NumberType=\"Float\" Precision=\"4\" Format=\"HDF\">\n"
    << "          " << file << ":/colors_" << round << "\n"
    << "        </DataItem>\n      </Attribute>\n\n    </Grid>\n";
  return s.str();
}

std::string xdmf_volume(const std::string& file, const std::array<uint64_t, 3>& shape,
                        const std::array<float, 3>& origin, const std::array<float, 3>& spacing) {
  std::ostringstream s;
  const std::string size = std::to_string(shape[0]) + " " + std::to_string(shape[1]) + " " +
                           std::to_string(shape[2]);
  s << "\n    <Grid Name=\"Grid\" GridType=\"Uniform\">\n"
    << "      <Topology TopologyType=\"3DCoRectMesh\" NumberOfElements=\"" << size << "\"/>\n"
    << "      <Geometry GeometryType=\"ORIGIN_DXDYDZ\">\n"
    << "        <DataItem Dimensions=\"3\" NumberType=\"Float\" Precision=\"4\" Format=\"XML\">\n"
    << "          " << std::to_string(origin[0]) << " " << std::to_string(origin[1]) << " "
    << std::to_string(origin[2]) << "\n        </DataItem>\n"
    << "        <DataItem Dimensions=\"3\" NumberType=\"Float\" Precision=\"4\" Format=\"XML\">\n"
    << "          " << std::to_string(spacing[0]) << " " << std::to_string(spacing[1]) << " "
    << std::to_string(spacing[2]) << "\n        </DataItem>\n      </Geometry>\n"
    << "      <Attribute Name=\"Volume\" AttributeType=\"Scalar\" Center=\"Node\">\n"
    << "        <DataItem Dimensions=\"" << size
    << "\" NumberType=\"Float\" Precision=\"4\" Format=\"HDF\">\n"
    << "          " << file << ":/data\n        </DataItem>\n      </Attribute>\n    </Grid>\n";
  return s.str();
}

void check(int status, dpa_context* ctx, const char* what) {
  if (status != DPA_OK)
    throw std::runtime_error(std::string(what) + ": " + (ctx ? dpa_last_error(ctx) : "failed"));
}

// One round's curve, assembled from the library's chunks.
struct round_curve {
  std::vector<float> vertices, colors;
  std::vector<uint32_t> indices32;
  std::vector<uint64_t> indices64;
  bool index64 = false;
};

// Writes each round's curve (integral_curve_saver.cpp:44-79: vertices_i,
// colors_i, indices_i) on a background thread while the next round advects.
// At most two finished rounds wait in memory; push() blocks beyond that.
class round_writer {
 public:
  round_writer(h5::writer& out, std::string file, bool index64)
      : out_(out), file_(std::move(file)), index64_(index64), thread_([this] { run(); }) {}
  ~round_writer() {
    if (thread_.joinable()) {
      {
        std::lock_guard<std::mutex> lock(mutex_);
        done_ = true;
      }
      wake_.notify_all();
      thread_.join();
    }
  }

  // Hands a round's curve over; returns the milliseconds spent waiting for
  // room (the writer falling behind the rounds).
  float push(uint64_t round, round_curve&& curve) {
    const auto t0 = std::chrono::high_resolution_clock::now();
    std::unique_lock<std::mutex> lock(mutex_);
    room_.wait(lock, [&] { return queue_.size() < 2 || failed_; });
    if (failed_) throw std::runtime_error(error_);
    queue_.emplace_back(round, std::move(curve));
    wake_.notify_all();
    return std::chrono::duration<float, std::milli>(std::chrono::high_resolution_clock::now() - t0)
        .count();
  }

  // Waits for every round to be written; returns the XDMF grids.
  std::string finish() {
    {
      std::lock_guard<std::mutex> lock(mutex_);
      done_ = true;
    }
    wake_.notify_all();
    thread_.join();
    if (failed_) throw std::runtime_error(error_);
    return xdmf_;
  }

 private:
  void run() {
    while (true) {
      std::pair<uint64_t, round_curve> item;
      {
        std::unique_lock<std::mutex> lock(mutex_);
        wake_.wait(lock, [&] { return !queue_.empty() || done_; });
        if (queue_.empty()) return;
        item = std::move(queue_.front());
      }
      try {
        const round_curve& c = item.second;
        const uint64_t v = c.vertices.size() / 3;
        const uint64_t ni = index64_ ? c.indices64.size() : c.indices32.size();
        const std::string r = std::to_string(item.first);
        out_.add_dataset("vertices_" + r, h5::element::f32, {3 * v}, c.vertices.data());
        out_.add_dataset("colors_" + r, h5::element::f32, {v}, c.colors.data());
        if (index64_)
          out_.add_dataset("indices_" + r, h5::element::u64, {ni}, c.indices64.data());
        else
          out_.add_dataset("indices_" + r, h5::element::u32, {ni}, c.indices32.data());
        xdmf_ += xdmf_polyline(file_, item.first, v, ni, index64_);
      } catch (const std::exception& e) {
        std::lock_guard<std::mutex> lock(mutex_);
        failed_ = true;
        error_ = e.what();
      }
      std::lock_guard<std::mutex> lock(mutex_);
      queue_.pop_front();
      room_.notify_all();
      if (failed_) return;
    }
  }

  h5::writer& out_;
  const std::string file_;
  const bool index64_;
  std::mutex mutex_;
  std::condition_variable wake_, room_;
  std::deque<std::pair<uint64_t, round_curve>> queue_;
  bool done_ = false, failed_ = false;
  std::string error_, xdmf_;
  std::thread thread_;
};

int collect_chunk(void* user, const dpa_curve_chunk* c) {
  auto* r = static_cast<round_curve*>(user);
  r->vertices.insert(r->vertices.end(), c->vertices, c->vertices + 3 * c->vertex_count);
  if (c->colors) r->colors.insert(r->colors.end(), c->colors, c->colors + c->vertex_count);
  if (r->index64) {
    const auto* i = static_cast<const uint64_t*>(c->indices);
    r->indices64.insert(r->indices64.end(), i, i + c->index_count);
  } else {
    const auto* i = static_cast<const uint32_t*>(c->indices);
    r->indices32.insert(r->indices32.end(), i, i + c->index_count);
  }
  return 0;
}

}  // namespace

arguments parse_arguments(const json::value& j) {
  arguments a;
  a.input_dataset_filepath = j["input_dataset_filepath"].as_string();
  a.input_dataset_name = j["input_dataset_name"].as_string();
  a.input_dataset_spacing_name = j["input_dataset_spacing_name"].as_string();
  a.particle_advector_load_balancer = j["particle_advector_load_balancer"].as_string();
  a.particle_advector_integrator = j["particle_advector_integrator"].as_string();
  a.particle_advector_step_size = j["particle_advector_step_size"].as_float();
  a.particle_advector_gather_particles = j["particle_advector_gather_particles"].as_bool();
  a.particle_advector_record = j["particle_advector_record"].as_bool();
  a.estimate_ftle = j["estimate_ftle"].as_bool();
  a.output_dataset_filepath = j["output_dataset_filepath"].as_string();
  a.seed_generation_iterations = u64_string(j["seed_generation_iterations"], "seed_generation_iterations");
  a.particle_advector_particles_per_round =
      u64_string(j["particle_advector_particles_per_round"], "particle_advector_particles_per_round");
  if (j.contains("seed_generation_stride")) a.seed_generation_stride = float3(j["seed_generation_stride"]);
  if (j.contains("seed_generation_count"))
    a.seed_generation_count = u64_string(j["seed_generation_count"], "seed_generation_count");
  if (j.contains("seed_generation_range")) {
    const auto& r = j["seed_generation_range"];
    a.seed_generation_range = std::array<uint64_t, 2>{u64_string(r[0], "seed_generation_range"),
                                                      u64_string(r[1], "seed_generation_range")};
  }
  if (j.contains("seed_generation_boundaries")) {
    const auto& b = j["seed_generation_boundaries"];
    const auto lo = float3(b["minimum"]);
    const auto hi = float3(b["maximum"]);
    a.seed_generation_boundaries = std::array<float, 6>{lo[0], lo[1], lo[2], hi[0], hi[1], hi[2]};
  }
  if (j.contains("dpa_b200_field_storage")) a.storage = j["dpa_b200_field_storage"].as_string();
  if (j.contains("dpa_b200_seed")) a.seed = u64_string(j["dpa_b200_seed"], "dpa_b200_seed");
  if (j.contains("dpa_b200_device")) a.device = int(j["dpa_b200_device"].as_double());
  if (j.contains("dpa_b200_ftle_mapping")) a.ftle_mapping = j["dpa_b200_ftle_mapping"].as_string();
  if (j.contains("dpa_b200_morton_order")) a.morton_order = j["dpa_b200_morton_order"].as_bool();
  return a;
}

std::vector<float> lattice_seeds(std::array<float, 3> offset, std::array<float, 3> size,
                                 const std::array<float, 3>& stride,
                                 const std::optional<std::array<float, 6>>& aabb,
                                 std::array<uint64_t, 3>* shape_out) {
  std::array<uint64_t, 3> shape = {0, 0, 0};
  std::vector<float> out;
  if (clip(offset, size, aabb)) {
    for (int i = 0; i < 3; ++i) {
      const float q = size[i] / stride[i];
      shape[i] = q > 0.0f ? uint64_t(q) : 0;
    }
    const uint64_t count = shape[0] * shape[1] * shape[2];
    out.resize(3 * count);
    for (uint64_t index = 0; index < count; ++index) {
      uint64_t rest = index, sub[3];
      for (int i = 2; i >= 0; --i) {
        sub[i] = rest % shape[i];
        rest /= shape[i];
      }
      for (int i = 0; i < 3; ++i) out[3 * index + i] = offset[i] + stride[i] * float(sub[i]);
    }
  }
  if (shape_out) *shape_out = shape;
  return out;
}

std::vector<float> random_seeds(std::array<float, 3> offset, std::array<float, 3> size,
                                uint64_t count, uint64_t seed,
                                const std::optional<std::array<float, 6>>& aabb) {
  if (!clip(offset, size, aabb)) return {};
  std::vector<float> out(3 * count);
  const uint64_t key = splitmix64(seed);
  for (uint64_t t = 0; t < count; ++t)
    for (int a = 0; a < 3; ++a) {
      const uint64_t r = splitmix64(key ^ (3 * t + uint64_t(a)));
      const float u = float(uint32_t(r >> 40)) * 0x1p-24f;
      out[3 * t + a] = offset[a] + size[a] * u;
    }
  return out;
}

uint64_t random_count(uint64_t lo, uint64_t hi, uint64_t seed) {
  if (hi < lo) std::swap(lo, hi);
  const uint64_t span = hi - lo + 1;
  const uint64_t r = splitmix64(splitmix64(seed) ^ 0x72616e6765ull);
  return span == 0 ? r : lo + r % span;
}

int run(const std::string& config_path) {
  dpa_context* ctx = nullptr;
  dpa_field* field = nullptr;
  try {
    single_rank world;
    char host[256] = {0};
    gethostname(host, sizeof(host) - 1);
    std::cout << "Started pipeline on " << host << "\n";
    const arguments args = parse_arguments(json::value::parse_file(config_path));

    int32_t integrator = 0;
    if (dpa_integrator_from_name(args.particle_advector_integrator.c_str(), &integrator) != DPA_OK)
      throw std::runtime_error("unknown integrator " + args.particle_advector_integrator);
    int32_t storage = DPA_STORAGE_F32;
    if (args.storage == "f16") storage = DPA_STORAGE_F16;
    else if (args.storage == "bf16") storage = DPA_STORAGE_BF16;
    else if (args.storage == "f32_edges") storage = DPA_STORAGE_F32_EDGES;
    else if (args.storage != "f32") throw std::runtime_error("unknown field storage " + args.storage);
    if (args.particle_advector_particles_per_round == 0)
      throw std::runtime_error("particle_advector_particles_per_round must be positive");

    recorder rec;
    std::cout << "domain_partitioning\n";
    h5::reader input(args.input_dataset_filepath);
    const h5::dataset_info info = input.info(args.input_dataset_name);
    if (info.dims.size() != 4 || info.dims[3] != 3)
      throw std::runtime_error("input dataset must be [X][Y][Z][3]");
    const std::array<uint64_t, 3> shape = {info.dims[0], info.dims[1], info.dims[2]};

    std::cout << "data_loading\n";
    std::vector<float> data(info.elements());
    input.read(args.input_dataset_name, h5::element::f32, data.data(), data.size());
    const std::vector<double> spacing_attr = input.root_attribute(args.input_dataset_spacing_name);
    if (spacing_attr.size() != 3) throw std::runtime_error("spacing attribute must hold 3 values");
    const std::array<float, 3> spacing = {float(spacing_attr[0]), float(spacing_attr[1]),
                                          float(spacing_attr[2])};
    // World size 1: the ghosted block is the whole grid (domain_partitioner.cpp:95-117).
    std::array<float, 3> field_offset, block_size;
    for (int i = 0; i < 3; ++i) {
      field_offset[i] = 0.0f * spacing[i];
      block_size[i] = spacing[i] * float(shape[i]);
    }
    check(dpa_context_create(args.device, &ctx), ctx, "dpa_context_create");
    check(dpa_field_create(ctx, data.data(), shape.data(), field_offset.data(), spacing.data(),
                           storage, &field),
          ctx, "dpa_field_create");
    data.clear();
    data.shrink_to_fit();

    std::cout << "seed_generation\n";
    std::vector<float> positions;
    std::array<uint64_t, 3> lattice_shape = {0, 0, 0};
    if (args.seed_generation_stride) {
      std::array<float, 3> stride;
      for (int i = 0; i < 3; ++i) stride[i] = spacing[i] * (*args.seed_generation_stride)[i];
      positions = lattice_seeds(field_offset, block_size, stride, args.seed_generation_boundaries,
                                &lattice_shape);
    } else if (args.seed_generation_count) {
      positions = random_seeds(field_offset, block_size, *args.seed_generation_count, args.seed,
                               args.seed_generation_boundaries);
    } else if (args.seed_generation_range) {
      const uint64_t n = random_count((*args.seed_generation_range)[0],
                                      (*args.seed_generation_range)[1], args.seed);
      positions = random_seeds(field_offset, block_size, n, args.seed,
                               args.seed_generation_boundaries);
    }
    const uint64_t total = positions.size() / 3;
    const std::vector<float> original = positions;
    std::vector<uint64_t> remaining(total, args.seed_generation_iterations);
    std::vector<uint8_t> termination(total, 0);

    std::cout << "particle_advection\n";
    // pipeline.cpp:155: particles_per_round * iterations > UINT32_MAX.
    const bool index64 = (unsigned __int128)args.particle_advector_particles_per_round *
                             args.seed_generation_iterations >
                         std::numeric_limits<uint32_t>::max();
    dpa_advect_options options{};
    options.integrator = integrator;
    options.step_size = args.particle_advector_step_size;
    options.record = args.particle_advector_record ? 1 : 0;
    options.index64 = index64 ? 1 : 0;
    options.colors = 1;
    options.morton_order = args.morton_order ? 1 : 0;

    const std::string curve_path =
        std::filesystem::path(args.output_dataset_filepath).replace_extension(".rank_0.h5").string();
    std::unique_ptr<h5::writer> curves;
    std::unique_ptr<round_writer> writer;
    std::string xdmf_bodies;
    const std::string curve_file = std::filesystem::path(curve_path).filename().string();
    if (args.particle_advector_record) {
      curves = std::make_unique<h5::writer>(curve_path);
      writer = std::make_unique<round_writer>(*curves, curve_file, index64);
    }

    uint64_t active = total;
    uint64_t rounds = 0;
    bool complete = false;
    float io_ms = 0.0f;
    world.barrier();
    const auto loop_start = std::chrono::high_resolution_clock::now();
    {
      while (!complete) {
        const std::string prefix = "round." + std::to_string(rounds);
        round_curve curve;
        curve.index64 = index64;
        rec.record(prefix + ".time", [&]() {
          rec.record(prefix + ".load_balancing_time",
                     [&]() { rec.set(prefix + ".load", float(active)); });
          rec.record(prefix + ".advection_time", [&]() {
            const uint64_t count = std::min(args.particle_advector_particles_per_round, active);
            const uint64_t lo = active - count;
            check(dpa_advect_round(ctx, field, &options, count, positions.data() + 3 * lo,
                                   remaining.data() + lo, termination.data() + lo,
                                   options.record ? collect_chunk : nullptr, &curve),
                  ctx, "dpa_advect_round");
            active = lo;
          });
          rec.record(prefix + ".communication_time", [&]() { complete = active == 0; });
        });
        // The round's curve is written in the background while the next
        // round advects.
        if (writer && !curve.vertices.empty()) io_ms += writer->push(rounds, std::move(curve));
        ++rounds;
      }
    }
    // total_time covers the round loop as in the reference (pipeline.cpp:98);
    // the curve writes overlap the rounds, and any wait for the writer is
    // taken out.
    const float loop_ms = std::chrono::duration<float, std::milli>(
                              std::chrono::high_resolution_clock::now() - loop_start)
                              .count();
    rec.set("total_time", loop_ms - io_ms);
    world.barrier();

    std::cout << "gather_particles\n";   // identity at world size 1
    std::cout << "index_generation\n";   // fused into the round's emission
    std::cout << "color_generation\n";
    std::cout << "save_integral_curves\n";
    if (curves) {
      xdmf_bodies = writer->finish();
      curves->close();
      if (!xdmf_bodies.empty()) {
        std::ofstream x(curve_path + ".xdmf");
        x << kXdmfHeader << xdmf_bodies << kXdmfFooter;
      }
    }

    std::cout << "estimate_ftle\n";
    if (args.estimate_ftle) {
      if (!args.seed_generation_stride)
        throw std::runtime_error("estimate_ftle needs seed_generation_stride");
      uint64_t ftle_shape[3] = {0, 0, 0};
      const int32_t mapping =
          args.ftle_mapping == "lattice" ? DPA_FTLE_MAPPING_LATTICE : DPA_FTLE_MAPPING_REFERENCE;
      check(dpa_ftle_estimate(ctx, field, args.seed_generation_stride->data(),
                              args.seed_generation_iterations, args.particle_advector_step_size,
                              total, original.data(), positions.data(), mapping, nullptr,
                              ftle_shape),
            ctx, "dpa_ftle_estimate");
      std::vector<float> ftle(ftle_shape[0] * ftle_shape[1] * ftle_shape[2]);
      check(dpa_ftle_estimate(ctx, field, args.seed_generation_stride->data(),
                              args.seed_generation_iterations, args.particle_advector_step_size,
                              total, original.data(), positions.data(), mapping, ftle.data(),
                              ftle_shape),
            ctx, "dpa_ftle_estimate");
      std::cout << "save_ftle_field\n";
      if (!ftle.empty()) {
        const std::string grid_path = std::filesystem::path(args.output_dataset_filepath)
                                          .replace_extension(".rank_0_grid.h5")
                                          .string();
        h5::writer w(grid_path);
        w.add_dataset("data", h5::element::f32, {ftle_shape[0], ftle_shape[1], ftle_shape[2]},
                      ftle.data());
        w.close();
        std::array<float, 3> ftle_spacing;
        for (int i = 0; i < 3; ++i) ftle_spacing[i] = spacing[i] * (*args.seed_generation_stride)[i];
        std::ofstream x(grid_path + ".xdmf");
        x << kXdmfHeader
          << xdmf_volume(std::filesystem::path(grid_path).filename().string(),
                         {ftle_shape[0], ftle_shape[1], ftle_shape[2]}, field_offset, ftle_spacing)
          << kXdmfFooter;
      }
    } else {
      std::cout << "save_ftle_field\n";
    }

    rec.to_csv(args.output_dataset_filepath + ".benchmark.csv");
    dpa_field_destroy(ctx, field);
    dpa_context_destroy(ctx);
    return 0;
  } catch (const std::exception& e) {
    std::cerr << "dpa_pipeline: " << e.what() << "\n";
    if (field) dpa_field_destroy(ctx, field);
    if (ctx) dpa_context_destroy(ctx);
    return 1;
  }
}

}  // namespace dpa_host
