// pipeline.hpp -- the host pipeline of the advection stage at world size 1.
//
// Mirrors dpa::pipeline::run (source/pipeline.cpp:22-176): read the JSON
// configuration, load the XYZV field, seed, advect in rounds through the C ABI
// of libdpa_b200, save the integral curves and the FTLE field as HDF5 + XDMF,
// and write the benchmark CSV with the reference's record names. The MPI rank
// layer runs at world size 1 (single_rank below).
#pragma once

#include <array>
#include <cstdint>
#include <optional>
#include <string>
#include <vector>

#include "json.hpp"

namespace dpa_host {

// dpa::arguments (include/dpa/types/arguments.hpp:11-29) plus the settings
// this build adds (all optional, all prefixed dpa_b200_).
struct arguments {
  std::string input_dataset_filepath;
  std::string input_dataset_name;
  std::string input_dataset_spacing_name;
  std::optional<std::array<float, 3>> seed_generation_stride;
  std::optional<uint64_t> seed_generation_count;
  std::optional<std::array<uint64_t, 2>> seed_generation_range;
  uint64_t seed_generation_iterations = 0;
  std::optional<std::array<float, 6>> seed_generation_boundaries;  // min xyz, max xyz
  uint64_t particle_advector_particles_per_round = 0;
  std::string particle_advector_load_balancer;
  std::string particle_advector_integrator;
  float particle_advector_step_size = 0.0f;
  bool particle_advector_gather_particles = false;
  bool particle_advector_record = false;
  bool estimate_ftle = false;
  std::string output_dataset_filepath;

  // Build settings.
  std::string storage = "f32";         // dpa_b200_field_storage: f32 | f16 | bf16
  uint64_t seed = 0;                   // dpa_b200_seed: random-seeding PRNG seed
  int device = 0;                      // dpa_b200_device
  std::string ftle_mapping = "reference";  // dpa_b200_ftle_mapping: reference | lattice
  bool morton_order = true;            // dpa_b200_morton_order
};

// argument_parser::parse (source/stages/argument_parser.cpp:10-60).
arguments parse_arguments(const json::value& config);

// The world-size-1 stand-in for the MPI communicator the reference builds
// (domain_partitioner.cpp:7-47): one rank, a 1x1x1 Cartesian grid, no
// neighbours, so every gather, broadcast and all-to-all is the identity.
struct single_rank {
  int rank() const { return 0; }
  int size() const { return 1; }
  void barrier() const {}
};

// Seeds of uniform_seed_generator (uniform_seed_generator.cpp:16-81): the
// lattice exactly as the reference computes it, random seeds from the
// counter-based stream of dpa_seed_random_device.
std::vector<float> lattice_seeds(std::array<float, 3> offset, std::array<float, 3> size,
                                 const std::array<float, 3>& stride,
                                 const std::optional<std::array<float, 6>>& aabb,
                                 std::array<uint64_t, 3>* shape_out);
std::vector<float> random_seeds(std::array<float, 3> offset, std::array<float, 3> size,
                                uint64_t count, uint64_t seed,
                                const std::optional<std::array<float, 6>>& aabb);
uint64_t random_count(uint64_t lo, uint64_t hi, uint64_t seed);

// Runs the whole pipeline for one configuration file; returns 0 on success
// and prints the failure otherwise.
int run(const std::string& config_path);

}  // namespace dpa_host
