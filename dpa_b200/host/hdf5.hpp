// hdf5.hpp -- a minimal HDF5 reader and writer for the pipeline's files.
//
// The reference links the HDF5 C library (regular_grid_loader.cpp,
// integral_curve_saver.cpp, regular_grid_saver.cpp); it is not available
// here, so this module writes and reads the subset of the HDF5 file format
// those files use, from the published format specification:
//   * superblock version 0, 8-byte offsets and lengths;
//   * one root group held as a symbol table (v1 B-tree, local heap, symbol
//     table node), the layout the HDF5 library writes by default;
//   * datasets of little-endian IEEE floats or unsigned integers, any rank,
//     contiguous storage, object header version 1;
//   * attributes of the root group (the reference's `spacing`).
// The reader also accepts layout messages versions 1 to 3, object header
// continuation blocks, multi-level group B-trees and a user block before the
// superblock; chunked or compressed datasets are reported as unsupported.
#pragma once

#include <cstdint>
#include <cstdio>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

namespace dpa_host {
namespace h5 {

struct error : std::runtime_error {
  using std::runtime_error::runtime_error;
};

// Element types the module can write: H5T_NATIVE_FLOAT, H5T_NATIVE_DOUBLE,
// H5T_NATIVE_UINT8, H5T_NATIVE_UINT32, H5T_NATIVE_UINT64 on little-endian hosts.
enum class element { f32, f64, u8, u32, u64 };

size_t element_size(element e);

// Streaming writer: raw data goes to the file as each dataset is added; the
// group and object headers are written by close(). Dataset names of the root
// group must be unique.
class writer {
 public:
  explicit writer(const std::string& path);
  ~writer();
  writer(const writer&) = delete;
  writer& operator=(const writer&) = delete;

  void add_dataset(const std::string& name, element type, const std::vector<uint64_t>& dims,
                   const void* data);
  void add_root_attribute(const std::string& name, element type,
                          const std::vector<uint64_t>& dims, const void* data);
  void close();

 private:
  struct item {
    std::string name;
    element type;
    std::vector<uint64_t> dims;
    uint64_t address;  // raw data (datasets)
    std::vector<uint8_t> value;  // attributes
  };
  uint64_t append(const void* data, uint64_t bytes);
  void write_at(uint64_t address, const void* data, uint64_t bytes);

  std::FILE* file_ = nullptr;
  std::string path_;
  uint64_t end_ = 0;
  std::vector<item> datasets_;
  std::vector<item> attributes_;
};

struct dataset_info {
  std::vector<uint64_t> dims;
  int type_class = -1;   // 0 fixed-point, 1 floating-point
  uint32_t type_size = 0;
  bool is_signed = false;
  bool big_endian = false;
  uint64_t address = 0;  // contiguous raw data
  uint64_t bytes = 0;
  uint64_t elements() const;
};

class reader {
 public:
  explicit reader(const std::string& path);
  ~reader();
  reader(const reader&) = delete;
  reader& operator=(const reader&) = delete;

  std::vector<std::string> names() const;       // root group members
  dataset_info info(const std::string& name) const;
  // Reads a dataset converted to float, double or uint64 (by out_type).
  void read(const std::string& name, element out_type, void* out, uint64_t elements) const;
  std::vector<double> root_attribute(const std::string& name) const;

 private:
  struct message {
    uint16_t type;
    std::vector<uint8_t> data;
  };
  std::vector<uint8_t> bytes_at(uint64_t address, uint64_t count) const;
  std::vector<message> object_messages(uint64_t address) const;
  void walk_group_btree(uint64_t address, const std::vector<uint8_t>& heap,
                        std::map<std::string, uint64_t>& out, int depth) const;

  std::FILE* file_ = nullptr;
  uint64_t base_ = 0;       // absolute position of the superblock (user block size)
  uint64_t root_header_ = 0;
  std::map<std::string, uint64_t> members_;
};

}  // namespace h5
}  // namespace dpa_host
