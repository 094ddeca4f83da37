// hdf5.cpp -- see hdf5.hpp. Structures follow the HDF5 file format
// specification (superblock v0, object header v1, symbol-table groups).
#include "hdf5.hpp"

#include <algorithm>
#include <cstring>
#include <numeric>

namespace dpa_host {
namespace h5 {

namespace {

constexpr uint64_t kUndefined = ~0ull;
constexpr uint8_t kSignature[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
constexpr uint64_t kSuperblockBytes = 96;
constexpr uint16_t kInternalK = 16;  // group B-tree nodes hold up to 2K children

// Object header message types.
constexpr uint16_t kNil = 0x0000;
constexpr uint16_t kDataspace = 0x0001;
constexpr uint16_t kLinkInfo = 0x0002;
constexpr uint16_t kDatatype = 0x0003;
constexpr uint16_t kFillValue = 0x0005;
constexpr uint16_t kLink = 0x0006;
constexpr uint16_t kLayout = 0x0008;
constexpr uint16_t kAttribute = 0x000c;
constexpr uint16_t kContinuation = 0x0010;
constexpr uint16_t kSymbolTable = 0x0011;

uint64_t align8(uint64_t n) { return (n + 7) & ~uint64_t(7); }

struct bytes {
  std::vector<uint8_t> b;
  void u8(uint8_t v) { b.push_back(v); }
  void u16(uint16_t v) { for (int i = 0; i < 2; ++i) b.push_back(uint8_t(v >> (8 * i))); }
  void u32(uint32_t v) { for (int i = 0; i < 4; ++i) b.push_back(uint8_t(v >> (8 * i))); }
  void u64(uint64_t v) { for (int i = 0; i < 8; ++i) b.push_back(uint8_t(v >> (8 * i))); }
  void raw(const void* p, size_t n) {
    const uint8_t* c = static_cast<const uint8_t*>(p);
    b.insert(b.end(), c, c + n);
  }
  void zeros(size_t n) { b.insert(b.end(), n, 0); }
  void pad8() { b.resize(align8(b.size()), 0); }
  size_t size() const { return b.size(); }
};

struct cursor {
  const std::vector<uint8_t>& b;
  size_t p = 0;
  void need(size_t n) const {
    if (p + n > b.size()) throw error("HDF5: truncated structure");
  }
  uint8_t u8() { need(1); return b[p++]; }
  uint16_t u16() { need(2); uint16_t v = uint16_t(b[p] | (b[p + 1] << 8)); p += 2; return v; }
  uint32_t u32() {
    need(4);
    uint32_t v = 0;
    for (int i = 3; i >= 0; --i) v = (v << 8) | b[p + i];
    p += 4;
    return v;
  }
  uint64_t u64() {
    need(8);
    uint64_t v = 0;
    for (int i = 7; i >= 0; --i) v = (v << 8) | b[p + i];
    p += 8;
    return v;
  }
  uint64_t uint(int n) {
    need(size_t(n));
    uint64_t v = 0;
    for (int i = n - 1; i >= 0; --i) v = (v << 8) | b[p + i];
    p += size_t(n);
    return v;
  }
  void skip(size_t n) { need(n); p += n; }
};

// Datatype message (version 1) of a little-endian element type.
bytes datatype_message(element e) {
  bytes m;
  switch (e) {
    case element::f32:
    case element::f64: {
      const bool dbl = e == element::f64;
      m.u8(0x11);             // version 1, class 1 (floating point)
      m.u8(0x20);             // little endian, no padding, implied msb mantissa normalization
      m.u8(dbl ? 63 : 31);    // sign bit location
      m.u8(0);
      m.u32(dbl ? 8 : 4);
      m.u16(0);               // bit offset
      m.u16(dbl ? 64 : 32);   // precision
      m.u8(dbl ? 52 : 23);    // exponent location
      m.u8(dbl ? 11 : 8);     // exponent size
      m.u8(0);                // mantissa location
      m.u8(dbl ? 52 : 23);    // mantissa size
      m.u32(dbl ? 1023 : 127);
      break;
    }
    default: {
      const uint32_t size = uint32_t(element_size(e));
      m.u8(0x10);             // version 1, class 0 (fixed point)
      m.u8(0x00);             // little endian, unsigned
      m.u8(0);
      m.u8(0);
      m.u32(size);
      m.u16(0);
      m.u16(uint16_t(8 * size));
      break;
    }
  }
  return m;
}

bytes dataspace_message(const std::vector<uint64_t>& dims) {
  bytes m;
  m.u8(1);  // version 1
  m.u8(uint8_t(dims.size()));
  m.u8(0);  // no maximum dimensions
  m.zeros(5);
  for (uint64_t d : dims) m.u64(d);
  return m;
}

// One version-1 object header holding the given messages.
bytes object_header(const std::vector<std::pair<uint16_t, bytes>>& messages) {
  bytes body;
  for (const auto& [type, data] : messages) {
    bytes d = data;
    d.pad8();
    body.u16(type);
    body.u16(uint16_t(d.size()));
    body.u8(type == kDataspace || type == kAttribute ? 0 : 1);  // constant messages
    body.zeros(3);
    body.raw(d.b.data(), d.size());
  }
  bytes h;
  h.u8(1);
  h.u8(0);
  h.u16(uint16_t(messages.size()));
  h.u32(1);  // reference count
  h.u32(uint32_t(body.size()));
  h.zeros(4);  // messages start 8-byte aligned
  h.raw(body.b.data(), body.size());
  return h;
}

}  // namespace

size_t element_size(element e) {
  switch (e) {
    case element::f32: return 4;
    case element::f64: return 8;
    case element::u8: return 1;
    case element::u32: return 4;
    case element::u64: return 8;
  }
  return 0;
}

uint64_t dataset_info::elements() const {
  uint64_t n = 1;
  for (uint64_t d : dims) n *= d;
  return n;
}

// ---------------------------------------------------------------------------
// writer
// ---------------------------------------------------------------------------

writer::writer(const std::string& path) : path_(path) {
  file_ = std::fopen(path.c_str(), "wb");
  if (!file_) throw error("HDF5: cannot create " + path);
  const std::vector<uint8_t> zeros(kSuperblockBytes, 0);
  append(zeros.data(), zeros.size());
}

writer::~writer() {
  if (file_) {
    try {
      close();
    } catch (...) {
      if (file_) std::fclose(file_);
      file_ = nullptr;
    }
  }
}

uint64_t writer::append(const void* data, uint64_t count) {
  const uint64_t address = end_;
  if (count && std::fwrite(data, 1, count, file_) != count)
    throw error("HDF5: short write to " + path_);
  end_ += count;
  const uint64_t padded = align8(end_);
  if (padded != end_) {
    static const uint8_t pad[8] = {0};
    if (std::fwrite(pad, 1, padded - end_, file_) != padded - end_)
      throw error("HDF5: short write to " + path_);
    end_ = padded;
  }
  return address;
}

void writer::write_at(uint64_t address, const void* data, uint64_t count) {
  if (std::fseek(file_, long(address), SEEK_SET) != 0 ||
      std::fwrite(data, 1, count, file_) != count)
    throw error("HDF5: short write to " + path_);
  std::fseek(file_, 0, SEEK_END);
}

void writer::add_dataset(const std::string& name, element type, const std::vector<uint64_t>& dims,
                         const void* data) {
  if (!file_) throw error("HDF5: writer is closed");
  if (name.empty()) throw error("HDF5: empty dataset name");
  for (const item& d : datasets_)
    if (d.name == name) throw error("HDF5: duplicate dataset " + name);
  uint64_t count = 1;
  for (uint64_t d : dims) count *= d;
  const uint64_t nbytes = count * element_size(type);
  item it{name, type, dims, 0, {}};
  it.address = nbytes ? append(data, nbytes) : kUndefined;
  datasets_.push_back(std::move(it));
}

void writer::add_root_attribute(const std::string& name, element type,
                                const std::vector<uint64_t>& dims, const void* data) {
  uint64_t count = 1;
  for (uint64_t d : dims) count *= d;
  item it{name, type, dims, 0, {}};
  const uint8_t* p = static_cast<const uint8_t*>(data);
  it.value.assign(p, p + count * element_size(type));
  attributes_.push_back(std::move(it));
}

void writer::close() {
  if (!file_) return;
  // Local heap: "" at offset 0, then the member names, then one free block.
  std::vector<const item*> sorted;
  for (const item& d : datasets_) sorted.push_back(&d);
  std::sort(sorted.begin(), sorted.end(),
            [](const item* a, const item* b) { return std::strcmp(a->name.c_str(), b->name.c_str()) < 0; });
  bytes heap_data;
  heap_data.zeros(8);
  std::vector<uint64_t> name_offsets;
  for (const item* d : sorted) {
    name_offsets.push_back(heap_data.size());
    heap_data.raw(d->name.c_str(), d->name.size() + 1);
    heap_data.pad8();
  }
  const uint64_t free_at = heap_data.size();
  heap_data.u64(1);   // next free block: none (the format's end-of-list value)
  heap_data.u64(16);  // this block's size
  const uint64_t heap_data_address = append(heap_data.b.data(), heap_data.size());
  bytes heap;
  heap.raw("HEAP", 4);
  heap.u8(0);
  heap.zeros(3);
  heap.u64(heap_data.size());
  heap.u64(free_at);
  heap.u64(heap_data_address);
  const uint64_t heap_address = append(heap.b.data(), heap.size());

  // Dataset object headers.
  std::vector<uint64_t> headers;
  for (const item* d : sorted) {
    uint64_t nbytes = element_size(d->type);
    for (uint64_t n : d->dims) nbytes *= n;
    bytes fill;
    const uint8_t fill_bytes[8] = {1, 2, 2, 1, 0, 0, 0, 0};  // v1: late, if set, default value
    fill.raw(fill_bytes, 8);
    bytes layout;
    layout.u8(3);  // version 3
    layout.u8(1);  // contiguous
    layout.u64(d->address);
    layout.u64(nbytes);
    const bytes h = object_header({{kFillValue, fill},
                                   {kDatatype, datatype_message(d->type)},
                                   {kDataspace, dataspace_message(d->dims)},
                                   {kLayout, layout}});
    headers.push_back(append(h.b.data(), h.size()));
  }

  // Symbol table node holding every member, sorted by name.
  const uint16_t leaf_k = uint16_t(std::max<size_t>(4, (sorted.size() + 1) / 2));
  uint64_t snod_address = kUndefined;
  if (!sorted.empty()) {
    bytes snod;
    snod.raw("SNOD", 4);
    snod.u8(1);
    snod.u8(0);
    snod.u16(uint16_t(sorted.size()));
    for (size_t i = 0; i < sorted.size(); ++i) {
      snod.u64(name_offsets[i]);
      snod.u64(headers[i]);
      snod.u32(0);  // nothing cached
      snod.u32(0);
      snod.zeros(16);
    }
    snod.zeros(size_t(2 * leaf_k - sorted.size()) * 40);
    snod_address = append(snod.b.data(), snod.size());
  }

  // Group B-tree: one level-0 node pointing at the symbol table node.
  bytes tree;
  tree.raw("TREE", 4);
  tree.u8(0);  // group node
  tree.u8(0);  // level 0
  tree.u16(sorted.empty() ? 0 : 1);
  tree.u64(kUndefined);
  tree.u64(kUndefined);
  tree.u64(0);  // key 0: ""
  if (!sorted.empty()) {
    tree.u64(snod_address);
    tree.u64(name_offsets.back());  // key 1: the largest name in the child
  }
  const size_t node_bytes = 24 + 8 * (4 * size_t(kInternalK) + 1);
  tree.b.resize(node_bytes, 0);
  const uint64_t tree_address = append(tree.b.data(), tree.size());

  // Root group object header: symbol table message and attributes.
  std::vector<std::pair<uint16_t, bytes>> root;
  bytes table;
  table.u64(tree_address);
  table.u64(heap_address);
  root.push_back({kSymbolTable, table});
  for (const item& a : attributes_) {
    const bytes type = datatype_message(a.type);
    const bytes space = dataspace_message(a.dims);
    bytes m;
    m.u8(1);
    m.u8(0);
    m.u16(uint16_t(a.name.size() + 1));
    m.u16(uint16_t(type.size()));
    m.u16(uint16_t(space.size()));
    m.raw(a.name.c_str(), a.name.size() + 1);
    m.pad8();
    m.raw(type.b.data(), type.size());
    m.pad8();
    m.raw(space.b.data(), space.size());
    m.pad8();
    m.raw(a.value.data(), a.value.size());
    root.push_back({kAttribute, m});
  }
  const bytes root_header = object_header(root);
  const uint64_t root_address = append(root_header.b.data(), root_header.size());

  // Superblock version 0.
  bytes sb;
  sb.raw(kSignature, 8);
  sb.u8(0);  // superblock version
  sb.u8(0);  // free-space storage version
  sb.u8(0);  // root group symbol table entry version
  sb.u8(0);
  sb.u8(0);  // shared header message format version
  sb.u8(8);  // size of offsets
  sb.u8(8);  // size of lengths
  sb.u8(0);
  sb.u16(leaf_k);
  sb.u16(kInternalK);
  sb.u32(0);  // file consistency flags
  sb.u64(0);  // base address
  sb.u64(kUndefined);  // free-space info
  sb.u64(end_);        // end of file
  sb.u64(kUndefined);  // driver information block
  sb.u64(0);           // root entry: link name offset
  sb.u64(root_address);
  sb.u32(1);           // cached: symbol table
  sb.u32(0);
  sb.u64(tree_address);
  sb.u64(heap_address);
  write_at(0, sb.b.data(), sb.size());
  const int rc = std::fclose(file_);
  file_ = nullptr;
  if (rc != 0) throw error("HDF5: cannot close " + path_);
}

// ---------------------------------------------------------------------------
// reader
// ---------------------------------------------------------------------------

reader::reader(const std::string& path) {
  file_ = std::fopen(path.c_str(), "rb");
  if (!file_) throw error("HDF5: cannot open " + path);
  // The superblock sits at 0 or after a user block of 512 * 2^k bytes.
  uint64_t at = 0;
  bool found = false;
  for (int k = -1; k < 20 && !found; ++k) {
    at = k < 0 ? 0 : (512ull << k);
    uint8_t sig[8];
    if (std::fseek(file_, long(at), SEEK_SET) != 0 || std::fread(sig, 1, 8, file_) != 8) break;
    found = std::memcmp(sig, kSignature, 8) == 0;
  }
  if (!found) {
    std::fclose(file_);
    file_ = nullptr;
    throw error("HDF5: no superblock in " + path);
  }
  base_ = at;
  std::vector<uint8_t> sb(100);
  std::fseek(file_, long(at), SEEK_SET);
  sb.resize(std::fread(sb.data(), 1, sb.size(), file_));
  cursor c{sb};
  c.skip(8);
  const uint8_t version = c.u8();
  if (version > 1) throw error("HDF5: superblock version " + std::to_string(version) + " is not supported");
  c.skip(4);
  if (c.u8() != 8 || c.u8() != 8) throw error("HDF5: only 8-byte offsets and lengths are supported");
  c.skip(1);
  c.skip(4);  // group K values
  c.skip(4);  // consistency flags
  if (version == 1) c.skip(4);
  const uint64_t base_address = c.u64();
  base_ = base_address;  // addresses are relative to the base address
  c.skip(24);            // free space, end of file, driver block
  c.skip(8);             // root entry: link name offset
  root_header_ = c.u64();
  const auto messages = object_messages(root_header_);
  for (const auto& m : messages) {
    if (m.type == kSymbolTable) {
      cursor t{m.data};
      const uint64_t tree = t.u64();
      const uint64_t heap = t.u64();
      const auto h = bytes_at(heap, 32);
      if (std::memcmp(h.data(), "HEAP", 4) != 0) throw error("HDF5: bad local heap");
      cursor hc{h};
      hc.skip(8);
      const uint64_t data_size = hc.u64();
      hc.skip(8);
      const uint64_t data = hc.u64();
      const std::vector<uint8_t> names = bytes_at(data, data_size);
      walk_group_btree(tree, names, members_, 0);
    } else if (m.type == kLink) {
      // Compact new-style group: hard links in the root object header.
      cursor l{m.data};
      const uint8_t v = l.u8();
      if (v != 1) continue;
      const uint8_t flags = l.u8();
      uint8_t link_type = 0;
      if (flags & 0x08) link_type = l.u8();
      if (flags & 0x04) l.skip(8);
      if (flags & 0x10) l.skip(1);
      const int len_bytes = 1 << (flags & 3);
      const uint64_t len = l.uint(len_bytes);
      l.need(len);
      std::string name(reinterpret_cast<const char*>(&m.data[l.p]), len);
      l.skip(len);
      if (link_type == 0) members_[name] = l.u64();
    }
  }
}

reader::~reader() {
  if (file_) std::fclose(file_);
}

std::vector<uint8_t> reader::bytes_at(uint64_t address, uint64_t count) const {
  std::vector<uint8_t> out(count);
  if (std::fseek(file_, long(base_ + address), SEEK_SET) != 0 ||
      std::fread(out.data(), 1, count, file_) != count)
    throw error("HDF5: read past the end of the file");
  return out;
}

std::vector<reader::message> reader::object_messages(uint64_t address) const {
  const auto prefix = bytes_at(address, 16);
  cursor c{prefix};
  const uint8_t version = c.u8();
  if (version != 1) throw error("HDF5: object header version " + std::to_string(version) + " is not supported");
  c.skip(1);
  const uint16_t count = c.u16();
  c.skip(4);
  const uint32_t size = c.u32();
  std::vector<message> out;
  std::vector<std::pair<uint64_t, uint64_t>> blocks = {{address + 16, size}};
  for (size_t b = 0; b < blocks.size() && out.size() < count; ++b) {
    const auto block = bytes_at(blocks[b].first, blocks[b].second);
    cursor m{block};
    while (m.p + 8 <= block.size() && out.size() < count) {
      message msg;
      msg.type = m.u16();
      const uint16_t len = m.u16();
      m.skip(4);
      m.need(len);
      msg.data.assign(block.begin() + long(m.p), block.begin() + long(m.p + len));
      m.skip(len);
      if (msg.type == kContinuation) {
        cursor cc{msg.data};
        const uint64_t at = cc.u64();
        const uint64_t length = cc.u64();
        blocks.push_back({at, length});
      }
      out.push_back(std::move(msg));
    }
  }
  return out;
}

void reader::walk_group_btree(uint64_t address, const std::vector<uint8_t>& heap,
                              std::map<std::string, uint64_t>& out, int depth) const {
  if (depth > 32) throw error("HDF5: group B-tree too deep");
  const auto head = bytes_at(address, 24);
  if (std::memcmp(head.data(), "TREE", 4) != 0) throw error("HDF5: bad group B-tree node");
  cursor c{head};
  c.skip(4);
  if (c.u8() != 0) throw error("HDF5: not a group B-tree");
  const uint8_t level = c.u8();
  const uint16_t entries = c.u16();
  const auto body = bytes_at(address + 24, 8 * (2 * uint64_t(entries) + 1));
  cursor b{body};
  for (uint16_t i = 0; i < entries; ++i) {
    b.skip(8);  // key
    const uint64_t child = b.u64();
    if (level > 0) {
      walk_group_btree(child, heap, out, depth + 1);
      continue;
    }
    const auto sh = bytes_at(child, 8);
    if (std::memcmp(sh.data(), "SNOD", 4) != 0) throw error("HDF5: bad symbol table node");
    const uint16_t symbols = uint16_t(sh[6] | (sh[7] << 8));
    const auto entries_bytes = bytes_at(child + 8, 40 * uint64_t(symbols));
    cursor e{entries_bytes};
    for (uint16_t s = 0; s < symbols; ++s) {
      const uint64_t name_offset = e.u64();
      const uint64_t header = e.u64();
      e.skip(24);
      if (name_offset >= heap.size()) throw error("HDF5: name outside the local heap");
      const auto first = heap.begin() + long(name_offset);
      const auto nul = std::find(first, heap.end(), uint8_t(0));
      out[std::string(first, nul)] = header;
    }
  }
}

std::vector<std::string> reader::names() const {
  std::vector<std::string> out;
  for (const auto& [name, _] : members_) out.push_back(name);
  return out;
}

dataset_info reader::info(const std::string& name) const {
  const auto it = members_.find(name);
  if (it == members_.end()) throw error("HDF5: no dataset " + name);
  dataset_info d;
  bool have_layout = false;
  for (const auto& m : object_messages(it->second)) {
    cursor c{m.data};
    if (m.type == kDataspace) {
      const uint8_t version = c.u8();
      const uint8_t rank = c.u8();
      c.skip(1);
      if (version == 1) c.skip(5);
      else c.skip(1);
      d.dims.clear();
      for (uint8_t i = 0; i < rank; ++i) d.dims.push_back(c.u64());
    } else if (m.type == kDatatype) {
      const uint8_t cv = c.u8();
      const uint8_t bits0 = c.u8();
      c.skip(2);
      d.type_class = cv & 0x0f;
      d.type_size = c.u32();
      d.big_endian = bits0 & 1;
      d.is_signed = d.type_class == 0 && (bits0 & 0x08);
    } else if (m.type == kLayout) {
      const uint8_t version = c.u8();
      if (version == 3) {
        const uint8_t cls = c.u8();
        if (cls == 1) {
          d.address = c.u64();
          d.bytes = c.u64();
        } else if (cls == 0) {
          d.bytes = c.u16();
          d.address = kUndefined;  // compact: data in the message
          throw error("HDF5: compact dataset " + name + " is not supported");
        } else {
          throw error("HDF5: chunked dataset " + name + " is not supported");
        }
      } else if (version == 1 || version == 2) {
        const uint8_t rank = c.u8();
        const uint8_t cls = c.u8();
        c.skip(5);
        if (cls != 1) throw error("HDF5: only contiguous datasets are supported (" + name + ")");
        d.address = c.u64();
        uint64_t total = 1;
        for (uint8_t i = 0; i < rank; ++i) total *= c.u32();
        d.bytes = total;
      } else {
        throw error("HDF5: layout version " + std::to_string(version) + " is not supported");
      }
      have_layout = true;
    }
  }
  if (!have_layout || d.type_class < 0) throw error("HDF5: " + name + " is not a dataset");
  return d;
}

namespace {

template <class Out>
void convert(const dataset_info& d, const std::vector<uint8_t>& raw, Out* out, uint64_t n) {
  for (uint64_t i = 0; i < n; ++i) {
    const uint8_t* p = raw.data() + i * d.type_size;
    uint8_t le[8] = {0};
    for (uint32_t k = 0; k < d.type_size; ++k) le[k] = d.big_endian ? p[d.type_size - 1 - k] : p[k];
    if (d.type_class == 1) {
      if (d.type_size == 4) {
        float f;
        std::memcpy(&f, le, 4);
        out[i] = Out(f);
      } else {
        double f;
        std::memcpy(&f, le, 8);
        out[i] = Out(f);
      }
    } else {
      uint64_t v = 0;
      std::memcpy(&v, le, 8);
      if (d.is_signed && d.type_size < 8 && (le[d.type_size - 1] & 0x80))
        v |= ~0ull << (8 * d.type_size);
      out[i] = d.is_signed ? Out(int64_t(v)) : Out(v);
    }
  }
}

}  // namespace

void reader::read(const std::string& name, element out_type, void* out, uint64_t elements) const {
  const dataset_info d = info(name);
  if (d.elements() != elements) throw error("HDF5: size mismatch reading " + name);
  if (d.type_class != 0 && d.type_class != 1) throw error("HDF5: unsupported element type in " + name);
  if (d.type_class == 1 && d.type_size != 4 && d.type_size != 8)
    throw error("HDF5: unsupported float size in " + name);
  if (elements == 0) return;
  const auto raw = bytes_at(d.address, elements * d.type_size);
  switch (out_type) {
    case element::f32: convert(d, raw, static_cast<float*>(out), elements); break;
    case element::f64: convert(d, raw, static_cast<double*>(out), elements); break;
    case element::u64: convert(d, raw, static_cast<uint64_t*>(out), elements); break;
    default: throw error("HDF5: unsupported output type");
  }
}

std::vector<double> reader::root_attribute(const std::string& name) const {
  for (const auto& m : object_messages(root_header_)) {
    if (m.type != kAttribute) continue;
    cursor c{m.data};
    const uint8_t version = c.u8();
    c.skip(1);
    const uint16_t name_size = c.u16();
    const uint16_t type_size = c.u16();
    const uint16_t space_size = c.u16();
    if (version == 3) c.skip(1);
    const auto pad = [&](uint64_t n) { return version == 1 ? align8(n) : n; };
    c.need(name_size);
    std::string attr(reinterpret_cast<const char*>(&m.data[c.p]));
    c.skip(size_t(pad(name_size)));
    if (attr != name) continue;
    std::vector<uint8_t> type(m.data.begin() + long(c.p), m.data.begin() + long(c.p + type_size));
    c.skip(size_t(pad(type_size)));
    std::vector<uint8_t> space(m.data.begin() + long(c.p), m.data.begin() + long(c.p + space_size));
    c.skip(size_t(pad(space_size)));
    dataset_info d;
    d.type_class = type[0] & 0x0f;
    d.big_endian = type[1] & 1;
    d.is_signed = d.type_class == 0 && (type[1] & 0x08);
    d.type_size = uint32_t(type[4] | (type[5] << 8) | (type[6] << 16) | (uint32_t(type[7]) << 24));
    cursor s{space};
    const uint8_t sv = s.u8();
    const uint8_t rank = s.u8();
    s.skip(1);
    s.skip(sv == 1 ? 5 : 1);
    for (uint8_t i = 0; i < rank; ++i) d.dims.push_back(s.u64());
    const uint64_t n = d.elements();
    c.need(n * d.type_size);
    std::vector<uint8_t> raw(m.data.begin() + long(c.p), m.data.begin() + long(c.p + n * d.type_size));
    std::vector<double> out(n);
    convert(d, raw, out.data(), n);
    return out;
  }
  throw error("HDF5: no root attribute " + name);
}

}  // namespace h5
}  // namespace dpa_host
