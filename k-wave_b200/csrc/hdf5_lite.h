// A self-contained reader / writer for the subset of HDF5 that the k-Wave
// file boundary uses (no libhdf5 dependency).
//
// Reader: superblock versions 0-3 (with or without a user block, e.g. MATLAB
// v7.3 files), object header versions 1 and 2 with continuation blocks,
// groups stored as symbol tables (B-tree v1 + local heap) or as compact link
// messages, datasets with contiguous, compact or chunked (B-tree v1 index)
// layout, the deflate / shuffle / fletcher32 filters, integer, floating
// point and fixed-length string types, and attributes.
//
// Writer: superblock version 2, object header version 2, compact link
// groups, contiguous datasets and scalar string attributes -- readable by
// libhdf5 1.8 and later (MATLAB h5read).
#pragma once
#include <stdint.h>

#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace h5 {

struct Error : std::runtime_error {
  explicit Error(const std::string& m) : std::runtime_error("HDF5: " + m) {}
};

enum class Kind { Int, Float, String, Other };

struct TypeInfo {
  Kind kind = Kind::Other;
  int size = 0;        // bytes per element
  bool sign = false;   // integers
  bool big_endian = false;
};

struct DatasetInfo {
  std::vector<uint64_t> dims;  // C order (slowest first), as stored
  TypeInfo type;
  uint64_t numel() const {
    uint64_t n = 1;
    for (auto d : dims) n *= d;
    return n;
  }
};

class Reader {
 public:
  explicit Reader(const std::string& path);
  ~Reader();
  Reader(const Reader&) = delete;
  Reader& operator=(const Reader&) = delete;

  bool exists(const std::string& path);
  DatasetInfo info(const std::string& path);
  std::vector<float> read_float(const std::string& path);
  std::vector<double> read_double(const std::string& path);
  std::vector<uint64_t> read_u64(const std::string& path);
  // string attribute of an object ("/" for the root group); "" if absent
  std::string attribute_string(const std::string& path, const std::string& name);

 private:
  struct Impl;
  std::unique_ptr<Impl> p_;
};

enum class DType { F32, F64, U64 };

class Writer {
 public:
  // Add a dataset; dims in C order (slowest first).  `data` must stay valid
  // until write().  Intermediate groups in the path are created.
  void dataset(const std::string& path, DType t, const std::vector<uint64_t>& dims, const void* data,
               const std::map<std::string, std::string>& attrs = {});
  void root_attribute(const std::string& name, const std::string& value);
  void write(const std::string& file);

 private:
  struct Node {
    bool is_group = true;
    std::map<std::string, std::unique_ptr<Node>> children;  // sorted names
    std::vector<std::string> order;                         // insertion order
    DType type = DType::F32;
    std::vector<uint64_t> dims;
    const void* data = nullptr;
    std::map<std::string, std::string> attrs;
    uint64_t addr = 0, data_addr = 0, header_size = 0;
  };
  Node root_;
  Node* group(const std::string& path, std::string* leaf);
};

// Bob Jenkins' lookup3 hashlittle(), the checksum of HDF5 metadata.
uint32_t lookup3(const void* key, size_t length, uint32_t initval);

}  // namespace h5
