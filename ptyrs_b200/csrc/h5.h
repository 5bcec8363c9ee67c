// A reader for the part of the HDF5 file format that the ptychography files of PyNX
// (`save_ptycho_data_cxi`) and PtyPy (`Ptycho.save_run`) use through libhdf5's default
// ("earliest") layouts, written from the published HDF5 file-format specification: superblocks
// of versions 0-3, object headers of versions 1 and 2, groups as symbol tables (v1 B-tree,
// local heap, symbol-table nodes) or as compact link messages, hard and soft links, datasets
// with compact, contiguous or chunked (v1 B-tree index) layout, the deflate, shuffle and
// Fletcher-32 filters, and fixed-point, floating-point, enumeration and compound datatypes.
// The reference reads these files with the pure-Rust `rust-hdf5` crate (physwkim/ptyrs
// ptyrs/src/io/mod.rs:1-8), which is not vendored; this is the host side of the library and
// no part of the GPU path.
#pragma once
#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <vector>

namespace ptyb::h5 {

// A datatype as the file stores it.
struct Type {
  enum Class { kFixed = 0, kFloat = 1, kString = 3, kCompound = 6, kEnum = 8, kOther = -1 };
  int cls = kOther;
  uint32_t size = 0;
  bool is_signed = false, big_endian = false;
  // compound members (name, byte offset, type), enumeration base type
  struct Member {
    std::string name;
    uint32_t offset;
    std::shared_ptr<Type> type;
  };
  std::vector<Member> members;
  std::shared_ptr<Type> base;
};

// A dataset read whole: its shape, its element type and its raw bytes in the file's element
// layout, row-major.
struct Dataset {
  std::vector<uint64_t> shape;
  Type type;
  std::vector<uint8_t> bytes;
  uint64_t count() const {
    uint64_t n = 1;
    for (uint64_t d : shape) n *= d;
    return n;
  }
};

class File {
 public:
  // Throws std::runtime_error with the reason when the file cannot be read.
  explicit File(const std::string& path);
  // The dataset at an absolute or root-relative path (links followed); throws if absent.
  Dataset dataset(const std::string& path) const;
  // Whether a dataset or group exists at the path.
  bool exists(const std::string& path) const;
  // The names of a group's members, in the order the group lists them.
  std::vector<std::string> members(const std::string& path) const;

 private:
  std::vector<uint8_t> buf_;
  int so_ = 8, sl_ = 8;  // sizes of offsets and lengths
  uint64_t base_ = 0, root_ = 0;
  // Work done by the current public call (header blocks, B-tree entries, decoded chunk
  // kilobytes), bounded so that a damaged file's cycles end with an error.
  mutable uint64_t work_ = 0;
  void spend(uint64_t units) const;

  struct Message {
    uint16_t type;
    const uint8_t* p;
    size_t size;
  };
  struct Link {
    bool soft = false;
    uint64_t addr = 0;
    std::string target;
  };

  uint64_t uint_at(uint64_t at, int n) const;
  const uint8_t* ptr(uint64_t addr, uint64_t n) const;
  std::vector<Message> messages(uint64_t header) const;
  void collect(uint64_t at, uint64_t len, int version, std::vector<Message>* out, int depth) const;
  std::map<std::string, Link> links(uint64_t header) const;
  void group_btree(uint64_t btree, uint64_t heap, std::map<std::string, Link>* out,
                   std::vector<std::string>* order, int depth) const;
  uint64_t resolve(const std::string& path, int depth = 0) const;
  std::vector<std::string> member_order(uint64_t header) const;
};

}  // namespace ptyb::h5
