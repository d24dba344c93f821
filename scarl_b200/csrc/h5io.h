// h5io.h -- a self-contained writer and reader of the classic HDF5 file
// format subset the reference's output uses (HDF5 File Format
// Specification, version 0 superblock): one root group held in a symbol
// table (v1 B-tree of group nodes, symbol table nodes, local heap), version 1
// object headers, contiguous datasets of IEEE floats, 32-bit integers or
// fixed-length strings, and version 1 attribute messages.  No HDF5 library is
// involved; the byte layout follows the specification.
#pragma once

#include <stdint.h>

#include <functional>
#include <string>
#include <vector>

namespace scarl {
namespace h5 {

enum Kind { F64 = 0, F32 = 1, I32 = 2, STR = 3 };

struct Attr {
  std::string name;
  Kind kind = F64;
  std::vector<uint64_t> dims;  // empty = scalar
  int strsize = 0;             // STR: bytes per string (space padded)
  std::vector<uint8_t> data;   // little-endian element bytes
};

struct Dataset {
  std::string name;
  Kind kind = F64;
  std::vector<uint64_t> dims;  // HDF5 order (slowest first)
  int strsize = 0;
  std::vector<Attr> attrs;
  uint64_t nbytes = 0;
  // writes exactly nbytes of raw data at the current file position
  std::function<bool(FILE*)> write;
};

Attr attr_f64(const std::string& n, const double* v, int count, bool scalar = false);
Attr attr_i32(const std::string& n, const int* v, int count, bool scalar = false);
Attr attr_str(const std::string& n, const std::string& v);
int elem_size(Kind k, int strsize);

// Writes root attributes and datasets; 0 on success.
int write_file(const std::string& path, const std::vector<Attr>& root,
               const std::vector<Dataset>& dsets, std::string* err);

struct RObject {
  std::string name;  // "" for the root group
  Kind kind = F64;
  int elsize = 0;
  bool is_dataset = false;
  std::vector<uint64_t> dims;
  std::vector<Attr> attrs;
  uint64_t data_addr = 0;  // absolute file offset of contiguous data
  uint64_t nbytes = 0;
};

// Parses the root group and its datasets (attributes included).
int read_file(const std::string& path, RObject* root, std::vector<RObject>* dsets,
              std::string* err);

// Adds (or replaces) root-group attributes of an existing classic-format
// file: a new root object header holding the old messages and the new
// attributes is appended at the end of the file and the superblock's root
// entry and end-of-file address are pointed at it (the old header becomes
// unused space).
int append_root_attrs(const std::string& path, const std::vector<Attr>& attrs, std::string* err);

// Overwrites the raw bytes of a contiguous dataset in place (same size).
int overwrite_dataset(const std::string& path, const std::string& name, const void* data,
                      uint64_t nbytes, std::string* err);

// Reads a dataset's elements converted to double or float.
int read_values(const std::string& path, const RObject& d, double* out64, float* out32,
                std::string* err);

}  // namespace h5
}  // namespace scarl
