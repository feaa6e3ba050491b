// h5_writer.h — writes named 1-D arrays (int32 / float32 / float64) as datasets
// of the root group of an HDF5 file, the output format of the reference's
// PhaseField::OutputQoIs / OutputField (3DgrainMPI/PhaseFieldCpu.cpp:464-613,
// h5write_1d :584-613: one 1-D dataset per array, native int or float).
//
// The file follows the HDF5 file format specification in its oldest, most
// widely readable form, so that every libhdf5 release and h5py can open it:
// superblock version 0, version-1 object headers, the root group as a symbol
// table (a version-1 B-tree of group nodes over symbol-table nodes, names in a
// local heap), and each dataset as a contiguous, little-endian array with a
// simple 1-D dataspace.  No compression, chunking or attributes.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace cupf_host {

class H5Writer {
 public:
  void add(const std::string& name, const std::vector<float>& v);
  void add(const std::string& name, const std::vector<int>& v);
  void add(const std::string& name, const std::vector<double>& v);
  // kind: 'i' (signed integer) or 'f' (IEEE float); elem: bytes per element
  void add_raw(const std::string& name, char kind, const void* data, size_t count, size_t elem);
  bool write(const std::string& path) const;
  // the whole file as bytes (what write() stores)
  std::string bytes() const;

 private:
  struct Entry {
    std::string name;
    char kind;
    size_t elem;
    size_t count;
    std::string data;
  };
  std::vector<Entry> mEntries;
};

}  // namespace cupf_host
