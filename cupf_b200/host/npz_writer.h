// npz_writer.h — writes named 1-D arrays as a NumPy .npz archive (an
// uncompressed zip of .npy files), readable with numpy.load.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace cupf_host {

class NpzWriter {
 public:
  void add(const std::string& name, const std::vector<float>& v);
  void add(const std::string& name, const std::vector<int>& v);
  void add_raw(const std::string& name, const char* descr, const void* data, size_t count,
               size_t elem);
  bool write(const std::string& path) const;

 private:
  struct Entry {
    std::string name;
    std::string bytes;  // full .npy file
  };
  std::vector<Entry> mEntries;
};

}  // namespace cupf_host
