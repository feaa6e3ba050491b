// array_file.h — output file of named 1-D arrays for the drivers: HDF5 (the
// reference's format, h5_writer.h) unless the environment variable
// CUPF_OUTPUT_FORMAT is "npz", which asks for a NumPy .npz archive
// (npz_writer.h) instead.
#pragma once

#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "h5_writer.h"
#include "npz_writer.h"

namespace cupf_host {

class ArrayFile {
 public:
  ArrayFile() {
    const char* f = std::getenv("CUPF_OUTPUT_FORMAT");
    mNpz = f && std::strcmp(f, "npz") == 0;
  }
  template <class T>
  void add(const std::string& name, const std::vector<T>& v) {
    if (mNpz) mNpzW.add(name, v);
    else mH5.add(name, v);
  }
  const char* extension() const { return mNpz ? ".npz" : ".h5"; }
  // writes base + extension(); returns false when the file cannot be written
  bool write(const std::string& base) const {
    return mNpz ? mNpzW.write(base + extension()) : mH5.write(base + extension());
  }

 private:
  bool mNpz = false;
  H5Writer mH5;
  NpzWriter mNpzW;
};

}  // namespace cupf_host
