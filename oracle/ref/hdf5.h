/* hdf5.h — TEST INFRASTRUCTURE ONLY.  Stand-in for the few libhdf5 calls of the
 * reference's PhaseFieldCpu.cpp (no libhdf5 exists in this image), so that file
 * compiles unmodified into the parity harness and its parseInputParams /
 * cpuSetup / initField run for real.  Names and argument lists follow libhdf5's
 * public API; every read returns zeros (the temperature table Temp.h5, which
 * only nucleation reads), writes and closes do nothing. */
#pragma once
#include <cstring>
#include <vector>

typedef long long hid_t;
typedef unsigned long long hsize_t;
typedef int herr_t;

#define H5F_ACC_RDONLY 0u
#define H5F_ACC_TRUNC 2u
#define H5P_DEFAULT ((hid_t)0)
#define H5S_ALL ((hid_t)0)
static const hid_t H5T_NATIVE_INT = 1;
static const hid_t H5T_NATIVE_FLOAT = 2;
static const hid_t H5T_NATIVE_FLOAT_g = 2;

/* element counts of the dataspaces made by H5Screate_simple (id = index + 1) */
static inline std::vector<hsize_t>& cupf_h5stub_spaces() {
  static std::vector<hsize_t> s;
  return s;
}
static inline hid_t H5Fopen(const char*, unsigned, hid_t) { return 1; }
static inline hid_t H5Fcreate(const char*, unsigned, hid_t, hid_t) { return 1; }
static inline herr_t H5Fclose(hid_t) { return 0; }
static inline hid_t H5Dopen2(hid_t, const char*, hid_t) { return 1; }
static inline hid_t H5Dcreate2(hid_t, const char*, hid_t, hid_t, hid_t, hid_t, hid_t) { return 1; }
static inline hid_t H5Dget_space(hid_t) { return 0; }
static inline hid_t H5Screate_simple(int rank, const hsize_t* dims, const hsize_t*) {
  hsize_t n = 1;
  for (int i = 0; i < rank; ++i) n *= dims[i];
  cupf_h5stub_spaces().push_back(n);
  return (hid_t)cupf_h5stub_spaces().size();
}
static inline herr_t H5Dread(hid_t, hid_t type, hid_t mem, hid_t, hid_t, void* buf) {
  if (mem > 0 && (size_t)mem <= cupf_h5stub_spaces().size())
    std::memset(buf, 0, cupf_h5stub_spaces()[mem - 1] * (type == H5T_NATIVE_INT ? sizeof(int)
                                                                                 : sizeof(float)));
  return 0;
}
static inline herr_t H5Dwrite(hid_t, hid_t, hid_t, hid_t, hid_t, const void*) { return 0; }
static inline herr_t H5Sclose(hid_t) { return 0; }
static inline herr_t H5Dclose(hid_t) { return 0; }
