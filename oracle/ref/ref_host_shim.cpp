// ref_host_shim.cpp — TEST INFRASTRUCTURE ONLY.
// extern "C" entry points into the reference's own host code (3DgrainMPI/QOI.cpp,
// helper.cpp, DesignSettingData.cpp), compiled unmodified from the reference
// tree by oracle/build.py, so CPU tests can compare the library's host logic
// (QoIs, input-file parser, CLI) with the reference's.
#include <cstring>
#include <getopt.h>
#include <string>
#include <vector>
#include "QOI.h"
#include "helper.h"
#include "DesignSettingData.h"

extern "C" {

// QOI::calculateQoIs (QOI.cpp:198-231).  Writes grainToPF/volume in first-seen
// order; returns the number of active grains (or -1 if cap is too small).
int refq_calculate_qois(int fnx, int fny, int fnz, int num_theta, int nts, const int* alpha,
                        int* grain_to_pf, int* volume, int cap) {
  GlobalConstants p;
  std::memset(&p, 0, sizeof(p));
  p.fnx = fnx; p.fny = fny; p.fnz = fnz; p.num_theta = num_theta; p.nts = nts;
  QOI3D q(p);
  q.calculateQoIs(p, alpha, 0);
  int n = q.mNumActiveGrains;
  if (n > cap) return -1;
  for (int i = 0; i < n; ++i) {
    grain_to_pf[i] = q.mQoIVectorIntData["grainToPF"][i];
    volume[i] = q.mQoIVectorIntData["volume"][i];
  }
  return n;
}

// QOI::calculateLineQoIs (QOI.cpp:38-101) for frame kt.  cur_tip in/out.
// Outputs tip_y[kt], total_area/extra_area rows kt (num_theta each).
int refq_calculate_line_qois(int fnx, int fny, int fnz, int num_theta, int nts, int num_nodes,
                             int* cur_tip, const int* alpha, int kt, const float* z,
                             const int* loss_area, int move_count, int* tip_y, int* total_area,
                             int* extra_area) {
  GlobalConstants p;
  std::memset(&p, 0, sizeof(p));
  p.fnx = fnx; p.fny = fny; p.fnz = fnz; p.num_theta = num_theta; p.nts = nts;
  p.num_nodes = num_nodes;
  QOILine q(p);
  q.calculateLineQoIs(p, *cur_tip, alpha, kt, z, loss_area, move_count);
  *tip_y = q.mQoIVectorIntData["tip_y"][kt];
  for (int g = 0; g < num_theta; ++g) {
    total_area[g] = q.mQoIVectorIntData["total_area"][kt * num_theta + g];
    extra_area[g] = q.mQoIVectorIntData["extra_area"][kt * num_theta + g];
  }
  return 0;
}

// QOI3D::searchJunctionsOnImage (QOI.cpp:233-311) after calculateQoIs.
int refq_junctions_3d(int fnx, int fny, int fnz, const int* alpha, int* nodes, int cap) {
  GlobalConstants p;
  std::memset(&p, 0, sizeof(p));
  p.fnx = fnx; p.fny = fny; p.fnz = fnz;
  QOI3D q(p);
  q.calculateQoIs(p, alpha, 0);
  q.searchJunctionsOnImage(p, alpha);
  const std::vector<int>& v = q.mQoIVectorIntData["node_region"];
  const int n = (int)v.size();
  for (int i = 0; i < n && i < cap; ++i) nodes[i] = v[i];
  return n;
}

// QOILine::searchJunctionsOnImage (QOI.cpp:103-160) on a full map whose frame
// kt has its tip layer at tip_y[kt].  Writes node_region (up to cap) and the
// cross sections (up to cross_cap); returns node_region's length.
int refq_line_junctions(int fnx, int fny, int nts, int num_nodes, const int* tip_y,
                        const int* alpha, int* nodes, int cap, int* cross, long long cross_cap) {
  GlobalConstants p;
  std::memset(&p, 0, sizeof(p));
  p.fnx = fnx; p.fny = fny; p.nts = nts; p.num_nodes = num_nodes; p.num_theta = 1;
  QOILine q(p);
  for (int kt = 0; kt <= nts; ++kt) q.mQoIVectorIntData["tip_y"][kt] = tip_y[kt];
  q.searchJunctionsOnImage(p, alpha);
  const std::vector<int>& v = q.mQoIVectorIntData["node_region"];
  const int n = (int)v.size();
  for (int i = 0; i < n && i < cap; ++i) nodes[i] = v[i];
  const std::vector<int>& c = q.mQoIVectorIntData["cross_sec"];
  for (long long i = 0; i < (long long)c.size() && i < cross_cap; ++i) cross[i] = c[i];
  return n;
}

// QOI::sampleHeights (QOI.cpp:162-185).
int refq_sample_heights(int* cur_tip, const int* alpha, int fnx, int fny, int fnz) {
  GlobalConstants p;
  std::memset(&p, 0, sizeof(p));
  QOI3D q(p);
  q.sampleHeights(*cur_tip, alpha, fnx, fny, fnz);
  return 0;
}

// getParam (helper.cpp:44-74), float and int overloads.
int refq_get_param_float(const char* line, const char* key, float* value) {
  getParam(std::string(line), std::string(key), *value);
  return 0;
}
int refq_get_param_int(const char* line, const char* key, int* value) {
  getParam(std::string(line), std::string(key), *value);
  return 0;
}

// read_input (helper.cpp:77-101) into a caller buffer of n floats.
int refq_read_input_float(const char* path, float* out) {
  read_input(std::string(path), out);
  return 0;
}

// DesignSettingData::getOptions (DesignSettingData.cpp:14-80).
// out: [useLineConfig, includeNucleation, pureNucleation, useAPT, save3DField,
//       mpiDim, seedValue, bcX, bcY, bcZ]
int refq_get_options(int argc, char** argv, int* out, char* input_file, char* folder,
                     char* outdir, int cap) {
  DesignSettingData d;
  optind = 0;  // getopt keeps global state; 0 forces a full re-scan
  d.getOptions(argc, argv);
  out[0] = d.useLineConfig; out[1] = d.includeNucleation; out[2] = d.pureNucleation;
  out[3] = d.useAPT; out[4] = d.save3DField; out[5] = d.mpiDim; out[6] = d.seedValue;
  out[7] = d.bcX; out[8] = d.bcY; out[9] = d.bcZ;
  std::strncpy(input_file, d.inputFile.c_str(), cap);
  std::strncpy(folder, d.thermalInputFolder.c_str(), cap);
  std::strncpy(outdir, d.outputFolder.c_str(), cap);
  return 0;
}

}  // extern "C"
