// host_capi.cpp — C entry points of include/cupf_host.h.
#include <cstring>
#include <string>
#include <vector>

#include "../../include/cupf_host.h"
#include "host_util.h"
#include "phase_field.h"
#include "h5_writer.h"
#include "qoi.h"

using namespace cupf_host;

extern "C" int cupf_host_grain_volumes(int fnx, int fny, int fnz, const int32_t* alpha,
                                       int32_t* grain_ids, int32_t* volumes, int cap) {
  QoiGrid g;
  g.fnx = fnx;
  g.fny = fny;
  g.fnz = fnz;
  QOI3D q(g);
  q.calculateQoIs(g, alpha, 0);
  const int n = q.mNumActiveGrains;
  if (n > cap) return -1;
  for (int i = 0; i < n; ++i) {
    grain_ids[i] = q.mQoIVectorIntData["grainToPF"][i];
    volumes[i] = q.mQoIVectorIntData["volume"][i];
  }
  return n;
}

extern "C" int cupf_host_line_qois(int fnx, int fny, int fnz, int num_theta, int* cur_tip,
                                   const int32_t* alpha, const int32_t* loss_area, int move_count,
                                   int32_t* tip_y, int32_t* total_area, int32_t* extra_area) {
  QoiGrid g;
  g.fnx = fnx;
  g.fny = fny;
  g.fnz = fnz;
  g.num_theta = num_theta;
  g.nts = 0;
  QOILine q(g);
  q.calculateLineQoIs(g, *cur_tip, alpha, 0, nullptr, loss_area, move_count);
  *tip_y = q.mQoIVectorIntData["tip_y"][0];
  for (int i = 0; i < num_theta; ++i) {
    total_area[i] = q.mQoIVectorIntData["total_area"][i];
    extra_area[i] = q.mQoIVectorIntData["extra_area"][i];
  }
  return 0;
}

extern "C" int cupf_host_sample_heights(int* cur_tip, const int32_t* alpha, int fnx, int fny,
                                        int fnz) {
  QoiGrid g;
  QOI3D q(g);
  q.sampleHeights(*cur_tip, alpha, fnx, fny, fnz);
  return 0;
}

extern "C" int cupf_host_junctions_3d(int fnx, int fny, int fnz, const int32_t* alpha,
                                      int32_t* nodes, int cap) {
  QoiGrid g;
  g.fnx = fnx;
  g.fny = fny;
  g.fnz = fnz;
  QOI3D q(g);
  q.calculateQoIs(g, alpha, 0);
  q.searchJunctionsOnImage(g, alpha);
  const std::vector<int>& v = q.mQoIVectorIntData["node_region"];
  const int n = (int)v.size();
  for (int i = 0; i < n && i < cap; ++i) nodes[i] = v[i];
  return n;
}

extern "C" int cupf_host_junctions_3d_cells(int fnx, int fny, int fnz, const int32_t* alpha,
                                            const int64_t* cells, int64_t ncells,
                                            const uint8_t* distinct, int32_t* nodes, int cap) {
  QoiGrid g;
  g.fnx = fnx;
  g.fny = fny;
  g.fnz = fnz;
  QOI3D q(g);
  q.calculateQoIs(g, alpha, 0);
  std::vector<long long> c(cells, cells + ncells);
  q.searchJunctionsOnCells(g, alpha, c.data(), ncells, distinct);
  const std::vector<int>& v = q.mQoIVectorIntData["node_region"];
  const int n = (int)v.size();
  for (int i = 0; i < n && i < cap; ++i) nodes[i] = v[i];
  return n;
}

// QOILine::searchJunctionsOnImage (or its candidate-cell form when cells is not
// NULL) on a full map whose frame kt has its tip layer at tip_y[kt].
static int line_junctions(int fnx, int fny, int nts, int num_nodes, const int32_t* tip_y,
                          const int32_t* alpha, const int64_t* cells, int64_t ncells,
                          int32_t* nodes, int cap, int32_t* cross, int64_t cross_cap) {
  if (fnx < 3 || fny < 3 || nts < 0 || num_nodes < 0 || !tip_y || !alpha) return -1;
  QoiGrid g;
  g.fnx = fnx;
  g.fny = fny;
  g.nts = nts;
  g.num_nodes = num_nodes;
  g.num_theta = 1;
  QOILine q(g);
  q.mQoIVectorIntData["tip_y"].assign(tip_y, tip_y + nts + 1);
  if (cells) {
    std::vector<long long> c(cells, cells + ncells);
    q.searchJunctionsOnCells(g, alpha, c.data(), ncells);
  } else {
    q.searchJunctionsOnImage(g, alpha);
  }
  const std::vector<int>& v = q.mQoIVectorIntData["node_region"];
  const int n = (int)v.size();
  for (int i = 0; i < n && i < cap; ++i) nodes[i] = v[i];
  const std::vector<int>& cs = q.mQoIVectorIntData["cross_sec"];
  if (cross)
    for (int64_t i = 0; i < (int64_t)cs.size() && i < cross_cap; ++i) cross[i] = cs[i];
  return n;
}

extern "C" int cupf_host_line_junctions(int fnx, int fny, int nts, int num_nodes,
                                        const int32_t* tip_y, const int32_t* alpha,
                                        int32_t* nodes, int cap, int32_t* cross,
                                        int64_t cross_cap) {
  return line_junctions(fnx, fny, nts, num_nodes, tip_y, alpha, nullptr, 0, nodes, cap, cross,
                        cross_cap);
}

extern "C" int cupf_host_line_junctions_cells(int fnx, int fny, int nts, int num_nodes,
                                              const int32_t* tip_y, const int32_t* alpha,
                                              const int64_t* cells, int64_t ncells,
                                              int32_t* nodes, int cap, int32_t* cross,
                                              int64_t cross_cap) {
  if (ncells < 0 || (ncells > 0 && !cells)) return -1;
  static const int64_t none = 0;
  return line_junctions(fnx, fny, nts, num_nodes, tip_y, alpha, cells ? cells : &none, ncells,
                        nodes, cap, cross, cross_cap);
}

extern "C" int cupf_host_h5_write(const char* path, int n, const char* const* names,
                                  const char* kinds, const int32_t* elem_bytes,
                                  const int64_t* counts, const void* const* data) {
  if (!path || n < 0 || (n > 0 && (!names || !kinds || !elem_bytes || !counts || !data))) return -1;
  H5Writer w;
  for (int i = 0; i < n; ++i) {
    const char k = kinds[i];
    const int e = elem_bytes[i];
    if (!names[i] || counts[i] < 0 || (counts[i] > 0 && !data[i])) return -1;
    if (!((k == 'i' && (e == 1 || e == 2 || e == 4 || e == 8)) || (k == 'f' && (e == 4 || e == 8))))
      return -1;
    w.add_raw(names[i], k, data[i], (size_t)counts[i], (size_t)e);
  }
  return w.write(path) ? 0 : -1;
}

extern "C" int cupf_host_get_param_float(const char* line, const char* key, float* value) {
  return getParam(std::string(line), std::string(key), *value) ? 1 : 0;
}

extern "C" int cupf_host_get_param_int(const char* line, const char* key, int32_t* value) {
  int v = *value;
  const bool ok = getParam(std::string(line), std::string(key), v);
  *value = v;
  return ok ? 1 : 0;
}

extern "C" int cupf_host_get_options(int argc, char** argv, int32_t* out, char* input_file,
                                     char* folder, char* outdir, int cap) {
  DesignSettingData d;
  if (!d.getOptions(argc, argv)) return -1;
  out[0] = d.useLineConfig;
  out[1] = d.includeNucleation;
  out[2] = d.pureNucleation;
  out[3] = d.useAPT;
  out[4] = d.save3DField;
  out[5] = d.mpiDim;
  out[6] = d.seedValue;
  out[7] = d.bcX;
  out[8] = d.bcY;
  out[9] = d.bcZ;
  std::strncpy(input_file, d.inputFile.c_str(), cap);
  std::strncpy(folder, d.thermalInputFolder.c_str(), cap);
  std::strncpy(outdir, d.outputFolder.c_str(), cap);
  return 0;
}

namespace {
class SetupOnly : public PhaseField {
 public:
  void cudaSetup() override {}
  void evolve() override {}
};
}  // namespace

extern "C" int cupf_host_setup(const char* input_file, const char* folder, int bcX, int bcY,
                               int bcZ, int flags, int32_t* dims, float* fparams, float* phi,
                               int32_t* alpha, int64_t length_cap, char* err, int err_cap) {
  DesignSettingData ds;
  ds.inputFile = input_file;
  ds.useLineConfig = (flags & 1) != 0;
  ds.pureNucleation = (flags & 2) != 0;
  ds.bcX = bcX;
  ds.bcY = bcY;
  ds.bcZ = bcZ;
  SetupOnly pf;
  pf.SetDesignSetting(&ds);
  pf.mac.folder = folder;
  std::string path = input_file;
  // the thermal type is chosen by the input file's name; the file itself may
  // live elsewhere: try the folder's parent when the bare name does not open
  MPIsetting1D mpi;
  mpi.domainPartition();
  pf.SetMPIManager(&mpi);
  pf.parseInputParams(path);
  pf.cpuSetup(&mpi);
  pf.initField();
  if (pf.failed()) {
    if (err && err_cap > 0) std::strncpy(err, pf.lastError().c_str(), err_cap);
    return -1;
  }
  dims[0] = pf.fnx;
  dims[1] = pf.fny;
  dims[2] = pf.fnz;
  dims[3] = pf.params.num_theta;
  const GlobalConstants& p = pf.params;
  const float fp[8] = {p.dt, p.tau0, p.lamd, p.hi, p.G, p.underCoolingRate, p.z0, p.kin_delta};
  std::memcpy(fparams, fp, sizeof(fp));
  if (phi && alpha && length_cap >= pf.length) {
    std::memcpy(phi, pf.phi.data(), sizeof(float) * pf.length);
    std::memcpy(alpha, pf.alpha.data(), sizeof(int) * pf.length);
  }
  return 0;
}

extern "C" int cupf_host_setup_state(const char* input_file, const char* folder, int bcX, int bcY,
                                     int bcZ, int flags, int32_t* dims, float* fparams, float* x,
                                     float* y, float* z, float* z_full, float* phi, float* psi,
                                     int32_t* alpha, float* sint, float* cost, int64_t cap,
                                     char* err, int err_cap) {
  if (!input_file || !folder || !dims || !fparams) return -1;
  DesignSettingData ds;
  ds.inputFile = input_file;
  ds.useLineConfig = (flags & 1) != 0;
  ds.pureNucleation = (flags & 2) != 0;
  ds.includeNucleation = (flags & 4) != 0;
  ds.bcX = bcX;
  ds.bcY = bcY;
  ds.bcZ = bcZ;
  SetupOnly pf;
  pf.SetDesignSetting(&ds);
  pf.mac.folder = folder;
  MPIsetting1D mpi;
  mpi.domainPartition();
  pf.SetMPIManager(&mpi);
  pf.parseInputParams(input_file);
  pf.cpuSetup(&mpi);
  pf.initField();
  if (pf.failed()) {
    if (err && err_cap > 0) std::strncpy(err, pf.lastError().c_str(), err_cap);
    return -1;
  }
  const GlobalConstants& p = pf.params;
  const int32_t d[8] = {pf.fnx, pf.fny, pf.fnz, p.num_theta, p.Mt, p.nts, p.thermalType, pf.fnz_f};
  std::memcpy(dims, d, sizeof(d));
  const float f[20] = {p.dt,  p.tau0, p.lamd, p.hi,  p.G,  p.underCoolingRate, p.z0,
                       p.kin_delta, p.lxd, p.lyd, p.lzd, p.R, p.V, p.top, p.r0, p.x0,
                       p.cfl, p.underCoolingRate0, p.W0, p.dx};
  std::memcpy(fparams, f, sizeof(f));
  if (x) std::memcpy(x, pf.x.data(), sizeof(float) * pf.fnx);
  if (y) std::memcpy(y, pf.y.data(), sizeof(float) * pf.fny);
  if (z) std::memcpy(z, pf.z.data(), sizeof(float) * pf.fnz);
  if (z_full) std::memcpy(z_full, pf.z_full.data(), sizeof(float) * pf.fnz_f);
  if (pf.length <= cap) {
    if (phi) std::memcpy(phi, pf.phi.data(), sizeof(float) * pf.length);
    if (psi && (long long)pf.psi.size() >= pf.length)
      std::memcpy(psi, pf.psi.data(), sizeof(float) * pf.length);
    if (alpha) std::memcpy(alpha, pf.alpha.data(), sizeof(int) * pf.length);
  }
  const long long nt = 2ll * p.num_theta + 1;
  if (nt <= cap) {
    if (sint) std::memcpy(sint, pf.mac.sint.data(), sizeof(float) * nt);
    if (cost) std::memcpy(cost, pf.mac.cost.data(), sizeof(float) * nt);
  }
  return pf.length <= cap ? 0 : 1;
}
