// phase_field.cpp — the APT driver (see phase_field.h).
#include "phase_field.h"
#include "../../include/cupf_host.h"

#include <getopt.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>

#include "host_util.h"
#include "array_file.h"

namespace cupf_host {

static const double kLS = -0.995;  // APTPhaseField.cu:25, PhaseFieldCpu.cpp:13
static const int kTIPP = 20;       // moving-domain check interval, APTPhaseField.cu:29

// ------------------------------------------------------------------ CLI
bool DesignSettingData::getOptions(int argc, char** argv, std::string* err) {
  if (argc < 2) {
    if (err) *err = "usage: phase_field <input file> [-s seed] [-b XYZ] [-l 1] [-n 1|2] [-d N] "
                    "[-o dir] [-f folder]";
    return false;
  }
  inputFile = argv[1];
  static struct option long_options[] = {{"help", 0, 0, '?'},
                                         {"macfile", 1, 0, 'f'},
                                         {"useAPT", 1, 0, 'a'},
                                         {"seed", 1, 0, 's'},
                                         {"output", 1, 0, 'o'},
                                         {"mpiDim", 1, 0, 'm'},
                                         {"saveField", 1, 0, 'd'},
                                         {"lineConfig", 1, 0, 'l'},
                                         {"includeNuclean", 1, 0, 'n'},
                                         {"boundaryCondition", 1, 0, 'b'},
                                         {0, 0, 0, 0}};
  optind = 0;  // allow repeated parsing in one process
  int opt;
  while ((opt = getopt_long(argc, argv, "b:f:o:a:s:m:l:n:d:?", long_options, nullptr)) != -1) {
    switch (opt) {
      case 'f': thermalInputFolder = optarg; break;
      case 'a': useAPT = false; break;
      case 's': seedValue = atoi(optarg); break;
      case 'o': outputFolder = outputFolder + optarg; break;
      case 'm': mpiDim = atoi(optarg); break;
      case 'd': save3DField = atoi(optarg); break;
      case 'l': useLineConfig = true; break;
      case 'n':
        includeNucleation = true;
        if (atoi(optarg) == 1) pureNucleation = true;
        break;
      case 'b':
        givenBC = atoi(optarg);
        bcX = givenBC / 100;
        bcY = (givenBC - 100 * bcX) / 10;
        bcZ = givenBC % 10;
        break;
      default: break;
    }
  }
  return true;
}

// ------------------------------------------------------------------ moving domain
void MovingDomain::allocateMovingDomain(int numGrains, int movingDirectionSize) {
  tip_thres = (int)(0.8 * movingDirectionSize);  // APTPhaseField.cu:641
  loss_area_host.assign(numGrains, 0);
}

// ------------------------------------------------------------------ PhaseField
PhaseField::~PhaseField() {
  if (mDense) cupf_dense_destroy(mDense);
  delete qois;
}

// The reference-named entry points: each runs its step unless an earlier one failed.
void PhaseField::parseInputParams(const std::string fileName) {
  if (!failed()) parseInputImpl(fileName);
}
void PhaseField::cpuSetup(MPIsetting* mpiManager) {
  if (!failed()) cpuSetupImpl(mpiManager);
}
void PhaseField::initField() {
  if (!failed()) initFieldImpl();
}
void PhaseField::cudaSetup() {
  if (!failed()) denseCudaSetup();
}
void PhaseField::evolve() {
  if (!failed()) denseEvolve();
}
void PhaseField::OutputQoIs() {
  if (!failed()) outputQoIsImpl();
}
void PhaseField::OutputField(int currentStep) {
  if (!failed()) outputFieldImpl(currentStep);
}
void APTPhaseField::cudaSetup() {
  if (!failed()) aptCudaSetup();
}
void APTPhaseField::evolve() {
  if (!failed()) aptEvolve();
}

void MPIsetting::printMPIsetting() const {
  std::printf("total/x/y/z number of processors: %d/%d/%d/%d\n", numProcessor, numProcessorX,
              numProcessorY, numProcessorZ);
  std::printf("rank/x/y/z processor IDs: %d/%d/%d/%d\n", rank, processorIDX, processorIDY,
              processorIDZ);
}

// MPIsetting1D/2D::domainPartition (MPIsetting.cpp:33-51) for rank 0 of 1
void MPIsetting1D::domainPartition() {
  numProcessorX = numProcessor;
  numProcessorY = numProcessorZ = 1;
  processorIDX = rank;
  processorIDY = processorIDZ = 0;
}

void MPIsetting2D::domainPartition() {
  numProcessorX = numProcessor;
  numProcessorY = numProcessorZ = 1;
  processorIDX = rank;
  processorIDY = processorIDZ = 0;
}

static QoiGrid qoi_grid_of(const GlobalConstants& p) {
  QoiGrid g;
  g.fnx = p.fnx;
  g.fny = p.fny;
  g.fnz = p.fnz;
  g.num_theta = p.num_theta;
  g.nts = p.nts;
  g.num_nodes = p.num_nodes;
  return g;
}
QOILine::QOILine(const GlobalConstants& params) : QOILine(qoi_grid_of(params)) {}
QOI3D::QOI3D(const GlobalConstants& params) : QOI3D(qoi_grid_of(params)) {}

bool PhaseField::setErr(const std::string& e) {
  if (mErr.empty()) {
    mErr = e;
    std::fprintf(stderr, "cupf PhaseField: %s\n", e.c_str());
  }
  return false;
}

bool PhaseField::check(cupf_status st, const char* what) {
  if (st == CUPF_OK) return true;
  return setErr(std::string(what) + ": " + cupf_last_error());
}

QoiGrid PhaseField::qoiGrid() const {
  QoiGrid g;
  g.fnx = fnx;
  g.fny = fny;
  g.fnz = fnz;
  g.num_theta = params.num_theta;
  g.nts = params.nts;
  g.num_nodes = params.num_nodes;
  return g;
}

// PhaseField::parseInputParams (PhaseFieldCpu.cpp:17-256)
bool PhaseField::parseInputImpl(const std::string& fileName) {
  const DesignSettingData* ds = GetSetDesignSetting();
  std::ifstream f(fileName);
  if (!f.good()) return setErr("cannot open input file " + fileName);
  GlobalConstants& p = params;
  std::string line;
  while (std::getline(f, line)) {
    getParam(line, "Tmelt", p.Tmelt);
    getParam(line, "Dh", p.Dh);
    getParam(line, "L_cp", p.L_cp);
    getParam(line, "beta0", p.beta0);
    getParam(line, "GT", p.GT);
    getParam(line, "mu_k", p.mu_k);
    getParam(line, "kin_delta", p.kin_delta);
    getParam(line, "delta", p.delta);
    getParam(line, "underCoolingRate0", p.underCoolingRate0);
    getParam(line, "nuc_Nmax0", p.nuc_Nmax0);
    getParam(line, "undcool_mean", p.undcool_mean);
    getParam(line, "undcool_std", p.undcool_std);
    getParam(line, "nuc_rad", p.nuc_rad);
    getParam(line, "eps", p.eps);
    getParam(line, "dx", p.dx);
    getParam(line, "W0", p.W0);
    getParam(line, "asp_ratio_yx", p.asp_ratio_yx);
    getParam(line, "asp_ratio_zx", p.asp_ratio_zx);
    getParam(line, "moving_ratio", p.moving_ratio);
    getParam(line, "Lx", p.lxd);
    getParam(line, "eta", p.eta);
    getParam(line, "nts", p.nts);
    getParam(line, "ictype", p.ictype);
    getParam(line, "noi_period", p.noi_period);
    getParam(line, "haloWidth", p.haloWidth);
    getParam(line, "xmin", p.xmin);
    getParam(line, "ymin", p.ymin);
    getParam(line, "zmin", p.zmin);
    getParam(line, "nx", p.Nx);
    getParam(line, "ny", p.Ny);
    getParam(line, "nz", p.Nz);
    getParam(line, "nt", p.Nt);
    getParam(line, "cfl", p.cfl);
    getParam(line, "preMt", p.preMt);
    getParam(line, "NUM_PF", p.NUM_PF);  // slot count (the reference fixes it at compile time)
  }
  mac.Nx = p.Nx;
  mac.Ny = p.Ny;
  mac.Nz = p.Nz;
  mac.Nt = p.Nt;
  if (mac.Nx < 2 || mac.Ny < 2 || mac.Nz < 2 || mac.Nt < 2)
    return setErr("macro grid nx, ny, nz, nt must each be >= 2");
  mac.X_mac.assign(mac.Nx, 0.f);
  mac.Y_mac.assign(mac.Ny, 0.f);
  mac.Z_mac.assign(mac.Nz, 0.f);
  mac.t_mac.assign(mac.Nt, 0.f);
  mac.psi_mac.assign((size_t)mac.Nx * mac.Ny * mac.Nz, 0.f);
  mac.T_3D.assign((size_t)mac.Nx * mac.Ny * mac.Nz * mac.Nt, 0.f);
  const std::string& d = mac.folder;
  struct FF {
    const char* name;
    float* dst;
    int n;
  };
  const FF floats[] = {{"x.txt", mac.X_mac.data(), mac.Nx},
                       {"y.txt", mac.Y_mac.data(), mac.Ny},
                       {"z.txt", mac.Z_mac.data(), mac.Nz},
                       {"t.txt", mac.t_mac.data(), mac.Nt},
                       {"psi.txt", mac.psi_mac.data(), mac.Nx * mac.Ny * mac.Nz},
                       {"G.txt", &p.G, 1},
                       {"Rmax.txt", &p.R, 1},
                       {"V.txt", &p.V, 1},
                       {"UC.txt", &p.underCoolingRate, 1},
                       {"Nmax.txt", &p.nuc_Nmax, 1},
                       {"z0.txt", &p.z0, 1},
                       {"r0.txt", &p.r0, 1},
                       {"x0.txt", &p.x0, 1},
                       {"top.txt", &p.top, 1},
                       {"angle.txt", &p.angle, 1},
                       {"min_angle.txt", &p.min_angle, 1},
                       {"order.txt", &p.order, 1}};
  for (const FF& ff : floats)
    if (read_input(d + "/" + ff.name, ff.dst, ff.n) < 1)
      return setErr("cannot read forcing file " + d + "/" + ff.name);
  if (read_input(d + "/NG.txt", &p.num_theta, 1) < 1) return setErr("cannot read NG.txt");
  if (read_input(d + "/NN.txt", &p.num_nodes, 1) < 1) p.num_nodes = 0;
  p.nuc_Nmax0 = p.nuc_Nmax;
  if (p.num_theta < 1) return setErr("NG.txt must hold a grain count >= 1");
  const int nth = 2 * p.num_theta + 1;
  mac.theta_arr.assign(nth, 0.f);
  mac.cost.assign(nth, 0.f);
  mac.sint.assign(nth, 0.f);
  if (read_input(d + "/theta.txt", mac.theta_arr.data(), nth) < nth) {
    // no two-angle file: orientations as unit quaternions (w, x, y, z per grain)
    std::vector<float> qf(4 * (size_t)p.num_theta);
    if (read_input(d + "/quaternions.txt", qf.data(), (int)qf.size()) < (int)qf.size())
      return setErr("theta.txt must hold 2*NG+1 angles (or quaternions.txt 4*NG values)");
    std::vector<double> q(qf.begin(), qf.end());
    if (cupf_host_quaternions_to_angles(p.num_theta, q.data(), mac.theta_arr.data()) != 0)
      return setErr("quaternions.txt holds a zero or non-finite quaternion");
  }
  // Temp.h5:/Temp (the 4-D temperature table, read only by nucleation): read from
  // Temp.txt (one value per line) when present, else zeros.
  read_input(d + "/Temp.txt", mac.T_3D.data(), (int)mac.T_3D.size());

  if (p.R < 0.3) {  // float R compared with double literals, as the reference does
    p.cfl *= 2;
    p.underCoolingRate0 /= 2;
  }
  if (p.R > 0.3 && p.R < 1) {
    p.cfl = (float)(p.cfl * 1.5);
    p.underCoolingRate0 = (float)(p.underCoolingRate0 / 1.5);
  }
  const float dxd = p.dx * p.W0;
  p.c_infm = p.c_infty * p.m_slope;
  p.Tliq = p.Tmelt - p.c_infm;
  p.d0 = p.GT / p.L_cp;
  p.beta0 = (float)(1.0 / (p.mu_k * p.L_cp));
  p.lamd = (float)(0.8839 * p.W0 / p.d0);
  p.tau0 = (float)(p.beta0 * p.lamd * p.W0 / 0.8839);
  p.beta0_tilde = p.beta0 * p.W0 / p.tau0;
  p.dt = p.cfl * p.dx * p.beta0_tilde;
  p.hi = (float)(1.0 / p.dx);
  p.sqrt2 = (float)std::sqrt(2.0);
  p.a_s = (float)(1 - 3.0 * p.delta);
  p.epsilon = (float)(4.0 * p.delta / p.a_s);
  p.dt_sqrt = (float)std::sqrt(p.dt);
  p.nx = (int)std::round(p.lxd / p.dx / p.W0);
  p.ny = (int)std::round(p.asp_ratio_yx * p.nx);
  p.nz = ds->useLineConfig ? (int)std::round(p.moving_ratio * p.nx)
                           : (int)std::round(p.asp_ratio_zx * p.nx);
  p.nz_full = (int)std::round(p.asp_ratio_zx * p.nx);
  p.lxd = p.nx * dxd;
  p.lyd = p.ny * dxd;
  p.lzd = p.nz * dxd;
  p.Mt = (int)(mac.t_mac[mac.Nt - 1] / p.tau0 / p.dt);
  p.Mt = (p.Mt / 2) * 2;
  if (p.nts < 1) return setErr("nts must be >= 1");
  int kts = p.Mt / p.nts;
  kts = (kts / 2) * 2;
  p.Mt = kts * p.nts;
  p.tmax = p.tau0 * p.dt * p.Mt;
  p.pts_cell = (float)(int)(p.nuc_rad / dxd);
  p.bcX = ds->bcX;
  p.bcY = ds->bcY;
  p.bcZ = ds->bcZ;
  const std::string& in = ds->inputFile;
  if (in == "line.py") p.thermalType = 1;
  else if (in == "cylinder.py") p.thermalType = 2;
  else if (in == "cone.py") p.thermalType = 3;
  else if (in == "paraboloid.py") {
    p.thermalType = 4;
    if (read_input(d + "/mp_len.txt", &p.mp_len, 1) < 1) return setErr("cannot read mp_len.txt");
  } else p.thermalType = 0;
  return true;
}

// PhaseField::cpuSetup (PhaseFieldCpu.cpp:258-374), single rank
bool PhaseField::cpuSetupImpl(MPIsetting* mpiManager) {
  // one process drives the whole domain (the reference splits it into MPI slabs)
  if (mpiManager && mpiManager->numProcessor != 1)
    return setErr("one process drives the whole domain: " +
                  std::to_string(mpiManager->numProcessor) + " ranks given");
  GlobalConstants& p = params;
  if (p.haloWidth != 1) return setErr("haloWidth must be 1");
  const float dxd = p.dx * p.W0;
  const float xmin_loc = p.xmin + 0 * (p.nx * dxd);
  const float ymin_loc = p.ymin + 0 * (p.ny * dxd);
  const float zmin_loc = p.zmin + 0 * (p.nz * dxd);
  p.fnx = p.nx + 1 + 2 * p.haloWidth;
  p.fny = p.ny + 1 + 2 * p.haloWidth;
  p.fnz = p.nz + 1 + 2 * p.haloWidth;
  p.fnz_f = p.nz_full + 1 + 2 * p.haloWidth;
  fnx = p.fnx;
  fny = p.fny;
  fnz = p.fnz;
  fnz_f = p.fnz_f;
  if (fnx < 4 || fny < 4 || fnz < 4) return setErr("grid too small");
  p.length = (long long)fnx * fny * fnz;
  p.full_length = (long long)fnx * fny * fnz_f;
  length = p.length;
  full_length = p.full_length;
  x.resize(fnx);
  y.resize(fny);
  z.resize(fnz);
  z_full.resize(fnz_f);
  for (int i = 0; i < fnx; i++) x[i] = (i - p.haloWidth) * dxd + xmin_loc;
  for (int i = 0; i < fny; i++) y[i] = (i - p.haloWidth) * dxd + ymin_loc;
  for (int i = 0; i < fnz; i++) z[i] = (i - p.haloWidth) * dxd + zmin_loc;
  for (int i = 0; i < fnz_f; i++) z_full[i] = (i - p.haloWidth) * dxd + zmin_loc;
  psi.assign(length, 0.f);
  phi.assign(length, 0.f);
  alpha.assign(length, 0);
  if (GetSetDesignSetting()->useLineConfig) alpha_i_full.assign(full_length, 0);
  return true;
}

// PhaseField::initField (PhaseFieldCpu.cpp:377-459)
bool PhaseField::initFieldImpl() {
  GlobalConstants& p = params;
  const DesignSettingData* ds = GetSetDesignSetting();
  for (int i = 0; i < 2 * p.num_theta + 1; i++) {
    mac.sint[i] = sinf(mac.theta_arr[i]);
    mac.cost[i] = cosf(mac.theta_arr[i]);
  }
  const bool use_sub = !ds->pureNucleation && ds->useLineConfig;
  if (use_sub) {
    const int n = (p.nx + 1) * (p.ny + 1);
    mac.alpha_mac.assign(n, 0);
    if (read_input(mac.folder + "/alpha.txt", mac.alpha_mac.data(), n) < n)
      return setErr("alpha.txt must hold (nx+1)*(ny+1) grain ids");
  }
  const float Dx = mac.X_mac[mac.Nx - 1] - mac.X_mac[mac.Nx - 2];
  const float Dy = mac.Y_mac[mac.Ny - 1] - mac.Y_mac[mac.Ny - 2];
  const float Dz = mac.Z_mac[mac.Nz - 1] - mac.Z_mac[mac.Nz - 2];
  const int h = p.haloWidth;
  const float* pm = mac.psi_mac.data();
  const int Nx = mac.Nx, Ny = mac.Ny;
  for (long long id = 0; id < length; id++) {
    const int k = (int)(id / ((long long)fnx * fny));
    const long long k_r = id - (long long)k * fnx * fny;
    const int j = (int)(k_r / fnx);
    const int i = (int)(k_r % fnx);
    if (i > h - 1 && i < fnx - h && j > h - 1 && j < fny - h && k > h - 1 && k < fnz - h) {
      int kx = (int)((x[i] - mac.X_mac[0]) / Dx);
      float delta_x = (x[i] - mac.X_mac[0]) / Dx - kx;
      int ky = (int)((y[j] - mac.Y_mac[0]) / Dy);
      float delta_y = (y[j] - mac.Y_mac[0]) / Dy - ky;
      int kz = (int)((z[k] - mac.Z_mac[0]) / Dz);
      float delta_z = (z[k] - mac.Z_mac[0]) / Dz - kz;
      if (kx == mac.Nx - 1) { kx = mac.Nx - 2; delta_x = 1.0f; }
      if (ky == mac.Ny - 1) { ky = mac.Ny - 2; delta_y = 1.0f; }
      if (kz == mac.Nz - 1) { kz = mac.Nz - 2; delta_z = 1.0f; }
      if (kx < 0 || ky < 0 || kz < 0 || kx > mac.Nx - 2 || ky > mac.Ny - 2 || kz > mac.Nz - 2)
        return setErr("grid point outside the macro grid of psi.txt");
      const long long o = kx + (long long)ky * Nx + (long long)kz * Nx * Ny;
      const long long on = kx + (long long)ky * Nx + (long long)(kz + 1) * Nx * Ny;
      float v = ((1.0f - delta_x) * (1.0f - delta_y) * pm[o] + (1.0f - delta_x) * delta_y * pm[o + Nx] +
                 delta_x * (1.0f - delta_y) * pm[o + 1] + delta_x * delta_y * pm[o + Nx + 1]) *
                    (1.0f - delta_z) +
                ((1.0f - delta_x) * (1.0f - delta_y) * pm[on] + (1.0f - delta_x) * delta_y * pm[on + Nx] +
                 delta_x * (1.0f - delta_y) * pm[on + 1] + delta_x * delta_y * pm[on + Nx + 1]) *
                    delta_z;
      psi[id] = v / p.W0;
      phi[id] = tanhf(psi[id] / p.sqrt2);
      if (phi[id] > kLS && use_sub) {
        const int a = mac.alpha_mac[(long long)(j - 1) * (fnx - 2 * h) + (i - 1)];
        if (a < 1 || a > p.num_theta) {
          std::ostringstream m;
          m << "alpha out of bounds at " << (j - 1) * (fnx - 2 * h) + (i - 1) << ": " << a;
          return setErr(m.str());
        }
        alpha[id] = a;
      } else {
        alpha[id] = 0;
      }
    } else {
      psi[id] = 0.0f;
      phi[id] = 0.0f;
      alpha[id] = 0;
    }
  }
  // A 3-D run that is neither a line run nor pure nucleation may start from a
  // full grain-id field: alpha3D.h5:/alpha of the additive-manufacturing driver
  // (AdditiveManufacturing/PhaseFieldCpu.cpp:430-447), read here from
  // alpha3D.txt, `length` ids in the grid layout (halos included), replacing the
  // zeros above.  Without the file the ids stay 0, as in 3DgrainMPI.
  if (!ds->pureNucleation && !ds->useLineConfig) {
    const int n = read_input(mac.folder + "/alpha3D.txt", alpha.data(), (int)length);
    if (n >= 0 && n < length) return setErr("alpha3D.txt must hold fnx*fny*fnz grain ids");
  }
  if (std::fabs(p.order - 100.0f) < 1e-3f) {
    if (read_input(mac.folder + "/statTemp.txt", mac.psi_mac.data(), (int)mac.psi_mac.size()) < 1)
      return setErr("order 100 needs statTemp.txt");
  }
  return true;
}

static std::string to_stringp(float v, int n) {
  std::ostringstream out;
  out.precision(n);
  out << std::fixed << v;
  return out.str();
}

// output file stem (PhaseFieldCpu.cpp:476-488)
std::string PhaseField::outputBaseName() const {
  const DesignSettingData* ds = GetSetDesignSetting();
  const GlobalConstants& p = params;
  std::string grainType =
      ds->includeNucleation
          ? "Mixed_density" + std::to_string(p.nuc_Nmax) + "_grains" +
                std::to_string(qois ? qois->mNumActiveGrains : 0)
          : "Epita_grains" + std::to_string(p.num_theta);
  return ds->inputFile.substr(0, 4) + "seed" + std::to_string(p.seed_val) + "_lxd" +
         std::to_string(p.lxd) + "_G" + to_stringp(p.G, 3) + "_Rmax" + to_stringp(p.R, 3) + "_V" +
         to_stringp(p.V, 3) + "_angle" + to_stringp(p.angle, 3) + "_minangle" +
         to_stringp(p.min_angle, 3) + "_order" + std::to_string((int)p.order) + grainType;
}

// The line-configuration junction search with its neighbourhood test on the
// device: the frames' tip layers of the full map go to
// cupf_line_junction_candidates, and the records are built for the candidate
// cells only (the same records, in the same order, as the full host scan).
bool PhaseField::lineJunctions(QOILine* q, const QoiGrid& g, const int* a) {
  const int nf = g.nts + 1;
  const long long plane = (long long)fnx * fny;
  const std::vector<int>& tip_y = q->mQoIVectorIntData["tip_y"];
  if ((int)tip_y.size() < nf) return setErr("line QoIs: fewer tip heights than frames");
  std::vector<int> layers((size_t)plane * nf);
  for (int kt = 0; kt < nf; ++kt) {
    if (tip_y[kt] < 0 || (long long)(tip_y[kt] + 1) * plane > full_length)
      return setErr("line QoIs: tip height outside the full map");
    std::memcpy(layers.data() + (size_t)plane * kt, a + (size_t)plane * tip_y[kt],
                sizeof(int) * (size_t)plane);
  }
  std::vector<long long> cells;
  int64_t cap = 1 << 16, count = 0;
  for (;;) {
    cells.assign((size_t)cap, 0);
    if (!check(cupf_line_junction_candidates(device, fnx, fny, layers.data(), nf,
                                             reinterpret_cast<int64_t*>(cells.data()), cap, &count),
               "cupf_line_junction_candidates"))
      return false;
    if (count <= cap) break;
    cap = count;
  }
  q->searchJunctionsOnCells(g, a, cells.data(), (long long)count);
  return true;
}

// PhaseField::OutputQoIs (PhaseFieldCpu.cpp:464-520): junction search, then the
// coordinates, geometry scalars and every QoI vector, one 1-D dataset each.
bool PhaseField::outputQoIsImpl() {
  const DesignSettingData* ds = GetSetDesignSetting();
  if (!qois) return setErr("no QoI object");
  const QoiGrid g = qoiGrid();
  std::vector<long long> cells;
  std::vector<unsigned char> distinct;
  QOI3D* q3 = dynamic_cast<QOI3D*>(qois);
  QOILine* ql = dynamic_cast<QOILine*>(qois);
  if (ds->useLineConfig && ql) {
    if (!lineJunctions(ql, g, alpha_i_full.data())) return false;
  } else if (ds->useLineConfig)
    qois->searchJunctionsOnImage(g, alpha_i_full.data());
  else if (q3 && deviceJunctionCandidates(cells, distinct))
    q3->searchJunctionsOnCells(g, alpha.data(), cells.data(), (long long)cells.size(),
                               distinct.data());
  else
    qois->searchJunctionsOnImage(g, alpha.data());
  const std::string name = outputBaseName() + "_walltime" + std::to_string(params.walltime) +
                           "_frames" + std::to_string(params.nts) + "_Mt" +
                           std::to_string(params.Mt) + "_rank0";
  ArrayFile w;
  w.add("x_coordinates", x);
  w.add("y_coordinates", y);
  w.add("z_coordinates", z_full);
  w.add("angles", mac.theta_arr);
  w.add("r0", std::vector<float>{params.r0});
  w.add("z0", std::vector<float>{params.z0});
  w.add("x0", std::vector<float>{params.x0});
  w.add("top", std::vector<float>{params.top});
  w.add("angle", std::vector<float>{params.angle});
  w.add("V", std::vector<float>{params.V});
  for (auto& q : qois->mQoIVectorFloatData) w.add(q.first, q.second);
  for (auto& q : qois->mQoIVectorIntData) w.add(q.first, q.second);
  const std::string path = ds->outputFolder + "/" + name;
  if (!w.write(path)) return setErr("cannot write " + path + w.extension());
  return true;
}

// PhaseField::OutputField (PhaseFieldCpu.cpp:522-573): the argmax grain map.
bool PhaseField::outputFieldImpl(int currentStep) {
  const DesignSettingData* ds = GetSetDesignSetting();
  const std::string name = outputBaseName() + "_frames" + std::to_string(params.nts) + "_Mt" +
                           std::to_string(params.Mt) + "_rank0_time" +
                           std::to_string(currentStep);
  ArrayFile w;
  w.add("x_coordinates", x);
  w.add("y_coordinates", y);
  w.add("z_coordinates", z_full);
  w.add("angles", mac.theta_arr);
  if (ds->useLineConfig) w.add("alpha", alpha_i_full);
  else w.add("alpha", alpha);
  const std::string path = ds->outputFolder + "/" + name;
  if (!w.write(path)) return setErr("cannot write " + path + w.extension());
  return true;
}

// ------------------------------------------------------------------ APTPhaseField
APTPhaseField::~APTPhaseField() {
  if (mHandle) cupf_apt_destroy(mHandle);
}


cupf_apt_params PhaseField::deviceParams() const {
  const GlobalConstants& p = params;
  cupf_apt_params d;
  std::memset(&d, 0, sizeof(d));
  d.fnx = fnx;
  d.fny = fny;
  d.fnz = fnz;
  d.num_pf = p.NUM_PF;
  d.num_theta = p.num_theta;
  d.bcX = p.bcX;
  d.bcY = p.bcY;
  d.bcZ = p.bcZ;
  d.thermalType = p.thermalType;
  d.Nx = mac.Nx;
  d.Ny = mac.Ny;
  d.Nz = mac.Nz;
  d.Nt = mac.Nt;
  d.kin_delta = p.kin_delta;
  d.eps = p.eps;
  d.G = p.G;
  d.z0 = p.z0;
  d.underCoolingRate = p.underCoolingRate;
  d.underCoolingRate0 = p.underCoolingRate0;
  d.L_cp = p.L_cp;
  d.hi = p.hi;
  d.lamd = p.lamd;
  d.dt = p.dt;
  d.tau0 = p.tau0;
  d.lyd = p.lyd;
  d.lzd = p.lzd;
  d.r0 = p.r0;
  d.x0 = p.x0;
  d.angle = p.angle;
  d.V = p.V;
  d.mp_len = p.mp_len;
  d.order = p.order;
  d.dx = p.dx;
  d.W0 = p.W0;
  d.undcool_mean = p.undcool_mean;
  d.undcool_std = p.undcool_std;
  d.nuc_Nmax = p.nuc_Nmax;
  d.nuc_Nmax0 = p.nuc_Nmax0;
  d.nuc_rad = p.nuc_rad;
  d.sqrt2 = p.sqrt2;
  d.pts_cell = (int)p.pts_cell;
  d.seed = p.seed_val;
  d.haloWidth = p.haloWidth;
  return d;
}

// APTPhaseField::cudaSetup (APTPhaseField.cu:569-637)
bool APTPhaseField::aptCudaSetup() {
  NUM_PF = params.NUM_PF;
  cupf_apt_params d = deviceParams();
  cupf_apt_inputs in;
  std::memset(&in, 0, sizeof(in));
  in.x = x.data();
  in.y = y.data();
  in.z = z.data();
  in.sint = mac.sint.data();
  in.cost = mac.cost.data();
  in.X_mac = mac.X_mac.data();
  in.Y_mac = mac.Y_mac.data();
  in.Z_mac = mac.Z_mac.data();
  in.t_mac = mac.t_mac.data();
  in.psi_mac = mac.psi_mac.data();
  in.T_3D = mac.T_3D.data();
  return check(cupf_apt_create(&d, &in, device, precision, &mHandle), "cupf_apt_create");
}

// The 19-point neighbourhood test of QOI3D::searchJunctionsOnImage on the device,
// over the argmax map of the last collect (the map `alpha` holds).
bool APTPhaseField::deviceJunctionCandidates(std::vector<long long>& cells,
                                             std::vector<unsigned char>& distinct) {
  if (!mHandle) return false;
  distinct.assign((size_t)(fnx - 2) * (fny - 2) * (fnz - 2), 0);
  int64_t cap = 1 << 16, count = 0;
  for (;;) {
    cells.assign((size_t)cap, 0);
    if (cupf_apt_junction_candidates(mHandle, reinterpret_cast<int64_t*>(cells.data()), cap, &count,
                                     distinct.data()) != CUPF_OK)
      return false;
    if (count <= cap) break;
    cap = count;
  }
  cells.resize((size_t)count);
  return true;
}

bool APTPhaseField::collectToHost(bool clear) {
  return check(cupf_apt_collect(mHandle, clear ? 1 : 0, nullptr, alpha.data()), "cupf_apt_collect");
}

// APTPhaseField::getLineQoIs (APTPhaseField.cu:655-676)
bool APTPhaseField::getLineQoIs(MovingDomain* md) {
  const float loc = (md->move_count + md->lowsl - 1) * params.W0 * params.dx;
  const float threshold = params.z0 + params.top * (md->samples + 1) / params.nts;
  if (loc > threshold) {
    if (!collectToHost(true)) return false;
    if (!check(cupf_apt_get_archive(mHandle, 0, nullptr, md->loss_area_host.data()),
               "cupf_apt_get_archive"))
      return false;
    if (!check(cupf_apt_get_z(mHandle, z.data()), "cupf_apt_get_z")) return false;
    md->cur_tip = 0;
    qois->calculateLineQoIs(qoiGrid(), md->cur_tip, alpha.data(), md->samples + 1, z.data(),
                            md->loss_area_host.data(), md->move_count);
    md->samples += 1;
  }
  return true;
}

// APTPhaseField::moveDomain (APTPhaseField.cu:678-697)
bool APTPhaseField::moveDomain(MovingDomain* md) {
  int moved = 0;
  if (!check(cupf_apt_move_domain(mHandle, &md->tip_front, md->tip_thres, &md->move_count, &moved),
             "cupf_apt_move_domain"))
    return false;
  md->lowsl = 1;
  if (!collectToHost(false)) return false;
  qois->sampleHeights(md->lowsl, alpha.data(), fnx, fny, fnz);
  return true;
}

// APTPhaseField::evolve (APTPhaseField.cu:710-946) without MPI.  With -n the
// liquid-start phase (:779-816) runs first when preMt > 0: from an all-liquid
// state, preMt steps at the liquid-start undercooling with a nucleation pass after
// every odd step; the grains it grew then label the solid cells of the initial
// phase field (APTini_PF from phi_old and the collected alpha, :820-822).  The
// main loop nucleates after every odd step (:866-870).  The reference's update at
// t = 0 on the freshly emptied state (:776) changes nothing and is not issued.
// Without -n, preMt is ignored: the reference's liquid-start phase launches
// add_nucl on the status and generator arrays that only -n allocates (:733-745).
bool APTPhaseField::aptEvolve() {
  const DesignSettingData* ds = GetSetDesignSetting();
  const bool nucl = ds->includeNucleation;
  MovingDomain md;
  if (nucl && params.preMt > 0) {
    const std::vector<float> liquid((size_t)length, -1.0f);
    if (!check(cupf_apt_init_from_argmax(mHandle, liquid.data(), alpha.data()), "init") ||
        !check(cupf_apt_nucl_init(mHandle), "nucleation init") ||
        !check(cupf_apt_nucl_reset(mHandle), "nucleation reset"))
      return false;
    for (int kt = 0; kt < params.preMt / 2; kt++) {
      if (!check(cupf_apt_step(mHandle, 1, 1), "cupf_apt_step") ||
          !check(cupf_apt_nucleate(mHandle, 1, nullptr), "cupf_apt_nucleate") ||
          !check(cupf_apt_step(mHandle, 1, 1), "cupf_apt_step"))
        return false;
    }
    if (!collectToHost(true)) return false;  // alpha_m of the grown grains
  }
  if (!check(cupf_apt_init_from_argmax(mHandle, phi.data(), alpha.data()), "init")) return false;
  if (nucl && params.preMt <= 0 && !check(cupf_apt_nucl_init(mHandle), "nucleation init"))
    return false;
  if (!collectToHost(true)) return false;
  if (ds->useLineConfig) {
    md.allocateMovingDomain(params.num_theta, fnz);
    qois->calculateLineQoIs(qoiGrid(), md.cur_tip, alpha.data(), 0, z.data(),
                            md.loss_area_host.data(), md.move_count);
  } else if (!nucl) {
    qois->calculateQoIs(qoiGrid(), alpha.data(), 0);
  }
  const int qoikts = params.Mt / params.nts;
  const int fieldkts = ds->save3DField > 0 ? params.Mt / ds->save3DField : 100000000;
  int kt_max = params.Mt / 2 + (ds->useLineConfig ? 1000 : 0);
  auto t0 = std::chrono::steady_clock::now();
  int kt = 0;
  for (kt = 0; kt < kt_max; kt++) {
    if (!check(cupf_apt_step(mHandle, 1, 0), "cupf_apt_step")) return false;
    if (nucl && !check(cupf_apt_nucleate(mHandle, 0, nullptr), "cupf_apt_nucleate")) return false;
    if (ds->useLineConfig) {
      if (!getLineQoIs(&md)) return false;
      if (md.samples == params.nts) break;
      if ((2 * kt + 2) % kTIPP == 0 && !moveDomain(&md)) return false;
    } else if (qoikts > 0 && (2 * kt + 2) % qoikts == 0) {
      if (!collectToHost(false)) return false;
      qois->calculateQoIs(qoiGrid(), alpha.data(), (2 * kt + 2) / qoikts);
    }
    if (fieldkts > 0 && (2 * kt + 2) % fieldkts == 0) {
      if (!collectToHost(true)) return false;
      if (ds->useLineConfig) {
        if (!check(cupf_apt_get_archive(mHandle, fnz_f, alpha_i_full.data(), nullptr), "archive"))
          return false;
        std::memcpy(alpha_i_full.data() + (size_t)md.move_count * fnx * fny, alpha.data(),
                    sizeof(int) * std::min<long long>(length, full_length - (long long)md.move_count * fnx * fny));
      }
      if (!outputFieldImpl(2 * kt + 2)) return false;
    }
    if (!check(cupf_apt_step(mHandle, 1, 0), "cupf_apt_step")) return false;
  }
  if (!check(cupf_apt_sync(mHandle, 0), "sync")) return false;
  params.walltime =
      (int)std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  params.Mt = 2 * kt;
  return true;
}

// PhaseField::cudaSetup (PhaseField.cu:431-493): the full-PF solver, one phi field
// per grain (params.NUM_PF = params.num_theta, :440).
bool PhaseField::denseCudaSetup() {
  params.NUM_PF = params.num_theta;
  NUM_PF = params.NUM_PF;
  cupf_apt_params d = deviceParams();
  cupf_apt_inputs in;
  std::memset(&in, 0, sizeof(in));
  in.x = x.data();
  in.y = y.data();
  in.z = z.data();
  in.sint = mac.sint.data();
  in.cost = mac.cost.data();
  return check(cupf_dense_create(&d, &in, params.R, device, &mDense), "cupf_dense_create");
}

// PhaseField::evolve (PhaseField.cu:495-632) without MPI: line QoIs every Mt/nts
// steps and the moving-domain check every TIPP steps, whatever the -l flag (the
// full-PF evolve does both unconditionally).  The reference's last update of the
// loop (:604) writes a buffer nothing reads afterwards (the final collect_PF at
// :617 reads the other one), so the loop stops before it.
bool PhaseField::denseEvolve() {
  const DesignSettingData* ds = GetSetDesignSetting();
  if (ds && ds->includeNucleation) return setErr("the full-PF mode has no nucleation");
  if (!mDense) return setErr("cudaSetup has not run");
  MovingDomain md;
  md.allocateMovingDomain(params.num_theta, fnz);
  md.tip_thres = (int)((1 - 0.2) * fnz);  // (1-BLANK)*fnz, PhaseField.cu:517
  if (!check(cupf_dense_init_from_argmax(mDense, phi.data(), alpha.data()), "init")) return false;
  if (!check(cupf_dense_prestep(mDense), "prestep")) return false;
  md.cur_tip = 1;
  qois->calculateLineQoIs(qoiGrid(), md.cur_tip, alpha.data(), 0, z.data(),
                          md.loss_area_host.data(), md.move_count);
  const int kts = params.nts > 0 ? params.Mt / params.nts : 0;
  const int kt_max = params.Mt / 2;
  auto t0 = std::chrono::steady_clock::now();
  for (int kt = 0; kt < kt_max; kt++) {
    if (!check(cupf_dense_step(mDense, 1), "cupf_dense_step")) return false;
    if (kts > 0 && (2 * kt + 2) % kts == 0) {
      if (!check(cupf_dense_collect(mDense, 1, nullptr, alpha.data()), "collect") ||
          !check(cupf_dense_get_archive(mDense, 0, nullptr, md.loss_area_host.data()), "archive") ||
          !check(cupf_dense_get_z(mDense, z.data()), "z"))
        return false;
      md.cur_tip = 0;
      qois->calculateLineQoIs(qoiGrid(), md.cur_tip, alpha.data(), (2 * kt + 2) / kts, z.data(),
                              md.loss_area_host.data(), md.move_count);
    }
    if ((2 * kt + 2) % kTIPP == 0) {
      int moved = 0;
      if (!check(cupf_dense_move_domain(mDense, &md.tip_front, md.tip_thres, &md.move_count, &moved),
                 "cupf_dense_move_domain"))
        return false;
    }
    if (kt + 1 < kt_max && !check(cupf_dense_step(mDense, 1), "cupf_dense_step")) return false;
  }
  if (!check(cupf_dense_collect(mDense, 1, phi.data(), alpha.data()), "collect")) return false;
  if (fnz_f > 0 && !alpha_i_full.empty()) {
    if (!check(cupf_dense_get_archive(mDense, fnz_f, alpha_i_full.data(), nullptr), "archive"))
      return false;
    const long long off = (long long)md.move_count * fnx * fny;
    if (off < full_length)
      std::memcpy(alpha_i_full.data() + off, alpha.data(),
                  sizeof(int) * std::min<long long>(length, full_length - off));
  }
  if (!check(cupf_dense_sync(mDense, 0), "sync")) return false;
  params.walltime =
      (int)std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return true;
}

}  // namespace cupf_host
