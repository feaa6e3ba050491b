// phase_field.h — C++ driver of the APT solver with the reference's surface.
//
// Class and method names, call order and input semantics follow the reference
// driver (3DgrainMPI/main.cpp:15-77, PhaseField.h:11-59, APTPhaseField.h:11-30,
// DesignSettingData.h, MovingDomain.h, ThermalInputData.h); the device work
// goes through the C ABI of include/cupf.h (include/cupf_dense.h for -a).  One
// process drives one GPU (the reference's MPI slabs are replaced by a
// whole-domain solver).
#pragma once

#include <memory>
#include <string>
#include <vector>

#include "../../include/cupf.h"
#include "../../include/cupf_dense.h"
#include "qoi.h"

namespace cupf_host {

// CLI options (DesignSettingData.cpp:21-78): argv[1] = input file name,
// -s seed, -b XYZ boundary digits (1 = periodic), -l line configuration,
// -n {1: pure nucleation / liquid start, 2: nucleation}, -a full-PF mode,
// -m MPI dimension (accepted, single rank), -d N field snapshots, -o output
// directory, -f forcing folder prefix.  -d takes its argument here (the
// reference declares it without one in the optstring but reads optarg).
class DesignSettingData {
 public:
  bool getOptions(int argc, char** argv, std::string* err = nullptr);

  bool useMPI = false;
  bool useLineConfig = false;
  bool includeNucleation = false;
  bool pureNucleation = false;
  bool useAPT = true;
  int save3DField = 1;
  int mpiDim = 1;
  int seedValue = 0;
  int givenBC = 0, bcX = 0, bcY = 0, bcZ = 0;
  std::string inputFile;
  std::string thermalInputFolder = "forcing/case";
  std::string outputFolder;
};

// Parameters parsed from the input file and the forcing folder, and derived
// (the reference's GlobalConstants fields that the APT path reads).
struct GlobalConstants {
  int thermalType = 0;
  float G = 0, R = 0, delta = 0, kin_delta = 0, underCoolingRate = 0, V = 0;
  float underCoolingRate0 = 0, nuc_Nmax0 = 0;
  float k = 0, c_infty = 0, m_slope = 0, c_infm = 0, Dl = 0, GT = 0;
  float Dh = 0, d0 = 0, W0 = 0, L_cp = 0;
  float lamd = 0, tau0 = 0, beta0 = 0, mu_k = 0, lT = 0;
  float beta0_tilde = 0;
  float alpha0 = 0, eps = 0, eta = 0;
  float lxd = 0, lyd = 0, lzd = 0, tmax = 0;
  float xmin = 0, ymin = 0, zmin = 0;
  float asp_ratio_yx = 1, asp_ratio_zx = 1, moving_ratio = 1;
  float z0 = 0, r0 = 0, x0 = 0, top = 0, angle = 0, min_angle = 0;
  float mp_len = 0, order = 0;
  int nx = 0, ny = 0, nz = 0, nz_full = 0, fnx = 0, fny = 0, fnz = 0, fnz_f = 0;
  long long length = 0, full_length = 0;
  int haloWidth = 1;
  int Mt = 0, preMt = 0, nts = 1, NUM_PF = 8;
  float dx = 0, dt = 0, hi = 0, cfl = 0, dt_sqrt = 0;
  int Nx = 2, Ny = 2, Nz = 2, Nt = 2;
  int ictype = 0;
  int bcX = 0, bcY = 0, bcZ = 0;
  int num_theta = 0, num_nodes = 0;
  float cosa = 1, sina = 0, sqrt2 = 0, a_s = 0, epsilon = 0, a_12 = 0;
  int noi_period = 0, seed_val = 0;
  float Tmelt = 0, Ti = 0, Tliq = 0, Tsol = 0;
  float undcool_mean = 0, undcool_std = 0, nuc_Nmax = 0, nuc_rad = 0, pts_cell = 0;
  int walltime = 0;
};

class ThermalInputData {
 public:
  std::string folder;
  int Nx = 0, Ny = 0, Nz = 0, Nt = 0;
  std::vector<float> X_mac, Y_mac, Z_mac, t_mac, psi_mac, T_3D, theta_arr, cost, sint;
  std::vector<int> alpha_mac;
};

class MovingDomain {
 public:
  void allocateMovingDomain(int numGrains, int movingDirectionSize);
  int move_count = 0;
  int cur_tip = 1;
  int tip_front = 1;
  int tip_thres = 0;
  int samples = 0, lowsl = 1;
  std::vector<int> loss_area_host;
};

// Single-process stand-in for the reference's MPI setting (MPIsetting.h:15-62,
// MPIsetting.cpp:33-51): one process drives the whole domain on one GPU, so
// every partition is 1 x 1 x 1 and rank 0 of 1.  The constructors accept the
// reference's communicator argument whatever its type.
class MPIsetting {
 public:
  MPIsetting() = default;
  template <class Comm>
  explicit MPIsetting(Comm) {}
  virtual ~MPIsetting() = default;
  void printMPIsetting() const;
  virtual void domainPartition() = 0;

  int rank = 0, numProcessor = 1;
  int processorIDX = 0, processorIDY = 0, processorIDZ = 0;
  int numProcessorX = 1, numProcessorY = 1, numProcessorZ = 1;
  int nxLocal = 0, nyLocal = 0, nzLocal = 0, nzLocalAll = 0;
  int haloWidth = 1;
};

class MPIsetting1D : public MPIsetting {
 public:
  MPIsetting1D() = default;
  template <class Comm>
  explicit MPIsetting1D(Comm c) : MPIsetting(c) {}
  void domainPartition() override;
};

class MPIsetting2D : public MPIsetting {
 public:
  MPIsetting2D() = default;
  template <class Comm>
  explicit MPIsetting2D(Comm c) : MPIsetting(c) {}
  void domainPartition() override;
};

// The solver interface of the reference (cuPDE.h:4-21).
class PDE {
 public:
  virtual ~PDE() = default;
  virtual void cpuSetup(MPIsetting* mpiManager) = 0;
  virtual void initField() = 0;
  virtual void cudaSetup() = 0;
  virtual void evolve() = 0;
};

// The full (non-APT) phase-field solver, one phi field per grain (the reference's
// PhaseField, PhaseField.cu:431-632, selected by -a); APTPhaseField overrides
// cudaSetup and evolve with the active-parameter-tracking solver.
//
// The methods keep the reference's names, arguments and void results
// (PhaseField.h:11-59).  The reference checks no error; here the first failure
// is recorded (failed(), lastError()) and every later call of the sequence
// returns without doing anything, so a caller checks once at the end.
class PhaseField : public PDE {
 public:
  ~PhaseField() override;
  void parseInputParams(const std::string fileName);
  void cpuSetup(MPIsetting* mpiManager) override;
  void initField() override;
  void cudaSetup() override;
  void evolve() override;
  void OutputQoIs();
  void OutputField(int currentStep);
  // Device candidates of the 3D junction search on the last collected argmax map
  // (cells ascending, per-cell distinct counts); false where there are none.
  virtual bool deviceJunctionCandidates(std::vector<long long>&, std::vector<unsigned char>&) {
    return false;
  }
  void SetMPIManager(MPIsetting* mpiManager) { mMPIManager = mpiManager; }
  MPIsetting* GetMPIManager() const { return mMPIManager; }
  void SetDesignSetting(const DesignSettingData* d) { mDesignSetting = d; }
  const DesignSettingData* GetSetDesignSetting() const { return mDesignSetting; }
  bool failed() const { return !mErr.empty(); }
  const std::string& lastError() const { return mErr; }

  int fnx = 0, fny = 0, fnz = 0, fnz_f = 0, NUM_PF = 0;
  long long length = 0, full_length = 0;
  std::vector<float> x, y, z, z_full, phi, psi;
  std::vector<int> alpha, alpha_i_full;
  ThermalInputData mac;
  GlobalConstants params;
  QOI* qois = nullptr;  // set by the caller (main.cpp:58-65); owned and deleted here
  QoiGrid qoiGrid() const;
  std::string outputBaseName() const;
  cupf_apt_params deviceParams() const;
  int device = 0;

 protected:
  // records the first failure and prints it to stderr (a caller written for the
  // reference's void methods, such as its main.cpp, checks nothing)
  bool setErr(const std::string& e);
  bool check(cupf_status st, const char* what);
  bool parseInputImpl(const std::string& fileName);
  bool cpuSetupImpl(MPIsetting* mpiManager);
  bool initFieldImpl();
  bool denseCudaSetup();
  bool denseEvolve();
  bool outputQoIsImpl();
  bool lineJunctions(QOILine* q, const QoiGrid& g, const int* a);
  bool outputFieldImpl(int currentStep);
  const DesignSettingData* mDesignSetting = nullptr;
  MPIsetting* mMPIManager = nullptr;
  std::string mErr;
  cupf_dense_handle* mDense = nullptr;
};

class APTPhaseField : public PhaseField {
 public:
  ~APTPhaseField() override;
  void cudaSetup() override;
  void evolve() override;
  bool deviceJunctionCandidates(std::vector<long long>& cells,
                                std::vector<unsigned char>& distinct) override;
  cupf_apt_handle* handle() const { return mHandle; }
  cupf_precision precision = CUPF_PREC_FP32;

 protected:
  bool aptCudaSetup();
  bool aptEvolve();
  bool moveDomain(MovingDomain* md);
  bool getLineQoIs(MovingDomain* md);
  bool collectToHost(bool clear);
  cupf_apt_handle* mHandle = nullptr;
};

}  // namespace cupf_host
