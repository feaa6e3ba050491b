// ref_setup_shim.cpp — TEST INFRASTRUCTURE ONLY.
// extern "C" entry into the reference's own host set-up: DesignSettingData,
// a single-rank MPIsetting1D, and PhaseField::parseInputParams, cpuSetup and
// initField (3DgrainMPI/PhaseFieldCpu.cpp:17-459, compiled unmodified against the
// stub hdf5.h of this folder), in main.cpp's order (main.cpp:19-66).  Tests
// compare what the library's C++ driver derives from the same input file and
// forcing folder with these results.
#include <cstring>
#include <string>

#include "DesignSettingData.h"
#include "MPIsetting.h"
#include "PhaseField.h"

// the coordinate arrays are protected members of the reference's PDE base
struct RefPhaseField : public PhaseField {
  using PDE::x;
  using PDE::y;
  using PDE::z;
};

extern "C" {

// flags bit 0 = line configuration, bit 1 = pure nucleation, bit 2 = nucleation.
// dims: fnx, fny, fnz, num_theta, Mt, nts, thermalType, fnz_f.
// fparams: dt, tau0, lamd, hi, G, underCoolingRate, z0, kin_delta, lxd, lyd, lzd,
//          R, V, top, r0, x0, cfl, underCoolingRate0, W0, dx.
// x/y/z/z_full (fnx/fny/fnz/fnz_f), phi/psi/alpha (fnx*fny*fnz) and
// sint/cost (2*num_theta+1) are copied when not NULL and cap allows.
int refh_setup(const char* input_file, const char* folder, int bcX, int bcY, int bcZ, int flags,
               int* dims, float* fparams, float* x, float* y, float* z, float* z_full, float* phi,
               float* psi, int* alpha, float* sint, float* cost, long long cap) {
  DesignSettingData* ds = new DesignSettingData();
  ds->useLineConfig = (flags & 1) != 0;
  ds->pureNucleation = (flags & 2) != 0;
  ds->includeNucleation = (flags & 4) != 0;
  ds->bcX = bcX;
  ds->bcY = bcY;
  ds->bcZ = bcZ;
  ds->inputFile = input_file;
  MPIsetting* mpi = new MPIsetting1D(MPI_COMM_WORLD);
  mpi->rank = 0;
  mpi->numProcessor = 1;
  mpi->domainPartition();
  RefPhaseField* pf = new RefPhaseField();
  pf->SetDesignSetting(ds);
  pf->SetMPIManager(mpi);
  pf->mac.folder = folder;
  pf->params.seed_val = 0;
  pf->parseInputParams(ds->inputFile);
  pf->cpuSetup(mpi);
  pf->initField();
  const GlobalConstants& p = pf->params;
  int d[8] = {pf->fnx, pf->fny, pf->fnz, p.num_theta, p.Mt, p.nts, p.thermalType, pf->fnz_f};
  std::memcpy(dims, d, sizeof(d));
  float f[20] = {p.dt, p.tau0, p.lamd, p.hi, p.G, p.underCoolingRate, p.z0, p.kin_delta,
                 p.lxd, p.lyd, p.lzd, p.R, p.V, p.top, p.r0, p.x0, p.cfl, p.underCoolingRate0,
                 p.W0, p.dx};
  std::memcpy(fparams, f, sizeof(f));
  const long long L = pf->length;
  if (x) std::memcpy(x, pf->x, sizeof(float) * pf->fnx);
  if (y) std::memcpy(y, pf->y, sizeof(float) * pf->fny);
  if (z) std::memcpy(z, pf->z, sizeof(float) * pf->fnz);
  if (z_full) std::memcpy(z_full, pf->z_full, sizeof(float) * pf->fnz_f);
  if (L <= cap) {
    if (phi) std::memcpy(phi, pf->phi, sizeof(float) * L);
    if (psi) std::memcpy(psi, pf->psi, sizeof(float) * L);
    if (alpha) std::memcpy(alpha, pf->alpha, sizeof(int) * L);
  }
  const int nt = 2 * p.num_theta + 1;
  if (nt <= cap) {
    if (sint) std::memcpy(sint, pf->mac.sint, sizeof(float) * nt);
    if (cost) std::memcpy(cost, pf->mac.cost, sizeof(float) * nt);
  }
  return L <= cap ? 0 : 1;  // the reference leaks its objects; so does this shim
}

}  // extern "C"
