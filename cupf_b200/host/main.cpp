// phase_field — command-line driver with the reference's call order
// (3DgrainMPI/main.cpp:15-77): options, solver, parseInputParams, cpuSetup, QoI
// object, initField, cudaSetup, evolve, OutputQoIs.  Single process, one GPU.
#include <cstdio>
#include <memory>

#include "phase_field.h"

using namespace cupf_host;

int main(int argc, char** argv) {
  DesignSettingData ds;
  std::string err;
  if (!ds.getOptions(argc, argv, &err)) {
    std::fprintf(stderr, "%s\n", err.c_str());
    return 2;
  }
  // -a selects the full (non-APT) solver, one phi field per grain (main.cpp:39-47)
  std::unique_ptr<PhaseField> pf(ds.useAPT ? static_cast<PhaseField*>(new APTPhaseField())
                                           : new PhaseField());
  MPIsetting1D mpiManager;  // rank 0 of 1: the whole domain on one GPU
  mpiManager.domainPartition();
  pf->SetDesignSetting(&ds);
  pf->SetMPIManager(&mpiManager);
  pf->mac.folder = ds.thermalInputFolder + std::to_string(ds.seedValue);
  pf->params.seed_val = ds.seedValue;
  pf->parseInputParams(ds.inputFile);
  pf->cpuSetup(&mpiManager);
  if (!pf->failed()) {
    if (ds.useLineConfig) pf->qois = new QOILine(pf->params);
    else pf->qois = new QOI3D(pf->params);
  }
  pf->initField();
  pf->cudaSetup();
  pf->evolve();
  pf->OutputQoIs();
  if (pf->failed()) {
    std::fprintf(stderr, "phase_field: %s\n", pf->lastError().c_str());
    return 1;
  }
  std::printf("phase_field: %d steps, walltime %d s, %d grains active\n", pf->params.Mt,
              pf->params.walltime, pf->qois->mNumActiveGrains);
  return 0;
}
