// ref_host_stubs.cpp — TEST INFRASTRUCTURE ONLY.
// The reference's PhaseFieldCpu.cpp needs libhdf5, which this image lacks, so
// the parity harness links these stand-ins for its five methods instead.  The
// harness never calls them; they exist so the reference's class vtables resolve.
#include <cstdio>
#include <cstdlib>
#include <string>
#include "PhaseField.h"

static void not_in_harness(const char* what) {
  std::fprintf(stderr, "ref harness: %s is not available (needs libhdf5)\n", what);
  std::abort();
}
void PhaseField::parseInputParams(std::string) { not_in_harness("parseInputParams"); }
void PhaseField::cpuSetup(MPIsetting*) { not_in_harness("cpuSetup"); }
void PhaseField::initField() { not_in_harness("initField"); }
void PhaseField::OutputQoIs() { not_in_harness("OutputQoIs"); }
void PhaseField::OutputField(int) { not_in_harness("OutputField"); }
