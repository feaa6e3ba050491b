// ek2d_host.h — host side of the 2D Echebarria–Karma line model: the
// reference's main.cpp (2DdendriteMPI/line_model/main.cpp) split into its
// parameter, macro-table, initial-field and output steps, plus the quantities
// of interest (tip position, primary spacing) the library adds.
#pragma once

#include <string>
#include <vector>

#include "../../include/cupf_ek2d.h"

namespace cupf_host {

// Macro tables of the folder given on the command line (main.cpp:186-196).
struct Ek2dMac {
  std::vector<float> t, G, R, y, psi, U;
};

// Reads t.txt, Gt.txt, Rt.txt (Nt values) and y.txt, psi.txt, U.txt (Ny values).
bool ek2d_read_mac(const std::string& folder, int Ny, int Nt, Ek2dMac& mac, std::string& err);

// Coordinates and the initial psi, phi, U of main.cpp:225-271 (reference layout,
// halos zero): x_i = (i-1) dx W0, y_j = (j-1) dx W0 + y_mac[0]; psi and U are
// the 1-D profiles interpolated linearly in y; phi = tanh(psi/sqrt2).
void ek2d_initial_fields(const cupf_ek2d_params& p, const std::vector<float>& y_mac,
                         const std::vector<float>& psi_mac, const std::vector<float>& U_mac,
                         std::vector<float>& x, std::vector<float>& y, std::vector<float>& psi,
                         std::vector<float>& phi, std::vector<float>& U);

// Seeded front perturbation (no counterpart in the reference, which relies on
// its noise term): `sites` Gaussian bumps evenly spaced in x, half a spacing
// wide, each adding amp*(2u-1) to psi (u uniform from Philox keyed on the site
// and seed_val), i.e. moving the front by that many W0.
void ek2d_perturb(const cupf_ek2d_params& p, int sites, float amp, std::vector<float>& psi,
                  std::vector<float>& phi);

// Quantities of interest of one frame (FP64).
struct Ek2dQois {
  double tip_y = 0;        // highest phi = 0 crossing over all columns, um
  double front_mean_y = 0; // mean over columns of each column's highest crossing, um
  double spacing = 0;      // primary spacing, um (0 if the front has no cells)
  int spacing_k = 0;       // dominant wavenumber index along x
  int mushy_row = -1;      // row whose solid fraction is nearest 1/2
};
Ek2dQois ek2d_qois(const float* phi, int fnx, int fny, const double* y, double dxd);

// Concentration c/c_inf written by the reference (main.cpp:275-279).
void ek2d_concentration(const cupf_ek2d_params& p, const std::vector<float>& phi,
                        std::vector<float>& U);

}  // namespace cupf_host
