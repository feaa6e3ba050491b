// ek2d_main.cpp — `phase_field_2d`, the command-line driver of the 2D
// Echebarria–Karma line model, in place of the reference's
// 2DdendriteMPI/line_model/main.cpp + setup() (PF.cu:699-842):
//
//   phase_field_2d <input_file> <mac_folder> [-o outdir] [-p fp32|fp16|bf16|fp64]
//                  [-s steps]
//
// Reads the `key = value` input file and the macro tables of mac_folder, builds
// the initial psi/U from the 1-D profiles, runs the psi-only pre-step and Mt
// fused steps (with the tip search and moving frame every TIPP steps), and
// writes phi, the concentration c/c_inf and the coordinates (y - ztip0) as
// line_nx<nx>_ny<ny>_Mt<Mt>_seed<seed>.h5, the reference's datasets, through the
// library's HDF5 writer (.npz when CUPF_OUTPUT_FORMAT=npz), plus the tip height
// and primary spacing.
//
// Input keys beyond the reference's: perturb_sites / perturb_amp add the seeded
// front perturbation of cupf_host_ek2d_perturb; cfl defaults to 0.8 when absent
// (the line model's input file has no cfl line, and its comment gives
// dt = 0.8 dx^2/(4 Dl_tilde)).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "../../include/cupf_ek2d.h"
#include "ek2d_host.h"
#include "host_util.h"
#include "array_file.h"

using namespace cupf_host;

static int die(const char* msg) {
  fprintf(stderr, "phase_field_2d: %s\n", msg);
  return 1;
}

int main(int argc, char** argv) {
  if (argc < 3)
    return die("usage: phase_field_2d <input_file> <mac_folder> [-o outdir] [-p fp32|fp16|bf16|fp64] [-s steps]");
  const std::string input = argv[1], mac_folder = argv[2];
  std::string outdir = mac_folder, prec_name = "fp32";
  long long steps_override = -1;
  for (int a = 3; a + 1 < argc; a += 2) {
    if (!strcmp(argv[a], "-o")) outdir = argv[a + 1];
    else if (!strcmp(argv[a], "-p")) prec_name = argv[a + 1];
    else if (!strcmp(argv[a], "-s")) steps_override = atoll(argv[a + 1]);
    else return die("unknown option");
  }
  int prec = CUPF_PREC_FP32;
  if (prec_name == "fp16") prec = CUPF_PREC_FP16;
  else if (prec_name == "bf16") prec = CUPF_PREC_BF16;
  else if (prec_name == "fp64") prec = CUPF_PREC_FP64;
  else if (prec_name != "fp32") return die("precision must be fp32, fp16, bf16 or fp64");

  cupf_ek2d_params p;
  memset(&p, 0, sizeof(p));
  p.cfl = 0.8f;
  int32_t Ny = 0, Nt = 0;
  float ztip0 = 0.0f;
  if (cupf_ek2d_parse_input(input.c_str(), &p, &Ny, &Nt, &ztip0) != CUPF_OK)
    return die("cannot read the input file");
  float sites = 0.0f, amp = 0.0f;
  {
    std::ifstream f(input);
    std::string line;
    while (std::getline(f, line)) {
      getParam(line, "perturb_sites", sites);
      getParam(line, "perturb_amp", amp);
    }
  }
  Ek2dMac mac;
  std::string err;
  if (!ek2d_read_mac(mac_folder, Ny, Nt, mac, err)) return die(err.c_str());
  cupf_ek2d_derive(&p, mac.t[Nt - 1]);
  p.y0 = mac.y[0];
  printf("nx = %d, ny = %d, Mt = %d, dt = %g, tau0 = %g, lT_tilde = %g, Dl_tilde = %g\n", p.nx,
         p.ny, p.Mt, p.dt, p.tau0, p.lT_tilde, p.Dl_tilde);

  std::vector<float> x, y, psi, phi, U;
  ek2d_initial_fields(p, mac.y, mac.psi, mac.U, x, y, psi, phi, U);
  ek2d_perturb(p, (int)sites, amp, psi, phi);

  cupf_ek2d_handle* h = nullptr;
  auto check = [&](cupf_status st) {
    if (st != CUPF_OK) {
      fprintf(stderr, "phase_field_2d: %s\n", cupf_last_error());
      if (h) cupf_ek2d_destroy(h);
      exit(2);
    }
  };
  check(cupf_ek2d_create(&p, prec, 0, &h));
  check(cupf_ek2d_set_thermal(h, Nt, mac.t.data(), mac.G.data(), mac.R.data()));
  check(cupf_ek2d_set_state(h, psi.data(), U.data(), nullptr));
  check(cupf_ek2d_prestep(h));
  const long long steps = steps_override >= 0 ? steps_override : p.Mt;
  float ms = 0.0f;
  for (long long done = 0; done < steps;) {
    const int chunk = (int)std::min<long long>(steps - done, 1 << 20);
    float part = 0.0f;
    check(cupf_ek2d_time_steps(h, chunk, &part));
    ms += part;
    done += chunk;
  }
  printf("time for %lld iterations: %f s\n", steps, ms / 1000.0);
  check(cupf_ek2d_get_state(h, psi.data(), phi.data(), U.data(), nullptr));
  const int fnx = p.nx + 2, fny = p.ny + 3;
  std::vector<double> yd(fny);
  check(cupf_ek2d_get_y(h, yd.data()));
  cupf_ek2d_info info;
  check(cupf_ek2d_info_get(h, &info));
  cupf_ek2d_destroy(h);

  const Ek2dQois q = ek2d_qois(phi.data(), fnx, fny, yd.data(), (double)p.dx * p.W0);
  printf("tip y = %.6f um, mean front y = %.6f um, primary spacing = %.6f um (k = %d), frame moved %lld rows\n",
         q.tip_y, q.front_mean_y, q.spacing, q.spacing_k, (long long)info.shifts);

  ek2d_concentration(p, phi, U);
  for (int j = 0; j < fny; ++j) y[j] = (float)(yd[j] - ztip0);
  ArrayFile w;
  w.add("phi", phi);
  w.add("Uc", U);
  w.add("x_coordinates", x);
  w.add("y_coordinates", y);
  std::vector<float> qv = {(float)q.tip_y, (float)q.front_mean_y, (float)q.spacing,
                           (float)info.shifts};
  w.add("qois_tip_front_spacing_shifts", qv);
  const std::string out = outdir + "/line_nx" + std::to_string(p.nx) + "_ny" + std::to_string(p.ny) +
                          "_Mt" + std::to_string(p.Mt) + "_seed" + std::to_string(p.seed_val);
  if (!w.write(out)) return die("cannot write the output file");
  printf("wrote %s%s\n", out.c_str(), w.extension());
  return 0;
}
