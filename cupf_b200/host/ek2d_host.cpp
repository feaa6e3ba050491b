// ek2d_host.cpp — host side of the 2D Echebarria–Karma line model (see
// ek2d_host.h), and the C entry points cupf_ek2d_derive / cupf_ek2d_parse_input
// and cupf_host_ek2d_*.
#include "ek2d_host.h"

#include <cuda_runtime.h>  // defines __host__/__device__ for philox.cuh

#include <algorithm>
#include <cmath>
#include <fstream>
#include <sstream>

#include "../../include/cupf_host.h"
#include "../csrc/philox.cuh"
#include "host_util.h"

namespace cupf_host {

bool ek2d_read_mac(const std::string& folder, int Ny, int Nt, Ek2dMac& mac, std::string& err) {
  struct F {
    const char* name;
    std::vector<float>* v;
    int n;
  } files[] = {{"t.txt", &mac.t, Nt},   {"Gt.txt", &mac.G, Nt},    {"Rt.txt", &mac.R, Nt},
               {"y.txt", &mac.y, Ny},   {"psi.txt", &mac.psi, Ny}, {"U.txt", &mac.U, Ny}};
  for (const F& f : files) {
    if (f.n < 2) {
      err = std::string("table length below 2 for ") + f.name;
      return false;
    }
    f.v->assign(f.n, 0.0f);
    const int got = read_input(folder + "/" + f.name, f.v->data(), f.n);
    if (got < 0) {
      err = "cannot open " + folder + "/" + f.name;
      return false;
    }
    if (got < f.n) {
      err = "short table " + folder + "/" + f.name;
      return false;
    }
  }
  return true;
}

void ek2d_initial_fields(const cupf_ek2d_params& p, const std::vector<float>& y_mac,
                         const std::vector<float>& psi_mac, const std::vector<float>& U_mac,
                         std::vector<float>& x, std::vector<float>& y, std::vector<float>& psi,
                         std::vector<float>& phi, std::vector<float>& U) {
  const int fnx = p.nx + 2, fny = p.ny + 3;
  const float dxd = p.dx * p.W0;
  x.resize(fnx);
  y.resize(fny);
  for (int i = 0; i < fnx; ++i) x[i] = (i - 1) * dxd;
  for (int j = 0; j < fny; ++j) y[j] = (j - 1) * dxd + y_mac[0];
  const size_t n = (size_t)fnx * fny;
  psi.assign(n, 0.0f);
  phi.assign(n, 0.0f);
  U.assign(n, 0.0f);
  const int ny_mac = (int)y_mac.size();
  const float Dy = y_mac[1] - y_mac[0];
  for (int j = 1; j < fny - 1; ++j) {
    // linear interpolation of the 1-D profiles (main.cpp:256-262); the interval
    // is clamped to the table, which the reference leaves to the caller
    const float s = (y[j] - y_mac[0]) / Dy;
    int ky = (int)s;
    float d = s - ky;
    if (ky < 0) {
      ky = 0;
      d = 0.0f;
    }
    if (ky > ny_mac - 2) {
      ky = ny_mac - 2;
      d = 1.0f;
    }
    const float ps = (1.0f - d) * psi_mac[ky] + d * psi_mac[ky + 1];
    const float u = (1.0f - d) * U_mac[ky] + d * U_mac[ky + 1];
    const float ph = tanhf(ps / p.sqrt2);
    for (int i = 1; i < fnx - 1; ++i) {
      const size_t id = (size_t)j * fnx + i;
      psi[id] = ps;
      U[id] = u;
      phi[id] = ph;
    }
  }
}

void ek2d_perturb(const cupf_ek2d_params& p, int sites, float amp, std::vector<float>& psi,
                  std::vector<float>& phi) {
  if (sites <= 0 || amp == 0.0f) return;
  const int fnx = p.nx + 2, fny = p.ny + 3, nx = p.nx;
  const double spacing = (double)nx / sites, w = 0.5 * spacing;
  std::vector<double> a(sites), xs(sites);
  for (int s = 0; s < sites; ++s) {
    const cupf::Philox4 r =
        cupf::philox4x32_10((uint32_t)s, 0u, 0u, 0x50455254u, (uint32_t)p.seed_val, 0x5EEDu);
    a[s] = (double)amp * (2.0 * (double)cupf::uniform01(r.v[0]) - 1.0);
    xs[s] = (s + 0.5) * spacing;
  }
  std::vector<double> bump(fnx, 0.0);
  for (int i = 1; i < fnx - 1; ++i) {
    double v = 0.0;
    for (int s = 0; s < sites; ++s) {
      double d = std::fabs((double)(i - 1) - xs[s]);
      d = std::min(d, nx - d);  // periodic distance
      v += a[s] * std::exp(-(d / w) * (d / w));
    }
    bump[i] = v;
  }
  for (int j = 1; j < fny - 1; ++j)
    for (int i = 1; i < fnx - 1; ++i) {
      const size_t id = (size_t)j * fnx + i;
      psi[id] = (float)((double)psi[id] + bump[i]);
      phi[id] = tanhf(psi[id] / p.sqrt2);
    }
}

Ek2dQois ek2d_qois(const float* phi, int fnx, int fny, const double* y, double dxd) {
  Ek2dQois q;
  const int nx = fnx - 2;
  // front height of each column: its highest phi = 0 crossing, interpolated
  double tip = -1e300, sum = 0.0;
  int ncol = 0;
  for (int i = 1; i <= nx; ++i) {
    for (int j = fny - 3; j >= 1; --j) {
      const double a = phi[(size_t)j * fnx + i], b = phi[(size_t)(j + 1) * fnx + i];
      if (a >= 0.0 && b < 0.0) {
        const double h = y[j] + dxd * a / (a - b);
        tip = std::max(tip, h);
        sum += h;
        ++ncol;
        break;
      }
    }
  }
  q.tip_y = ncol ? tip : 0.0;
  q.front_mean_y = ncol ? sum / ncol : 0.0;
  // primary spacing: dominant wavenumber of the solid indicator along x, over
  // the rows around the one whose solid fraction is nearest 1/2
  std::vector<double> frac(fny, 0.0);
  int best = -1;
  double bestd = 1e300;
  for (int j = 1; j < fny - 1; ++j) {
    int cnt = 0;
    for (int i = 1; i <= nx; ++i) cnt += phi[(size_t)j * fnx + i] > 0.0f;
    frac[j] = (double)cnt / nx;
    if (frac[j] > 0.05 && frac[j] < 0.95 && std::fabs(frac[j] - 0.5) < bestd) {
      bestd = std::fabs(frac[j] - 0.5);
      best = j;
    }
  }
  q.mushy_row = best;
  if (best < 0 || nx < 4) return q;
  const int kmax = nx / 2;
  std::vector<double> power(kmax + 1, 0.0), cs(nx), sn(nx), s(nx);
  for (int i = 0; i < nx; ++i) {
    cs[i] = std::cos(2.0 * M_PI * i / nx);
    sn[i] = std::sin(2.0 * M_PI * i / nx);
  }
  for (int j = std::max(1, best - 2); j <= std::min(fny - 2, best + 2); ++j) {
    if (!(frac[j] > 0.05 && frac[j] < 0.95)) continue;
    for (int i = 0; i < nx; ++i) s[i] = (phi[(size_t)j * fnx + i + 1] > 0.0f ? 1.0 : 0.0) - frac[j];
    for (int k = 1; k <= kmax; ++k) {
      double re = 0.0, im = 0.0;
      long long idx = 0;
      for (int i = 0; i < nx; ++i) {
        re += s[i] * cs[idx];
        im -= s[i] * sn[idx];
        idx += k;
        if (idx >= nx) idx -= nx;
      }
      power[k] += re * re + im * im;
    }
  }
  int kbest = 1;
  for (int k = 2; k <= kmax; ++k)
    if (power[k] > power[kbest]) kbest = k;
  q.spacing_k = kbest;
  q.spacing = (double)nx * dxd / kbest;
  return q;
}

void ek2d_concentration(const cupf_ek2d_params& p, const std::vector<float>& phi,
                        std::vector<float>& U) {
  const float cinf_cl0 = 1.0f + (1.0f - p.k) * p.U0;
  for (size_t id = 0; id < U.size(); ++id)
    U[id] = (1.0f + (1.0f - p.k) * U[id]) * (p.k * (1.0f + phi[id]) / 2.0f + (1.0f - phi[id]) / 2.0f) /
            cinf_cl0;
}

}  // namespace cupf_host

using namespace cupf_host;

extern "C" cupf_status cupf_ek2d_derive(cupf_ek2d_params* p, float t_last) {
  if (!p) return CUPF_ERR_INVALID;
  // main.cpp:158-185; each float field takes the value of its expression as the
  // reference evaluates it (double where a double literal or pow() enters)
  p->lT = p->c_infm * (1.0 / p->k - 1) / p->G;
  p->lamd = 5 * std::sqrt(2.0) / 8 * p->W0 / p->d0;
  p->tau0 = 0.6267 * p->lamd * p->W0 * p->W0 / p->Dl;
  p->R_tilde = p->R * p->tau0 / p->W0;
  p->Dl_tilde = p->Dl * p->tau0 / std::pow((double)p->W0, 2);
  p->lT_tilde = p->lT / p->W0;
  p->dt = p->cfl * std::pow((double)p->dx, 2) / (4 * p->Dl_tilde);
  const float dxd = p->dx * p->W0;
  p->nx = (int)(p->lxd / dxd);
  p->ny = (int)(p->asp_ratio * p->nx);
  p->Mt = (int)(t_last / p->tau0 / p->dt);
  p->Mt = (p->Mt / 2) * 2;
  p->lyd = p->asp_ratio * p->lxd;
  p->hi = 1.0 / p->dx;
  p->cosa = std::cos(p->alpha0 / 180 * M_PI);
  p->sina = std::sin(p->alpha0 / 180 * M_PI);
  p->sqrt2 = std::sqrt(2.0);
  p->a_s = 1 - 3.0 * p->delta;
  p->epsilon = 4.0 * p->delta / p->a_s;
  p->a_12 = 4.0 * p->a_s * p->epsilon;
  p->dt_sqrt = std::sqrt(p->dt);
  if (p->tipp <= 0) p->tipp = 100;     // TIPP (PF.cu:11)
  if (p->blank <= 0.0f) p->blank = 0.3f;  // BLANK (PF.cu:12)
  if (p->ls == 0.0f) p->ls = -0.995f;   // LS (PF.cu:10)
  return CUPF_OK;
}

extern "C" cupf_status cupf_ek2d_parse_input(const char* path, cupf_ek2d_params* p, int32_t* mac_Ny,
                                             int32_t* mac_Nt, float* ztip0) {
  if (!path || !p) return CUPF_ERR_INVALID;
  std::ifstream f(path);
  if (!f.good()) return CUPF_ERR_IO;
  struct K {
    const char* key;
    float* v;
  } keys[] = {{"G", &p->G},           {"R", &p->R},         {"delta", &p->delta},
              {"k", &p->k},           {"c_infm", &p->c_infm}, {"Dl", &p->Dl},
              {"d0", &p->d0},         {"W0", &p->W0},       {"c_infty", &p->c_infty},
              {"eps", &p->eps},       {"alpha0", &p->alpha0}, {"dx", &p->dx},
              {"asp_ratio", &p->asp_ratio}, {"lxd", &p->lxd}, {"eta", &p->eta},
              {"U0", &p->U0},         {"cfl", &p->cfl}};
  float seed = (float)p->seed_val, nprd = (float)p->noi_period;
  float ny = mac_Ny ? (float)*mac_Ny : 0.0f, nt = mac_Nt ? (float)*mac_Nt : 0.0f;
  float zt = ztip0 ? *ztip0 : 0.0f;
  std::string line;
  while (std::getline(f, line)) {
    for (const K& k : keys) getParam(line, k.key, *k.v);
    getParam(line, "seed_val", seed);
    getParam(line, "noi_period", nprd);
    getParam(line, "Ny", ny);
    getParam(line, "Nt", nt);
    getParam(line, "ztip0", zt);
  }
  p->seed_val = (int)seed;
  p->noi_period = (int)nprd;
  if (mac_Ny) *mac_Ny = (int)ny;
  if (mac_Nt) *mac_Nt = (int)nt;
  if (ztip0) *ztip0 = zt;
  return CUPF_OK;
}

extern "C" int cupf_host_ek2d_initial_fields(const cupf_ek2d_params* p, int Ny, const float* y_mac,
                                             const float* psi_mac, const float* U_mac, float* x,
                                             float* y, float* psi, float* phi, float* U) {
  if (!p || Ny < 2 || !y_mac || !psi_mac || !U_mac) return -1;
  std::vector<float> ym(y_mac, y_mac + Ny), pm(psi_mac, psi_mac + Ny), um(U_mac, U_mac + Ny);
  std::vector<float> vx, vy, vps, vph, vU;
  ek2d_initial_fields(*p, ym, pm, um, vx, vy, vps, vph, vU);
  if (x) std::copy(vx.begin(), vx.end(), x);
  if (y) std::copy(vy.begin(), vy.end(), y);
  if (psi) std::copy(vps.begin(), vps.end(), psi);
  if (phi) std::copy(vph.begin(), vph.end(), phi);
  if (U) std::copy(vU.begin(), vU.end(), U);
  return 0;
}

extern "C" int cupf_host_ek2d_perturb(const cupf_ek2d_params* p, int sites, float amp, float* psi,
                                      float* phi) {
  if (!p || !psi || !phi) return -1;
  const size_t n = (size_t)(p->nx + 2) * (p->ny + 3);
  std::vector<float> vps(psi, psi + n), vph(phi, phi + n);
  ek2d_perturb(*p, sites, amp, vps, vph);
  std::copy(vps.begin(), vps.end(), psi);
  std::copy(vph.begin(), vph.end(), phi);
  return 0;
}

extern "C" int cupf_host_ek2d_qois(const float* phi, int fnx, int fny, const double* y, double dxd,
                                   double* out) {
  if (!phi || !y || !out || fnx < 3 || fny < 4) return -1;
  const Ek2dQois q = ek2d_qois(phi, fnx, fny, y, dxd);
  out[0] = q.tip_y;
  out[1] = q.front_mean_y;
  out[2] = q.spacing;
  out[3] = q.spacing_k;
  out[4] = q.mushy_row;
  return 0;
}
