// substrate.cpp — seeded 2D Voronoi substrate and grain orientations in the
// reference's forcing-folder format.
//
// The reference makes its substrate in Python (graph_datastruct.py:194-271:
// scipy Voronoi cells of seeded points rasterised with PIL, angles from a
// Gaussian random vector, :256-269) and writes it with numpy.savetxt
// (input_file.py:148-152): alpha.txt, one grain id per line for the
// (nx+1) x (ny+1) macro pixel map, rows of constant y in order of y;
// theta.txt, one angle per line as "%1.4e", [0, theta_x[1..NG], theta_z[1..NG]];
// NG.txt, the grain count.  PhaseField::initField reads alpha.txt as
// alpha_mac[(j-1)*(nx+1) + (i-1)] (PhaseFieldCpu.cpp:388-391, 429).
//
// This generator needs no Python: each pixel (centre at (i+1/2, j+1/2)) takes
// the id of the nearest of num_grains points placed uniformly in the map
// (minimum-image distance when periodic; the lowest id on a tie), and each
// grain's angles follow the reference's formula from a Gaussian random vector
// u: theta_x = atan2(u_y, u_x) mod pi, theta_z = atan2(|u_xy|, u_z) mod pi.
// Random numbers come from splitmix64 (a published 64-bit mixing generator),
// uniform doubles from its top 53 bits, normals by the Box-Muller transform.
// Points and angles use two streams of the same seed.
//
// Orientations given as unit quaternions map to the same two angles: the
// kernel's rotation (APTPhaseField.cu:41-46) sends the lab direction with
// azimuth theta_x and polar angle theta_z to the crystal z axis, so a grain's
// angles are those of its crystal [001] axis in the lab frame, the third column
// of the quaternion's rotation matrix.  The rotation about that axis, which the
// two-angle model has no parameter for, is dropped.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/cupf_host.h"

namespace {

struct SplitMix64 {
  uint64_t s;
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  double uniform() { return (double)(next() >> 11) * 0x1p-53; }  // [0, 1)
};

constexpr double kPi = 3.14159265358979323846;

}  // namespace

extern "C" int cupf_host_voronoi_substrate(int nxp, int nyp, int num_grains, uint64_t seed,
                                           int periodic, int32_t* alpha, float* theta) {
  if (nxp < 1 || nyp < 1 || num_grains < 1 || !alpha || !theta) return -1;
  SplitMix64 pts{seed};
  std::vector<double> px(num_grains), py(num_grains);
  for (int g = 0; g < num_grains; ++g) {
    px[g] = pts.uniform() * nxp;
    py[g] = pts.uniform() * nyp;
  }
  for (int j = 0; j < nyp; ++j)
    for (int i = 0; i < nxp; ++i) {
      const double cx = i + 0.5, cy = j + 0.5;
      double best = INFINITY;
      int id = 1;
      for (int g = 0; g < num_grains; ++g) {
        double dx = std::fabs(cx - px[g]), dy = std::fabs(cy - py[g]);
        if (periodic) {
          dx = std::fmin(dx, nxp - dx);
          dy = std::fmin(dy, nyp - dy);
        }
        const double d = dy * dy + dx * dx;
        if (d < best) {
          best = d;
          id = g + 1;
        }
      }
      alpha[(long long)j * nxp + i] = id;
    }
  SplitMix64 ang{seed ^ 0x5DEECE66Dull};
  theta[0] = 0.0f;
  for (int g = 0; g < num_grains; ++g) {
    const double u1 = 1.0 - ang.uniform(), u2 = ang.uniform();
    const double u3 = 1.0 - ang.uniform(), u4 = ang.uniform();
    const double a = std::sqrt(-2.0 * std::log(u1)), b = std::sqrt(-2.0 * std::log(u3));
    const double ux = a * std::cos(2.0 * kPi * u2), uy = a * std::sin(2.0 * kPi * u2);
    const double uz = b * std::cos(2.0 * kPi * u4);
    double tx = std::fmod(std::atan2(uy, ux), kPi);
    if (tx < 0) tx += kPi;
    const double tz = std::fmod(std::atan2(std::sqrt(ux * ux + uy * uy), uz), kPi);
    theta[1 + g] = (float)tx;
    theta[1 + num_grains + g] = (float)tz;
  }
  return 0;
}

extern "C" int cupf_host_quaternions_to_angles(int num_grains, const double* q, float* theta) {
  if (num_grains < 1 || !q || !theta) return -1;
  theta[0] = 0.0f;
  for (int g = 0; g < num_grains; ++g) {
    double w = q[4 * g], x = q[4 * g + 1], y = q[4 * g + 2], z = q[4 * g + 3];
    const double nrm = std::sqrt(w * w + x * x + y * y + z * z);
    if (!(nrm > 0.0) || !std::isfinite(nrm)) return -1;
    w /= nrm;
    x /= nrm;
    y /= nrm;
    z /= nrm;
    // crystal [001] in the lab frame: R(q) (0, 0, 1)
    const double ux = 2.0 * (x * z + w * y), uy = 2.0 * (y * z - w * x);
    const double uz = 1.0 - 2.0 * (x * x + y * y);
    double tx = std::fmod(std::atan2(uy, ux), kPi);
    if (tx < 0) tx += kPi;
    const double tz = std::fmod(std::atan2(std::sqrt(ux * ux + uy * uy), uz), kPi);
    theta[1 + g] = (float)tx;
    theta[1 + num_grains + g] = (float)tz;
  }
  return 0;
}

extern "C" int cupf_host_write_substrate(const char* folder, int nxp, int nyp,
                                         const int32_t* alpha, int num_grains,
                                         const float* theta) {
  if (!folder || nxp < 1 || nyp < 1 || num_grains < 1 || !alpha || !theta) return -1;
  const std::string dir(folder);
  FILE* f = std::fopen((dir + "/alpha.txt").c_str(), "w");
  if (!f) return -1;
  for (long long n = 0; n < (long long)nxp * nyp; ++n) std::fprintf(f, "%d\n", alpha[n]);
  if (std::fclose(f) != 0) return -1;
  f = std::fopen((dir + "/theta.txt").c_str(), "w");
  if (!f) return -1;
  for (int n = 0; n < 2 * num_grains + 1; ++n) std::fprintf(f, "%1.4e\n", (double)theta[n]);
  if (std::fclose(f) != 0) return -1;
  f = std::fopen((dir + "/NG.txt").c_str(), "w");
  if (!f) return -1;
  std::fprintf(f, "%d\n", num_grains);
  return std::fclose(f) != 0 ? -1 : 0;
}
