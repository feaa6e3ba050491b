// ref_dense_harness.cu — TEST INFRASTRUCTURE ONLY: launchers for the reference's
// own full (non-APT) phase-field kernels (cuPF 3DgrainMPI/PhaseField.cu), compiled
// unmodified from where they lie (the build adds that directory to the include
// path).  All pointers are device pointers.  Nothing here is used by the library.
#include "PhaseField.cu"

#include <cstring>

#include "../../include/cupf.h"

static GlobalConstants g_dense;
static float* g_dummy = nullptr;  // the rhs_psi macro-grid / noise arguments it never reads

extern "C" {

// The constants PhaseField::cudaSetup uploads (NUM_PF = num_theta, :440), with
// R = Rmax (m/s) for the line undercooling of rhs_psi (:277).
int refd_set_params(const cupf_apt_params* p, float R) {
  GlobalConstants& c = g_dense;
  memset(&c, 0, sizeof(c));
  c.fnx = p->fnx;
  c.fny = p->fny;
  c.fnz = p->fnz;
  c.length = p->fnx * p->fny * p->fnz;
  c.num_theta = p->num_theta;
  c.NUM_PF = p->num_theta;
  c.kin_delta = p->kin_delta;
  c.eps = p->eps;
  c.G = p->G;
  c.R = R;
  c.L_cp = p->L_cp;
  c.hi = p->hi;
  c.lamd = p->lamd;
  c.dt = p->dt;
  c.tau0 = p->tau0;
  c.z0 = p->z0;
  c.dx = p->dx;
  c.W0 = p->W0;
  if (!g_dummy) {
    if (cudaMalloc((void**)&g_dummy, 64 * sizeof(float)) != cudaSuccess) return 1;
    cudaMemset(g_dummy, 0, 64 * sizeof(float));
  }
  return (int)cudaMemcpyToSymbol(cP, &c, sizeof(GlobalConstants));
}

static int max_area() {
  int fnx = g_dense.fnx, fny = g_dense.fny, fnz = g_dense.fnz;
  return max(fnz * fny, max(fny * fnx, fnx * fnz));
}

int refd_set_bc(float* ph) {
  int ma = max_area();
  set_BC_3D<<<(ma * g_dense.NUM_PF + 127) / 128, 128>>>(ph, ma);
  return (int)cudaGetLastError();
}

int refd_rhs_psi(float t, const float* x, const float* y, const float* z, float* ph, float* ph_new,
                 const float* sint, const float* cost) {
  int nb = (g_dense.length * g_dense.NUM_PF + 127) / 128;
  rhs_psi<<<nb, 128>>>((float*)x, (float*)y, (float*)z, ph, ph_new, 0, t, g_dummy, g_dummy,
                       g_dummy, g_dummy, g_dummy, 2, 2, 2, 2, (curandState*)g_dummy, (float*)cost,
                       (float*)sint);
  return (int)cudaGetLastError();
}

int refd_set_minus1(float* u, int size) {
  set_minus1<<<(size + 127) / 128, 128>>>(u, size);
  return (int)cudaGetLastError();
}

int refd_ini(float* PFs, float* phi, int* alpha) {
  ini_PF<<<(g_dense.length * g_dense.NUM_PF + 127) / 128, 128>>>(PFs, phi, alpha);
  return (int)cudaGetLastError();
}

int refd_collect(float* PFs, float* phi, int* alpha, int* argmax) {
  collect_PF<<<(g_dense.length + 127) / 128, 128>>>(PFs, phi, alpha, argmax);
  return (int)cudaGetLastError();
}

int refd_move_frame(float* ph_buff, float* z_buff, float* ph, float* z, int* alpha, int* alpha_full,
                    int* loss_area, int move_count) {
  int nb = (g_dense.length * g_dense.NUM_PF + 127) / 128;
  move_frame<<<nb, 128>>>(ph_buff, z_buff, ph, z, alpha, alpha_full, loss_area, move_count);
  return (int)cudaGetLastError();
}

int refd_copy_frame(float* ph_buff, float* z_buff, float* ph, float* z) {
  int nb = (g_dense.length * g_dense.NUM_PF + 127) / 128;
  copy_frame<<<nb, 128>>>(ph_buff, z_buff, ph, z);
  return (int)cudaGetLastError();
}

int refd_tip_mvf(int* cur_tip, float* PFs, float* meanx_dev, float* meanx_host) {
  tip_mvf(cur_tip, PFs, meanx_dev, meanx_host, g_dense.fnx, g_dense.fny, g_dense.fnz,
          g_dense.NUM_PF);
  return (int)cudaGetLastError();
}

int refd_sync(void) { return (int)cudaDeviceSynchronize(); }

// nsteps of evolve's step pair (set_BC_3D on the buffer read, rhs_psi into the
// other, PhaseField.cu:563-566) from buffer a at step index step0 (t of step n =
// n*dt*tau0 in float); device time through *ms (CUDA events, legacy stream).
int refd_run_steps(int nsteps, int step0, const float* x, const float* y, const float* z,
                   float* ph_a, float* ph_b, const float* sint, const float* cost, float* ms) {
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, 0);
  float* pin = ph_a;
  float* pout = ph_b;
  for (int n = 0; n < nsteps; ++n) {
    float t = (float)(step0 + n + 1) * g_dense.dt * g_dense.tau0;
    int r = refd_set_bc(pin);
    if (r) return r;
    if ((r = refd_rhs_psi(t, x, y, z, pin, pout, sint, cost))) return r;
    float* tp = pin;
    pin = pout;
    pout = tp;
  }
  cudaEventRecord(e1, 0);
  cudaEventSynchronize(e1);
  cudaEventElapsedTime(ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return (int)cudaGetLastError();
}

}  // extern "C"
