// ref_ek2d_harness.cu — TEST INFRASTRUCTURE ONLY: launchers for the reference's
// own 2D line-model kernels (cuPF 2DdendriteMPI/line_model/PF.cu), compiled
// unmodified from where they lie (the build adds that directory to the include
// path).  Nothing here is used by the library.
//
//   ref2d_step   one set_BC + merge_PF (or the pre-loop rhs_psi) on given fields
//   ref2d_setup  the reference's whole setup() time loop (PF.cu:699-842)
#include "PF.cu"

#include "../../include/cupf_ek2d.h"

// Declared extern by PF.cu and defined in a helper file the line model's
// Makefile expects from elsewhere (INC_FLAGS -I../common); unused by the kernels.
float toBW(int bytes, float sec) { return (float)bytes / sec / 1e9f; }

static GlobalConstants to_ref(const cupf_ek2d_params* p) {
  GlobalConstants g;
  memset(&g, 0, sizeof(g));
  g.nx = p->nx;
  g.ny = p->ny;
  g.Mt = p->Mt;
  g.G = p->G;
  g.R = p->R;
  g.delta = p->delta;
  g.k = p->k;
  g.c_infm = p->c_infm;
  g.Dl = p->Dl;
  g.d0 = p->d0;
  g.W0 = p->W0;
  g.lT = p->lT;
  g.lamd = p->lamd;
  g.tau0 = p->tau0;
  g.c_infty = p->c_infty;
  g.R_tilde = p->R_tilde;
  g.Dl_tilde = p->Dl_tilde;
  g.lT_tilde = p->lT_tilde;
  g.eps = p->eps;
  g.alpha0 = p->alpha0;
  g.dx = p->dx;
  g.dt = p->dt;
  g.asp_ratio = p->asp_ratio;
  g.lxd = p->lxd;
  g.lyd = p->lyd;
  g.eta = p->eta;
  g.U0 = p->U0;
  g.seed_val = p->seed_val;
  g.hi = p->hi;
  g.cosa = p->cosa;
  g.sina = p->sina;
  g.sqrt2 = p->sqrt2;
  g.a_s = p->a_s;
  g.epsilon = p->epsilon;
  g.a_12 = p->a_12;
  g.dt_sqrt = p->dt_sqrt;
  g.noi_period = p->noi_period;
  g.cfl = p->cfl;
  return g;
}

#define RK(call)                                   \
  do {                                             \
    if ((call) != cudaSuccess) return __LINE__;    \
  } while (0)

// One step of the reference on host arrays (reference layout, fnx*fny):
// set_BC on the inputs, then merge_PF (prestep == 0) or rhs_psi (prestep == 1,
// U_n receives U).  Returns 0 or the failing line.
extern "C" int ref2d_step(const cupf_ek2d_params* p, const float* ps, const float* ph,
                          const float* U, const float* D, const float* y, float intR, float lT,
                          int prestep, float* ps_n, float* ph_n, float* U_n, float* D_n) {
  const int fnx = p->nx + 2, fny = p->ny + 3, n = fnx * fny;
  GlobalConstants g = to_ref(p);
  RK(cudaMemcpyToSymbol(cP, &g, sizeof(g)));
  float* d = nullptr;
  RK(cudaMalloc((void**)&d, sizeof(float) * ((size_t)8 * n + fny)));
  float *dps = d, *dph = d + n, *dU = d + 2 * n, *dD = d + 3 * n;
  float *nps = d + 4 * n, *nph = d + 5 * n, *nU = d + 6 * n, *nD = d + 7 * n, *dy = d + 8 * n;
  curandState* st = nullptr;
  RK(cudaMalloc((void**)&st, sizeof(curandState) * n));
  RK(cudaMemcpy(dps, ps, sizeof(float) * n, cudaMemcpyHostToDevice));
  RK(cudaMemcpy(dph, ph, sizeof(float) * n, cudaMemcpyHostToDevice));
  RK(cudaMemcpy(dU, U, sizeof(float) * n, cudaMemcpyHostToDevice));
  RK(cudaMemcpy(dD, D, sizeof(float) * n, cudaMemcpyHostToDevice));
  RK(cudaMemcpy(dy, y, sizeof(float) * fny, cudaMemcpyHostToDevice));
  RK(cudaMemcpy(nps, ps, sizeof(float) * n, cudaMemcpyHostToDevice));
  RK(cudaMemcpy(nph, ph, sizeof(float) * n, cudaMemcpyHostToDevice));
  RK(cudaMemcpy(nU, U, sizeof(float) * n, cudaMemcpyHostToDevice));
  RK(cudaMemcpy(nD, D, sizeof(float) * n, cudaMemcpyHostToDevice));
  const int b1 = (fnx + fny + 127) / 128, b2 = (n + 127) / 128;
  const int bsh = (fnx * (fny - 2) + REAL_DIM - 1) / REAL_DIM;
  init_rand_num<<<b2, 128>>>(st, p->seed_val, n);
  set_BC<<<b1, 128>>>(dps, dph, dU, dD, fnx, fny);
  if (prestep)
    rhs_psi<<<b2, 128>>>(dps, dph, dU, nps, nph, dy, nD, fnx, fny, 0, st, intR, lT);
  else
    merge_PF<<<bsh, BLOCK_DIM_X>>>(dps, dph, dU, nps, nph, nU, dD, nD, dy, fnx, fny, 1, st, intR, lT);
  RK(cudaGetLastError());
  RK(cudaDeviceSynchronize());
  RK(cudaMemcpy(ps_n, nps, sizeof(float) * n, cudaMemcpyDeviceToHost));
  RK(cudaMemcpy(ph_n, nph, sizeof(float) * n, cudaMemcpyDeviceToHost));
  RK(cudaMemcpy(U_n, nU, sizeof(float) * n, cudaMemcpyDeviceToHost));
  RK(cudaMemcpy(D_n, nD, sizeof(float) * n, cudaMemcpyDeviceToHost));
  cudaFree(st);
  cudaFree(d);
  return 0;
}

// The reference's setup(): Mt steps of its own time loop from host psi/phi/U,
// with the macro tables of the run; psi, phi, U and y are overwritten with what
// setup() copies back (PF.cu:822-825).
extern "C" int ref2d_setup(const cupf_ek2d_params* p, int Nt, float* t_mac, float* Gt, float* Rt,
                           float* x, float* y, float* phi, float* psi, float* U) {
  GlobalConstants g = to_ref(p);
  Mac_input mac;
  memset(&mac, 0, sizeof(mac));
  mac.Nt = Nt;
  mac.t_mac = t_mac;
  mac.Gt = Gt;
  mac.Rt = Rt;
  setup(mac, g, p->nx + 2, p->ny + 3, x, y, phi, psi, U);
  return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

// Device time of nsteps iterations of the reference's step pair (set_BC +
// merge_PF, PF.cu:793-809) on the given state, ping-ponging its buffers as
// setup() does; CUDA events around the launches.
extern "C" int ref2d_time_steps(const cupf_ek2d_params* p, const float* ps, const float* ph,
                                const float* U, const float* D, const float* y, float intR,
                                float lT, int nsteps, float* ms) {
  const int fnx = p->nx + 2, fny = p->ny + 3, n = fnx * fny;
  GlobalConstants g = to_ref(p);
  RK(cudaMemcpyToSymbol(cP, &g, sizeof(g)));
  float* d = nullptr;
  RK(cudaMalloc((void**)&d, sizeof(float) * ((size_t)8 * n + fny)));
  float *aps = d, *aph = d + n, *aU = d + 2 * n, *aD = d + 3 * n;
  float *bps = d + 4 * n, *bph = d + 5 * n, *bU = d + 6 * n, *bD = d + 7 * n, *dy = d + 8 * n;
  curandState* st = nullptr;
  RK(cudaMalloc((void**)&st, sizeof(curandState) * n));
  const float* src[4] = {ps, ph, U, D};
  float* dst[8] = {aps, aph, aU, aD, bps, bph, bU, bD};
  for (int f = 0; f < 8; ++f) RK(cudaMemcpy(dst[f], src[f % 4], sizeof(float) * n, cudaMemcpyHostToDevice));
  RK(cudaMemcpy(dy, y, sizeof(float) * fny, cudaMemcpyHostToDevice));
  const int b1 = (fnx + fny + 127) / 128, b2 = (n + 127) / 128;
  const int bsh = (fnx * (fny - 2) + REAL_DIM - 1) / REAL_DIM;
  init_rand_num<<<b2, 128>>>(st, p->seed_val, n);
  cudaEvent_t e0, e1;
  RK(cudaEventCreate(&e0));
  RK(cudaEventCreate(&e1));
  for (int rep = 0; rep < 2; ++rep) {  // first pass warms up
    RK(cudaEventRecord(e0));
    for (int s = 0; s < nsteps; ++s) {
      float *ips = (s & 1) ? bps : aps, *iph = (s & 1) ? bph : aph, *iU = (s & 1) ? bU : aU,
            *iD = (s & 1) ? bD : aD;
      float *ops = (s & 1) ? aps : bps, *oph = (s & 1) ? aph : bph, *oU = (s & 1) ? aU : bU,
            *oD = (s & 1) ? aD : bD;
      set_BC<<<b1, 128>>>(ips, iph, iU, iD, fnx, fny);
      merge_PF<<<bsh, BLOCK_DIM_X>>>(ips, iph, iU, ops, oph, oU, iD, oD, dy, fnx, fny, s + 1, st,
                                      intR, lT);
    }
    RK(cudaEventRecord(e1));
    RK(cudaEventSynchronize(e1));
  }
  RK(cudaGetLastError());
  RK(cudaEventElapsedTime(ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(st);
  cudaFree(d);
  return 0;
}
