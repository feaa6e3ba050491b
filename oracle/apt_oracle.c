/*
 * apt_oracle.c — TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the reference cuPF 3D APT (active parameter tracking)
 * phase-field step, used as the checker for the CUDA library: only the tests,
 * the smoke check and the CPU-baseline leg of the benchmark call it.  Nothing in
 * the product links it.
 *
 * It restates, in reference layout (idx = i + j*fnx + k*fnx*fny + slot*length):
 *   oracle_rhs_psi_f32 / _f64  APTrhs_psi            3DgrainMPI/APTPhaseField.cu:178-354
 *                              kine_ani              3DgrainMPI/APTPhaseField.cu:36-52
 *                              interp3Dtemperature   3DgrainMPI/devicefunc.cu_inl:85-125
 *   oracle_set_bc_*            APTsetBC3D            3DgrainMPI/APTPhaseField.cu:93-174
 *   oracle_collect             APTcollect_PF         3DgrainMPI/APTPhaseField.cu:55-75
 *   oracle_ini                 APTini_PF             3DgrainMPI/APTPhaseField.cu:78-89
 *   oracle_move_frame          APTmove_frame+APTcopy_frame  3DgrainMPI/APTPhaseField.cu:357-410
 *   oracle_tip_scan            ave_x + tip_mvf       3DgrainMPI/PhaseField.cu:366-399
 * and the full (non-APT, -a) mode of PhaseField.cu in the last section
 * (oracle_dense_*: set_BC_3D, rhs_psi, collect_PF, ini_PF, move/copy_frame).
 *
 * Two arithmetic modes:
 *   f32: single precision with the same operation order as the reference source.
 *        nvcc contracts a*b+c into fused multiply-adds; which sums it fuses is a
 *        compiler decision, so every site where a product meets a sum is a
 *        switch (oracle_set_contraction).  The switches are pinned by comparing
 *        this mode bit-for-bit against dumps of the reference kernels compiled
 *        for sm_100a (tests/golden).  Compiled with -ffp-contract=off so the C
 *        compiler adds no fusions of its own.
 *   f64: the same algorithm in double precision (state, coordinates, angles and
 *        time in double) — the FP64 transcription used for tolerance checks and
 *        as the CPU baseline.
 *
 * Semantics pinned explicitly where the reference is undefined:
 *   H1 merge overflow (more than NUM_PF distinct ids in a 7-point stencil): the
 *      reference writes local_phs[s][NUM_PF], which aliases local_phs[s+1][0]
 *      for s < 6 (restated here; entries counted in stats[0]), and lands past
 *      the array for s == 6 (dropped here; counted in stats[1]).
 *   Boundary edges/corners: APTsetBC3D fills faces in parallel, so cells on two
 *      or three halo faces race in the reference.  Here every halo coordinate is
 *      mapped independently, which is what sequential z, y, x face fills give.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/cupf.h"

#define LS (-0.995)
#define NPMAX CUPF_MAX_PF

/* ---------------------------------------------------------------- contraction sites */
enum {
  S_AS = 0,  /* a_s = 1 + 3*kd                         : 0 add, 1 fma */
  S_UX_IN,   /* (cosa*cosb)*ux + (sina*cosb)*uy         : 0 none, 1 fuse left, 2 fuse right */
  S_UX_OUT,  /* s - sinb*uz                             : 0 none, 1 fma */
  S_UY,      /* (-sina)*ux + cosa*uy                    : 0/1/2 */
  S_UZ_IN,   /* (cosa*sinb)*ux + (sina*sinb)*uy         : 0/1/2 */
  S_UZ_OUT,  /* s + cosb*uz                             : 0/1 */
  S_MAG_IN,  /* ux2 + uy2 (squares)                     : 0/1/2 */
  S_MAG_OUT, /* + uz2                                   : 0/1 */
  S_Q_IN,    /* ux2*ux2 + uy2*uy2                       : 0/1/2 */
  S_Q_OUT,   /* + uz2*uz2                               : 0/1 */
  S_DIFF,    /* sum6 - 6*phC                            : 0/1 */
  S_REP,     /* repul + (0.25*(p+1))*(p+1)              : 0/1 */
  S_W,       /* 1 - phC*phC                             : 0/1 */
  S_E1,      /* (diff*hi)*hi + w*phC                    : 0/1/2 */
  S_INNER,   /* w*w - (6*(phC+1))*repul                 : 0 none, 1 fma(w,w,-m*r), 2 fma(-m,r,w*w) */
  S_RHS,     /* E1 - (lamd*Up)*inner                    : 0/1 */
  S_NEW,     /* phC + dt*dphi                           : 0/1 */
  S_TD,      /* (double)a - (UC*1e6)*t in double        : 0/1 */
  /* thermalType 3 (cone) and 4 (paraboloid table) */
  S_T3_YU,   /* y - 0.5*lyd                             : 0/1 */
  S_T3_SQ,   /* u*u + zt*zt                             : 0/1/2 */
  S_T3_SKIP, /* lm + (V*t)*1e6 in double                : 0/1 */
  S_T3_TD,   /* (double)(-G*dist) - (UC*1e6)*t          : 0/1 */
  S_T4_XQ,   /* (double)x - (V*t)*1e6                   : 0/1 */
  S_T4_P1,   /* a*u0 + b*u1 (trilinear corner weights)  : 0/1/2 */
  S_T4_P2,   /* + c*u2                                  : 0/1 */
  S_T4_P3,   /* + d*u3                                  : 0/1 */
  S_T4_Z,    /* p0*(1-dz) + p1*dz                       : 0/1/2 */
  S_T4_Q1,   /* the upper bracket's a*u0 + b*u1         : 0/1/2 */
  S_T4_Q2,   /* + c*u2                                  : 0/1 */
  S_T4_Q3,   /* + d*u3                                  : 0/1 */
  S_NSITES
};

static int g_cfg[S_NSITES] = {1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1,
                              0, 1, 1, 1, 0, 1, 1, 1, 1, 1, 1, 1};

int oracle_num_sites(void) { return S_NSITES; }

void oracle_set_contraction(const int32_t* cfg, int n) {
  for (int i = 0; i < n && i < S_NSITES; ++i) g_cfg[i] = cfg[i];
}

void oracle_get_contraction(int32_t* cfg, int n) {
  for (int i = 0; i < n && i < S_NSITES; ++i) cfg[i] = g_cfg[i];
}

/* x*y + u*v under contraction mode m */
static inline float sop(float x, float y, float u, float v, int m) {
  if (m == 1) return fmaf(x, y, u * v);
  if (m == 2) return fmaf(u, v, x * y);
  return x * y + u * v;
}

/* ---------------------------------------------------------------- index helpers */
typedef struct {
  int fnx, fny, fnz, np;
  int64_t len;
} grid_t;

static inline grid_t mkgrid(const cupf_apt_params* p) {
  grid_t g;
  g.fnx = p->fnx;
  g.fny = p->fny;
  g.fnz = p->fnz;
  g.np = p->num_pf;
  g.len = (int64_t)p->fnx * p->fny * p->fnz;
  return g;
}

/* ---------------------------------------------------------------- merge (shared by both modes)
 * Builds, for the cell C, the list of active grain ids in first-seen order over
 * stencil points (D,B,L,C,R,T,U) x slots, exactly as APTPhaseField.cu:211-233,
 * and src[s][j] = flat index whose phi feeds local_phs[s][j] (-1 -> -1.0). */
static inline void apt_merge(const grid_t* g, int64_t C, const int32_t* aarg, int32_t* L,
                             int64_t src[7][NPMAX], int64_t* n_overflow_u, int64_t* n_alias) {
  const int np = g->np;
  for (int a = 0; a < np; ++a) {
    L[a] = -1;
    for (int s = 0; s < 7; ++s) src[s][a] = -1;
  }
  const int64_t sx = 1, sy = g->fnx, sz = (int64_t)g->fnx * g->fny;
  const int64_t off[7] = {-sz, -sy, -sx, 0, sx, sy, sz};
  for (int s = 0; s < 7; ++s) {
    for (int pf = 0; pf < np; ++pf) {
      int64_t gc = C + off[s] + (int64_t)pf * g->len;
      int32_t id = aarg[gc];
      if (id == -1) continue;
      int a;
      for (a = 0; a < np; ++a) {
        if (L[a] == id) break;
        if (L[a] == -1) {
          L[a] = id;
          break;
        }
      }
      if (a < np) {
        src[s][a] = gc;
      } else if (s < 6) {
        src[s + 1][0] = gc; /* local_phs[s][NUM_PF] == local_phs[s+1][0] */
        (*n_alias)++;
      } else {
        (*n_overflow_u)++;
      }
    }
  }
}

/* ---------------------------------------------------------------- FP32 mode */
static float kine_ani_f32(float ux, float uy, float uz, float cosa, float sina, float cosb,
                          float sinb, float kd, float eps) {
  float a_s = g_cfg[S_AS] ? fmaf(3.0f, kd, 1.0f) : 1.0f + 3.0f * kd;
  float epsilon = -4.0f * kd / a_s;
  float s = sop(cosa * cosb, ux, sina * cosb, uy, g_cfg[S_UX_IN]);
  float rx = g_cfg[S_UX_OUT] ? fmaf(-sinb, uz, s) : s - sinb * uz;
  float ry = sop(-sina, ux, cosa, uy, g_cfg[S_UY]) + 0.0f;
  s = sop(cosa * sinb, ux, sina * sinb, uy, g_cfg[S_UZ_IN]);
  float rz = g_cfg[S_UZ_OUT] ? fmaf(cosb, uz, s) : s + cosb * uz;
  float ux2 = rx * rx, uy2 = ry * ry, uz2 = rz * rz;
  float mag = sop(rx, rx, ry, ry, g_cfg[S_MAG_IN]);
  mag = g_cfg[S_MAG_OUT] ? fmaf(rz, rz, mag) : mag + uz2;
  float mag2 = mag * mag;
  if (mag > eps) {
    float q = sop(ux2, ux2, uy2, uy2, g_cfg[S_Q_IN]);
    q = g_cfg[S_Q_OUT] ? fmaf(uz2, uz2, q) : q + uz2 * uz2;
    return a_s * (1.0f + epsilon * q / mag2);
  }
  return 1.0f;
}

/* interp3Dtemperature, devicefunc.cu_inl:85-125 (single precision, left-to-right) */
static float interp3d_f32(const float* u, float x, float y, float z, int Nx, int Ny, int Nz,
                          float Dx) {
  int kx = (int)(x / Dx), ky = (int)(y / Dx), kz = (int)(z / Dx);
  float dx = x / Dx - (float)kx, dy = y / Dx - (float)ky, dz = z / Dx - (float)kz;
  if (kx == Nx - 1) { kx = Nx - 2; dx = 1.0f; }
  if (ky == Ny - 1) { ky = Ny - 2; dy = 1.0f; }
  if (kz == Nz - 1) { kz = Nz - 2; dz = 1.0f; }
  int64_t o = kx + (int64_t)ky * Nx + (int64_t)kz * Nx * Ny;
  int64_t on = kx + (int64_t)ky * Nx + (int64_t)(kz + 1) * Nx * Ny;
  float a = (1.0f - dx) * (1.0f - dy), b = (1.0f - dx) * dy, c = dx * (1.0f - dy), d = dx * dy;
  float p0 = sop(a, u[o], b, u[o + Nx], g_cfg[S_T4_P1]);
  p0 = g_cfg[S_T4_P2] ? fmaf(c, u[o + 1], p0) : p0 + c * u[o + 1];
  p0 = g_cfg[S_T4_P3] ? fmaf(d, u[o + Nx + 1], p0) : p0 + d * u[o + Nx + 1];
  float p1 = sop(a, u[on], b, u[on + Nx], g_cfg[S_T4_Q1]);
  p1 = g_cfg[S_T4_Q2] ? fmaf(c, u[on + 1], p1) : p1 + c * u[on + 1];
  p1 = g_cfg[S_T4_Q3] ? fmaf(d, u[on + Nx + 1], p1) : p1 + d * u[on + Nx + 1];
  return sop(p0, 1.0f - dz, p1, dz, g_cfg[S_T4_Z]);
}

/* Thermal undercooling at (i,j,k,t); returns 0 when the reference `continue`s
 * (slot left unwritten), 1 otherwise.  APTPhaseField.cu:278-327 */
static int tinterp_f32(const cupf_apt_params* p, const cupf_apt_inputs* th, int i, int j, int k,
                       float t, int use_iuc, float* Tout) {
  float T = 0.0f;
  if (use_iuc) {
    double r = (double)(-p->underCoolingRate0) * 1e6 * (double)t;
    T = (float)r;
  } else if (p->thermalType == 1) {
    float a = p->G * (th->z[k] - p->z0);
    double m = (double)p->underCoolingRate * 1e6;
    double r = g_cfg[S_TD] ? fma(-m, (double)t, (double)a) : (double)a - m * (double)t;
    T = (float)r;
  } else if (p->thermalType == 2) {
    float a = th->y[j] - 0.5f * p->lyd;
    float b = th->z[k] - p->z0 - p->lzd;
    float dist = sqrtf(fmaf(a, a, b * b)) - p->r0;
    double m = (double)p->underCoolingRate * 1e6;
    T = (float)fma(-m, (double)t, (double)(-p->G * dist));
  } else if (p->thermalType == 3) {
    float lm = (p->r0 - p->z0) / tanf(p->angle);
    float xl = th->x[i] - 0.0f;
    float r0x = p->z0 + (p->r0 - p->z0) * xl / lm;
    float a = g_cfg[S_T3_YU] ? fmaf(-0.5f, p->lyd, th->y[j]) : th->y[j] - 0.5f * p->lyd;
    float zt = p->z0 + p->lzd - th->z[k];
    float dist = cosf(p->angle) * (sqrtf(sop(a, a, zt, zt, g_cfg[S_T3_SQ])) - r0x);
    double vt = (double)(p->V * t);
    if ((double)xl > (g_cfg[S_T3_SKIP] ? fma(vt, 1e6, (double)lm) : (double)lm + vt * 1e6)) return 0;
    double m = (double)p->underCoolingRate * 1e6;
    double gd = (double)(-p->G * dist);
    T = (float)(g_cfg[S_T3_TD] ? fma(-m, (double)t, gd) : gd - m * (double)t);
  } else if (p->thermalType == 4) {
    double vt = (double)(p->V * t);
    float xq = (float)(g_cfg[S_T4_XQ] ? fma(-vt, 1e6, (double)th->x[i]) : (double)th->x[i] - vt * 1e6);
    if (xq > p->mp_len + p->x0 || xq < 0.0f) return 0;
    float Dx = th->X_mac[1] - th->X_mac[0];
    float v = interp3d_f32(th->psi_mac, xq - th->X_mac[0], th->y[j] - th->Y_mac[0],
                           th->z[k] - th->Z_mac[0], p->Nx, p->Ny, p->Nz, Dx);
    T = (p->order == 100.0f) ? -v : -p->G * v;
  } else if (p->thermalType == 5) {
    /* the library's analytic paraboloid melt pool (apt_update.cuh tinterp, no
       counterpart in the reference), every operation rounded separately */
    float vt = p->V * t;
    float xb = (float)((double)p->x0 + (double)vt * 1e6);
    float xi = xb - th->x[i];
    float u = th->y[j] - 0.5f * p->lyd;
    float w = (p->z0 + p->lzd) - th->z[k];
    float uu = u * u, ww = w * w;
    float rr = uu + ww;
    float dist;
    if (xi <= 0.0f) {
      float xx = xi * xi;
      dist = sqrtf(rr + xx) - p->r0;
    } else if (xi < p->mp_len) {
      float q = xi / p->mp_len;
      float R = p->r0 * sqrtf(1.0f - q);
      dist = sqrtf(rr) - R;
    } else {
      dist = sqrtf(rr);
    }
    double m = (double)p->underCoolingRate * 1e6;
    float gd = -p->G * dist;
    double mt = m * (double)t;
    T = (float)((double)gd - mt);
  }
  *Tout = T;
  return 1;
}

/* One explicit step, single precision.  stats (may be NULL): [0] cells with a
 * merge overflow entries at s<6 (aliased), [1] entries dropped at s==6. */
void oracle_rhs_psi_f32(const cupf_apt_params* p, const cupf_apt_inputs* th, float t,
                        const float* ph, float* ph_new, const int32_t* aarg, int32_t* aarg_new,
                        int use_iuc, int64_t* stats) {
  grid_t g = mkgrid(p);
  const int np = g.np;
  int64_t ovf_u = 0, ovf_a = 0;
#pragma omp parallel for collapse(2) schedule(static) reduction(+ : ovf_u, ovf_a)
  for (int j = 1; j < g.fny - 1; ++j) {
    for (int i = 1; i < g.fnx - 1; ++i) {
      for (int k = 1; k < g.fnz - 1; ++k) {
        int64_t C = (int64_t)k * g.fnx * g.fny + (int64_t)j * g.fnx + i;
        int32_t L[NPMAX];
        int64_t src[7][NPMAX];
        apt_merge(&g, C, aarg, L, src, &ovf_u, &ovf_a);
        float lp[7][NPMAX];
        for (int s = 0; s < 7; ++s)
          for (int a = 0; a < np; ++a) lp[s][a] = src[s][a] >= 0 ? ph[src[s][a]] : -1.0f;
        for (int a = 0; a < np; ++a) {
          int64_t o = C + (int64_t)a * g.len;
          if (L[a] == -1) {
            aarg_new[o] = -1;
            ph_new[o] = -1.0f;
            continue;
          }
          int id = L[a];
          float phD = lp[0][a], phB = lp[1][a], phL = lp[2][a], phC = lp[3][a], phR = lp[4][a],
                phT = lp[5][a], phU = lp[6][a];
          float phx = (phR - phL) * 0.5f, phy = (phT - phB) * 0.5f, phz = (phU - phD) * 0.5f;
          float cosa, sina, cosb, sinb;
          if ((double)phC > LS) {
            int tid = id <= p->num_theta ? id : (id % p->num_theta) + 1;
            sina = th->sint[tid];
            cosa = th->cost[tid];
            sinb = th->sint[tid + p->num_theta];
            cosb = th->cost[tid + p->num_theta];
          } else {
            sina = 0.0f;
            cosa = 1.0f;
            sinb = 0.0f;
            cosb = 1.0f;
          }
          float A2 = kine_ani_f32(phx, phy, phz, cosa, sina, cosb, sinb, p->kin_delta, p->eps);
          float sum = phR + phL + phT + phB + phU + phD;
          float diff = g_cfg[S_DIFF] ? fmaf(-6.0f, phC, sum) : sum - 6.0f * phC;
          float Tinterp;
          if (!tinterp_f32(p, th, i, j, k, t, use_iuc, &Tinterp)) continue;
          float Up = Tinterp / p->L_cp;
          float repul = 0.0f;
          for (int b = 0; b < np; ++b) {
            if (b == a) continue;
            float q = lp[3][b] + 1.0f;
            repul = g_cfg[S_REP] ? fmaf(0.25f * q, q, repul) : repul + 0.25f * q * q;
          }
          float w = g_cfg[S_W] ? fmaf(-phC, phC, 1.0f) : 1.0f - phC * phC;
          float dh = diff * p->hi;
          float E1 = sop(dh, p->hi, w, phC, g_cfg[S_E1]);
          float m6 = 6.0f * (phC + 1.0f);
          float inner;
          if (g_cfg[S_INNER] == 1) inner = fmaf(w, w, -(m6 * repul));
          else if (g_cfg[S_INNER] == 2) inner = fmaf(-m6, repul, w * w);
          else inner = w * w - m6 * repul;
          float lu = p->lamd * Up;
          float rhs = g_cfg[S_RHS] ? fmaf(-lu, inner, E1) : E1 - lu * inner;
          float dphi = rhs / A2;
          float nv = g_cfg[S_NEW] ? fmaf(p->dt, dphi, phC) : phC + p->dt * dphi;
          ph_new[o] = nv;
          aarg_new[o] = ((double)nv < -0.9999) ? -1 : id;
        }
      }
    }
  }
  if (stats) {
    stats[0] += ovf_a;
    stats[1] += ovf_u;
  }
}

/* ---------------------------------------------------------------- FP64 mode */
typedef struct {
  const double* x;
  const double* y;
  const double* z;
  const double* sint;
  const double* cost;
} oracle_thermal_f64;

static double kine_ani_f64(double ux, double uy, double uz, double cosa, double sina, double cosb,
                           double sinb, double kd, double eps) {
  double a_s = 1.0 + 3.0 * kd;
  double epsilon = -4.0 * kd / a_s;
  double rx = cosa * cosb * ux + sina * cosb * uy - sinb * uz;
  double ry = -sina * ux + cosa * uy;
  double rz = cosa * sinb * ux + sina * sinb * uy + cosb * uz;
  double ux2 = rx * rx, uy2 = ry * ry, uz2 = rz * rz;
  double mag = ux2 + uy2 + uz2;
  if (mag > eps) return a_s * (1.0 + epsilon * (ux2 * ux2 + uy2 * uy2 + uz2 * uz2) / (mag * mag));
  return 1.0;
}

/* One explicit step in double precision; thermalType 0, 1 and the initial
 * undercooling only (the analytic line profile of the benchmark configs). */
int oracle_rhs_psi_f64(const cupf_apt_params* p, const oracle_thermal_f64* th, double t,
                       const double* ph, double* ph_new, const int32_t* aarg, int32_t* aarg_new,
                       int use_iuc, int64_t* stats) {
  if (!use_iuc && p->thermalType != 0 && p->thermalType != 1 && p->thermalType != 5) return -1;
  grid_t g = mkgrid(p);
  const int np = g.np;
  int64_t ovf_u = 0, ovf_a = 0;
#pragma omp parallel for collapse(2) schedule(static) reduction(+ : ovf_u, ovf_a)
  for (int j = 1; j < g.fny - 1; ++j) {
    for (int i = 1; i < g.fnx - 1; ++i) {
      for (int k = 1; k < g.fnz - 1; ++k) {
        int64_t C = (int64_t)k * g.fnx * g.fny + (int64_t)j * g.fnx + i;
        int32_t L[NPMAX];
        int64_t src[7][NPMAX];
        apt_merge(&g, C, aarg, L, src, &ovf_u, &ovf_a);
        double lp[7][NPMAX];
        for (int s = 0; s < 7; ++s)
          for (int a = 0; a < np; ++a) lp[s][a] = src[s][a] >= 0 ? ph[src[s][a]] : -1.0;
        double T = 0.0;
        if (use_iuc) T = -(double)p->underCoolingRate0 * 1e6 * t;
        else if (p->thermalType == 1)
          T = (double)p->G * (th->z[k] - (double)p->z0) - (double)p->underCoolingRate * 1e6 * t;
        else if (p->thermalType == 5) {
          /* analytic paraboloid melt pool in double (apt_update.cuh tinterp64) */
          double xi = (double)p->x0 + (double)p->V * 1e6 * t - th->x[i];
          double u = th->y[j] - 0.5 * (double)p->lyd;
          double w = (double)p->z0 + (double)p->lzd - th->z[k];
          double rr = u * u + w * w, dist;
          if (xi <= 0.0) dist = sqrt(rr + xi * xi) - (double)p->r0;
          else if (xi < (double)p->mp_len)
            dist = sqrt(rr) - (double)p->r0 * sqrt(1.0 - xi / (double)p->mp_len);
          else dist = sqrt(rr);
          T = -(double)p->G * dist - (double)p->underCoolingRate * 1e6 * t;
        }
        double Up = T / (double)p->L_cp;
        for (int a = 0; a < np; ++a) {
          int64_t o = C + (int64_t)a * g.len;
          if (L[a] == -1) {
            aarg_new[o] = -1;
            ph_new[o] = -1.0;
            continue;
          }
          int id = L[a];
          double phD = lp[0][a], phB = lp[1][a], phL = lp[2][a], phC = lp[3][a], phR = lp[4][a],
                 phT = lp[5][a], phU = lp[6][a];
          double cosa = 1, sina = 0, cosb = 1, sinb = 0;
          if (phC > LS) {
            int tid = id <= p->num_theta ? id : (id % p->num_theta) + 1;
            sina = th->sint[tid];
            cosa = th->cost[tid];
            sinb = th->sint[tid + p->num_theta];
            cosb = th->cost[tid + p->num_theta];
          }
          double A2 = kine_ani_f64((phR - phL) * 0.5, (phT - phB) * 0.5, (phU - phD) * 0.5, cosa,
                                   sina, cosb, sinb, (double)p->kin_delta, (double)p->eps);
          double diff = phR + phL + phT + phB + phU + phD - 6.0 * phC;
          double repul = 0.0;
          for (int b = 0; b < np; ++b)
            if (b != a) repul += 0.25 * (lp[3][b] + 1.0) * (lp[3][b] + 1.0);
          double w = 1.0 - phC * phC;
          double hi = (double)p->hi;
          double rhs = diff * hi * hi + w * phC -
                       (double)p->lamd * Up * (w * w - 6.0 * (phC + 1.0) * repul);
          double nv = phC + (double)p->dt * rhs / A2;
          ph_new[o] = nv;
          aarg_new[o] = nv < -0.9999 ? -1 : id;
        }
      }
    }
  }
  if (stats) {
    stats[0] += ovf_a;
    stats[1] += ovf_u;
  }
  return 0;
}

/* ---------------------------------------------------------------- boundary fill */
static inline int bc_map(int c, int fn, int bc) {
  if (c == 0) return bc == 0 ? 2 : fn - 2;
  if (c == fn - 1) return bc == 0 ? fn - 3 : 1;
  return c;
}

#define DEFINE_SET_BC(NAME, T)                                                              \
  void NAME(const cupf_apt_params* p, T* ph, int32_t* ids) {                                \
    grid_t g = mkgrid(p);                                                                   \
    for (int pf = 0; pf < g.np; ++pf)                                                       \
      for (int k = 0; k < g.fnz; ++k)                                                       \
        for (int j = 0; j < g.fny; ++j)                                                     \
          for (int i = 0; i < g.fnx; ++i) {                                                 \
            int hk = (k == 0 || k == g.fnz - 1), hj = (j == 0 || j == g.fny - 1),           \
                hi = (i == 0 || i == g.fnx - 1);                                            \
            if (!(hk || hj || hi)) continue;                                                \
            int si = bc_map(i, g.fnx, p->bcX), sj = bc_map(j, g.fny, p->bcY),               \
                sk = bc_map(k, g.fnz, p->bcZ);                                              \
            int64_t d = i + (int64_t)j * g.fnx + (int64_t)k * g.fnx * g.fny + pf * g.len;   \
            int64_t s = si + (int64_t)sj * g.fnx + (int64_t)sk * g.fnx * g.fny + pf * g.len; \
            ph[d] = ph[s];                                                                  \
            ids[d] = ids[s];                                                                \
          }                                                                                 \
  }

DEFINE_SET_BC(oracle_set_bc_f32, float)
DEFINE_SET_BC(oracle_set_bc_f64, double)

/* ---------------------------------------------------------------- argmax / init */
void oracle_collect(const cupf_apt_params* p, const float* PFs, const int32_t* ids, float* phi,
                    int32_t* alpha) {
  grid_t g = mkgrid(p);
  for (int64_t C = 0; C < g.len; ++C) {
    int am = 0;
    for (int pf = 0; pf < g.np; ++pf)
      if (PFs[C + pf * g.len] > PFs[C + am * g.len]) am = pf;
    float v = PFs[C + am * g.len];
    if ((double)v > LS) {
      phi[C] = v;
      alpha[C] = ids[C + am * g.len];
    }
  }
}

void oracle_collect_f64(const cupf_apt_params* p, const double* PFs, const int32_t* ids,
                        double* phi, int32_t* alpha) {
  grid_t g = mkgrid(p);
  for (int64_t C = 0; C < g.len; ++C) {
    int am = 0;
    for (int pf = 0; pf < g.np; ++pf)
      if (PFs[C + pf * g.len] > PFs[C + am * g.len]) am = pf;
    double v = PFs[C + am * g.len];
    if (v > LS) {
      phi[C] = v;
      alpha[C] = ids[C + am * g.len];
    }
  }
}

void oracle_ini(const cupf_apt_params* p, float* PFs, int32_t* ids, const float* phi,
                const int32_t* alpha) {
  grid_t g = mkgrid(p);
  for (int64_t C = 0; C < (int64_t)g.np * g.len; ++C) {
    PFs[C] = -1.0f;
    ids[C] = -1;
  }
  for (int64_t C = 0; C < g.len; ++C)
    if ((double)phi[C] > LS) {
      PFs[C] = phi[C];
      ids[C] = alpha[C];
    }
}

/* ---------------------------------------------------------------- moving domain */
/* Per-layer sum of phi over all slots and cells, then the tip scan of tip_mvf:
 * advance *tip while mean(layer) > LS and tip < fnz-1. */
void oracle_tip_scan(const cupf_apt_params* p, const float* PFs, double* meanx, int32_t* tip) {
  grid_t g = mkgrid(p);
  int64_t plane = (int64_t)g.fnx * g.fny;
  for (int k = 0; k < g.fnz; ++k) {
    double s = 0.0;
    for (int pf = 0; pf < g.np; ++pf)
      for (int64_t c = 0; c < plane; ++c) s += PFs[pf * g.len + k * plane + c];
    meanx[k] = s;
  }
  float denom = (float)(g.np * g.fnx * g.fny);
  while (((double)((float)meanx[*tip] / denom) > LS) && (*tip < g.fnz - 1)) (*tip)++;
}

/* One layer shift: APTmove_frame followed by APTcopy_frame.  alpha is the argmax
 * map collected just before; its layer k=1 (all i, j) is archived at
 * alpha_full[move_count*fnx*fny + fnx*fny + j*fnx + i] (the reference indexes
 * with the cell's own C, which includes the k=1 plane offset) and counted into
 * loss_area[alpha-1] for alpha in 1..num_theta. */
void oracle_move_frame(const cupf_apt_params* p, float* PFs, int32_t* ids, float* z,
                       const int32_t* alpha, int32_t* alpha_full, int32_t* loss_area,
                       int move_count) {
  grid_t g = mkgrid(p);
  int64_t plane = (int64_t)g.fnx * g.fny;
  for (int64_t c = 0; c < plane; ++c) {
    int32_t a = alpha[plane + c];
    alpha_full[(int64_t)move_count * plane + plane + c] = a;
    if (a >= 1 && a <= p->num_theta) loss_area[a - 1] += 1;
  }
  for (int pf = 0; pf < g.np; ++pf)
    for (int k = 1; k < g.fnz - 1; ++k)
      for (int j = 1; j < g.fny - 1; ++j)
        for (int i = 1; i < g.fnx - 1; ++i) {
          int64_t C = pf * g.len + k * plane + (int64_t)j * g.fnx + i;
          if (k < g.fnz - 2) {
            PFs[C] = PFs[C + plane];
            ids[C] = ids[C + plane];
          } else {
            PFs[C] = -1.0f;
            ids[C] = -1;
          }
        }
  float ztop = 2.0f * z[g.fnz - 2] - z[g.fnz - 3];
  for (int k = 1; k < g.fnz - 2; ++k) z[k] = z[k + 1];
  z[g.fnz - 2] = ztop;
}

/* ---------------------------------------------------------------- nucleation
 * add_nucl (APTPhaseField.cu:459-536) with the library's defined draw: Philox4x32-10
 * (Salmon et al., SC 2011) keyed on (seed, coarse cell, step) instead of curand.
 * Same probability (nuncl_possibility :446-455, evaluated in double), same table
 * interpolation (interp4Dtemperature, devicefunc.cu_inl:32-83, separate roundings),
 * same nucleus profile table and id rule as the CUDA kernel. */
typedef struct { uint32_t v[4]; } philox4_t;

static philox4_t philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0,
                               uint32_t k1) {
  for (int r = 0; r < 10; ++r) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0, hi1 = (uint32_t)(p1 >> 32),
             lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
    c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  philox4_t o = {{c0, c1, c2, c3}};
  return o;
}

void oracle_philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1,
                   uint32_t* out) {
  philox4_t r = philox4x32_10(c0, c1, c2, c3, k0, k1);
  for (int i = 0; i < 4; ++i) out[i] = r.v[i];
}

static float uniform01(uint32_t x) { return (float)((x >> 8) + 1u) * (1.0f / 16777216.0f); }

static float interp4d_f32(const float* u, float x, float y, float z, float t, int Nx, int Ny,
                          int Nz, int Nt, float Dx, float Dt) {
  float fx = x / Dx, fy = y / Dx, fz = z / Dx, ft = t / Dt;
  int kx = (int)fx, ky = (int)fy, kz = (int)fz, kt = (int)ft;
  float dx = fx - (float)kx, dy = fy - (float)ky, dz = fz - (float)kz, dtt = ft - (float)kt;
  if (kx == Nx - 1) { kx = Nx - 2; dx = 1.0f; }
  if (ky == Ny - 1) { ky = Ny - 2; dy = 1.0f; }
  if (kz == Nz - 1) { kz = Nz - 2; dz = 1.0f; }
  if (kt == Nt - 1) { kt = Nt - 2; dtt = 1.0f; }
  if (kx < 0) kx = 0; if (kx > Nx - 2) kx = Nx - 2;
  if (ky < 0) ky = 0; if (ky > Ny - 2) ky = Ny - 2;
  if (kz < 0) kz = 0; if (kz > Nz - 2) kz = Nz - 2;
  if (kt < 0) kt = 0; if (kt > Nt - 2) kt = Nt - 2;
  int64_t sx = 1, sy = Nx, sz = (int64_t)Nx * Ny, st = sz * Nz;
  float ex = 1.0f - dx, ey = 1.0f - dy;
  float wa = ex * ey, wb = ex * dy, wc = dx * ey, wd = dx * dy;
  int64_t o = kx + ky * sy + kz * sz + kt * st;
  float q[4];
  int64_t base[4] = {o, o + sz, o + st, o + st + sz};
  for (int m = 0; m < 4; ++m) {
    int64_t b = base[m];
    float r = wa * u[b];
    r = r + wb * u[b + sy];
    r = r + wc * u[b + sx];
    q[m] = r + wd * u[b + sy + sx];
  }
  float t0 = q[0] * (1.0f - dz) + q[1] * dz;
  float t1 = q[2] * (1.0f - dz) + q[3] * dz;
  return (1.0f - dtt) * t0 + dtt * t1;
}

static double nucl_probability(double delT, double d_delT, double nmax, double mean, double sd,
                               double rad) {
  double q = (delT - mean) / sd;
  double density = nmax / (sqrt(2.0 * 3.14159265358979323846) * sd) * exp(-0.5 * q * q) * d_delT;
  return 8.0 * rad * rad * rad * density;
}

/* Nucleus profile of add_nucl (APTPhaseField.cu:515-528): tanh(dx*((1+pts)/2 - r)/sqrt2)
 * over the (2*pts+1)^3 cube, in float with the C library's tanhf. */
void oracle_nucleus_table(const cupf_apt_params* p, float* out) {
  const int pts = p->pts_cell, w = 2 * pts + 1;
  const float pf = (float)pts;
  for (int k = -pts; k <= pts; ++k)
    for (int j = -pts; j <= pts; ++j)
      for (int i = -pts; i <= pts; ++i) {
        const float d = p->dx * ((1.0f + pf) / 2.0f - sqrtf((float)(i * i + j * j + k * k)));
        out[((k + pts) * w + (j + pts)) * w + (i + pts)] = tanhf(d / p->sqrt2);
      }
}

int oracle_nucl_dims(const cupf_apt_params* p, int32_t* cdims) {
  int w = 2 * p->pts_cell + 1;
  cdims[0] = (p->fnx - 3) / w;
  cdims[1] = (p->fny - 3) / w;
  cdims[2] = (p->fnz - 3) / w;
  return cdims[0] * cdims[1] * cdims[2];
}

/* init_nucl_status (APTPhaseField.cu:420-444), centre index without the halo offset */
void oracle_nucl_status_init(const cupf_apt_params* p, const float* PFs, int32_t* status) {
  int32_t cd[3];
  oracle_nucl_dims(p, cd);
  int w = 2 * p->pts_cell + 1;
  for (int k = 0; k < cd[2]; ++k)
    for (int j = 0; j < cd[1]; ++j)
      for (int i = 0; i < cd[0]; ++i) {
        int64_t g = (int64_t)(w * k + p->pts_cell) * p->fnx * p->fny +
                    (int64_t)(w * j + p->pts_cell) * p->fnx + (w * i + p->pts_cell);
        status[i + (int64_t)cd[0] * (j + (int64_t)cd[1] * k)] = ((double)PFs[g] > LS) ? 1 : 0;
      }
}

/* One add_nucl pass; returns the number of new nuclei. */
int oracle_nucleate(const cupf_apt_params* p, const cupf_apt_inputs* th, float* PFs, int32_t* ids,
                    int32_t* status, const float* sphere, float t, float dt2, uint32_t step,
                    int use_iuc, int id_space) {
  int32_t cd[3];
  oracle_nucl_dims(p, cd);
  grid_t g = mkgrid(p);
  int w = 2 * p->pts_cell + 1, pts = p->pts_cell, count = 0;
  for (int64_t C = 0; C < (int64_t)cd[0] * cd[1] * cd[2]; ++C) {
    if (status[C]) continue;
    int i = (int)(C % cd[0]), j = (int)((C / cd[0]) % cd[1]), k = (int)(C / ((int64_t)cd[0] * cd[1]));
    int gi = w * i + pts + 1, gj = w * j + pts + 1, gk = w * k + pts + 1;
    int64_t gc = (int64_t)gk * g.fnx * g.fny + (int64_t)gj * g.fnx + gi;
    int solid = 0;
    for (int pf = 0; pf < g.np; ++pf) solid |= (double)PFs[gc + pf * g.len] > LS;
    if (solid) { status[C] = 1; continue; }
    double P;
    if (use_iuc) {
      float delT = (float)((double)p->underCoolingRate0 * 1e6 * (double)(t + dt2));
      float d_delT = (float)((double)p->underCoolingRate0 * 1e6 * (double)dt2);
      P = nucl_probability(delT, d_delT, p->nuc_Nmax0, p->undcool_mean, p->undcool_std, p->nuc_rad);
    } else if (th->T_3D) {
      float Dx = th->X_mac[1] - th->X_mac[0], Dt = th->t_mac[1] - th->t_mac[0];
      float xq = th->x[gi] - th->X_mac[0], yq = th->y[gj] - th->Y_mac[0], zq = th->z[gk] - th->Z_mac[0];
      float T0 = interp4d_f32(th->T_3D, xq, yq, zq, t - th->t_mac[0], p->Nx, p->Ny, p->Nz, p->Nt, Dx, Dt);
      float T1 = interp4d_f32(th->T_3D, xq, yq, zq, (t + dt2) - th->t_mac[0], p->Nx, p->Ny, p->Nz, p->Nt, Dx, Dt);
      P = nucl_probability(-T1, T0 - T1, p->nuc_Nmax, p->undcool_mean, p->undcool_std, p->nuc_rad);
    } else {
      continue;
    }
    philox4_t r = philox4x32_10((uint32_t)C, step, 0x4E55434Cu, 0u, (uint32_t)p->seed, 0x5EEDu);
    if (!((double)uniform01(r.v[0]) < P)) continue;
    int id = p->num_theta + 1 + (int)(r.v[1] % (uint32_t)id_space);
    for (int dk = -pts; dk <= pts; ++dk)
      for (int dj = -pts; dj <= pts; ++dj)
        for (int di = -pts; di <= pts; ++di) {
          float v = sphere[((dk + pts) * w + (dj + pts)) * w + (di + pts)];
          int64_t o = gc + (int64_t)dk * g.fnx * g.fny + (int64_t)dj * g.fnx + di;
          PFs[o] = v;
          if (v > -0.9999f) ids[o] = id; /* float literal in add_nucl :524 */
        }
    status[C] = 1;
    count++;
  }
  return count;
}

/* ---------------------------------------------------------------- full-PF mode
 * The dense solver of PhaseField (3DgrainMPI/PhaseField.cu), one phi field per
 * grain, NUM_PF = num_theta, reference layout ph[g*length + C]:
 *   oracle_dense_set_bc     set_BC_3D   PhaseField.cu:111-166 (mirror on every face)
 *   oracle_dense_rhs_f32    rhs_psi     PhaseField.cu:168-301, kine_ani :32-50
 *   oracle_dense_collect    collect_PF  PhaseField.cu:60-88 (persistent argmax)
 *   oracle_dense_ini        set_minus1 + ini_PF  PhaseField.cu:51-57, 91-107
 *   oracle_dense_move_frame move_frame + copy_frame  PhaseField.cu:316-363
 * The sums of the full-PF rotation are switched like the APT sites (g_dcfg); the
 * sites of the same shape as the APT kernel's (a_s, magnitude, quartic,
 * diffusion, repulsion, update) have switches of their own (g_dsh), pinned
 * separately against dumps of the full-PF kernels. */
enum {
  D_X_IN = 0, /* (ca*cb)*ux + sa*uy                  : 0/1/2 */
  D_X_OUT,    /* s + (ca*sb)*uz                      : 0/1 */
  D_Y_IN,     /* ((-sa)*cb)*ux + ca*uy               : 0/1/2 */
  D_Y_OUT,    /* s - (sa*sb)*uz                      : 0/1 */
  D_Z_OUT,    /* ((-sb)*ux + 0) + cb*uz              : 0/1 */
  D_TD,       /* z - (R*1e6)*t in double             : 0/1 */
  D_NSITES
};
static int g_dcfg[D_NSITES] = {1, 1, 1, 1, 1, 1};
/* the sites the full-PF kernel shares with the APT one, switched separately
 * (nvcc fuses some of them differently in the two kernels) */
static int g_dsh[S_NSITES] = {1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1};

/* D_NSITES full-PF sites followed by S_NSITES shared ones */
int oracle_dense_num_sites(void) { return D_NSITES + S_NSITES; }
void oracle_dense_set_contraction(const int32_t* cfg, int n) {
  for (int i = 0; i < n && i < D_NSITES + S_NSITES; ++i) {
    if (i < D_NSITES) g_dcfg[i] = cfg[i];
    else g_dsh[i - D_NSITES] = cfg[i];
  }
}

static float kine_ani_full_f32(float ux, float uy, float uz, float cosa, float sina, float cosb,
                               float sinb, float kd, float eps) {
  float a_s = g_dsh[S_AS] ? fmaf(3.0f, kd, 1.0f) : 1.0f + 3.0f * kd;
  float epsilon = -4.0f * kd / a_s;
  float s = sop(cosa * cosb, ux, sina, uy, g_dcfg[D_X_IN]);
  float rx = g_dcfg[D_X_OUT] ? fmaf(cosa * sinb, uz, s) : s + (cosa * sinb) * uz;
  s = sop(-sina * cosb, ux, cosa, uy, g_dcfg[D_Y_IN]);
  float ry = g_dcfg[D_Y_OUT] ? fmaf(-(sina * sinb), uz, s) : s - (sina * sinb) * uz;
  s = (-sinb * ux) + 0.0f;
  float rz = g_dcfg[D_Z_OUT] ? fmaf(cosb, uz, s) : s + cosb * uz;
  float ux2 = rx * rx, uy2 = ry * ry, uz2 = rz * rz;
  float mag = sop(rx, rx, ry, ry, g_dsh[S_MAG_IN]);
  mag = g_dsh[S_MAG_OUT] ? fmaf(rz, rz, mag) : mag + uz2;
  float mag2 = mag * mag;
  if (mag > eps) {
    float q = sop(ux2, ux2, uy2, uy2, g_dsh[S_Q_IN]);
    q = g_dsh[S_Q_OUT] ? fmaf(uz2, uz2, q) : q + uz2 * uz2;
    return a_s * (1.0f + epsilon * q / mag2);
  }
  return 1.0f;
}

void oracle_dense_set_bc(const cupf_apt_params* p, float* ph) {
  const int fnx = p->fnx, fny = p->fny, fnz = p->fnz, np = p->num_theta;
  const int64_t len = (int64_t)fnx * fny * fnz;
  for (int g = 0; g < np; ++g)
    for (int k = 0; k < fnz; ++k)
      for (int j = 0; j < fny; ++j)
        for (int i = 0; i < fnx; ++i) {
          int hk = (k == 0 || k == fnz - 1), hj = (j == 0 || j == fny - 1),
              hi = (i == 0 || i == fnx - 1);
          if (!(hk || hj || hi)) continue;
          int si = bc_map(i, fnx, 0), sj = bc_map(j, fny, 0), sk = bc_map(k, fnz, 0);
          ph[g * len + i + (int64_t)j * fnx + (int64_t)k * fnx * fny] =
              ph[g * len + si + (int64_t)sj * fnx + (int64_t)sk * fnx * fny];
        }
}

/* rhs_psi of every grain at every interior cell from a buffer whose halo is
 * filled; t in seconds, R = Rmax in m/s. */
void oracle_dense_rhs_f32(const cupf_apt_params* p, const float* z, const float* sint,
                          const float* cost, float R, float t, const float* ph, float* ph_new) {
  const int fnx = p->fnx, fny = p->fny, fnz = p->fnz, np = p->num_theta;
  const int64_t len = (int64_t)fnx * fny * fnz, sx = 1, sy = fnx, sz = (int64_t)fnx * fny;
  const double Rm = (double)R * 1e6;
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 1; k < fnz - 1; ++k)
    for (int j = 1; j < fny - 1; ++j) {
      /* Tinterp = cP.G*(z[k] - cP.R*1e6*t - 2) in double (PhaseField.cu:277) */
      double r = g_dcfg[D_TD] ? fma(-Rm, (double)t, (double)z[k]) : (double)z[k] - Rm * (double)t;
      float Tinterp = (float)((double)p->G * (r - 2.0));
      float Up = Tinterp / p->L_cp;
      for (int i = 1; i < fnx - 1; ++i) {
        int64_t C0 = i + (int64_t)j * sy + (int64_t)k * sz;
        for (int g = 0; g < np; ++g) {
          int64_t C = C0 + g * len;
          float phC = ph[C], phR = ph[C + sx], phL = ph[C - sx], phT = ph[C + sy],
                phB = ph[C - sy], phU = ph[C + sz], phD = ph[C - sz];
          float phxn = (phR - phL) * 0.5f, phyn = (phT - phB) * 0.5f, phzn = (phU - phD) * 0.5f;
          float cosa, sina, cosb, sinb;
          if ((double)phC > LS) {
            sina = sint[g + 1];
            cosa = cost[g + 1];
            sinb = sint[g + 1 + np];
            cosb = cost[g + 1 + np];
          } else {
            sina = 0.0f;
            cosa = 1.0f;
            sinb = 0.0f;
            cosb = 1.0f;
          }
          float A2 = kine_ani_full_f32(phxn, phyn, phzn, cosa, sina, cosb, sinb, p->kin_delta,
                                       p->eps);
          float sum = phR + phL + phT + phB + phU + phD;
          float diff = g_dsh[S_DIFF] ? fmaf(-6.0f, phC, sum) : sum - 6.0f * phC;
          float repul = 0.0f;
          for (int b = 0; b < np; ++b) {
            if (b == g) continue;
            float q = ph[C0 + b * len] + 1.0f;
            repul = g_dsh[S_REP] ? fmaf(0.25f * q, q, repul) : repul + 0.25f * q * q;
          }
          float w = g_dsh[S_W] ? fmaf(-phC, phC, 1.0f) : 1.0f - phC * phC;
          float dh = diff * p->hi;
          float E1 = sop(dh, p->hi, w, phC, g_dsh[S_E1]);
          float m6 = 6.0f * (phC + 1.0f);
          float inner;
          if (g_dsh[S_INNER] == 1) inner = fmaf(w, w, -(m6 * repul));
          else if (g_dsh[S_INNER] == 2) inner = fmaf(-m6, repul, w * w);
          else inner = w * w - m6 * repul;
          float lu = p->lamd * Up;
          float rhs = g_dsh[S_RHS] ? fmaf(-lu, inner, E1) : E1 - lu * inner;
          float dphi = rhs / A2;
          ph_new[C] = g_dsh[S_NEW] ? fmaf(p->dt, dphi, phC) : phC + p->dt * dphi;
        }
      }
    }
}

/* argmax starts from argmax[C] and moves only to a strictly larger grain; phi /
 * alpha written only where the max is above LS */
void oracle_dense_collect(const cupf_apt_params* p, const float* ph, float* phi, int32_t* alpha,
                          int32_t* argmax) {
  const int np = p->num_theta;
  const int64_t len = (int64_t)p->fnx * p->fny * p->fnz;
  for (int64_t C = 0; C < len; ++C) {
    for (int g = 0; g < np; ++g)
      if (ph[C + g * len] > ph[C + (int64_t)argmax[C] * len]) argmax[C] = g;
    float v = ph[C + (int64_t)argmax[C] * len];
    if ((double)v > LS) {
      phi[C] = v;
      alpha[C] = argmax[C] + 1;
    }
  }
}

void oracle_dense_ini(const cupf_apt_params* p, float* ph, const float* phi, const int32_t* alpha) {
  const int np = p->num_theta;
  const int64_t len = (int64_t)p->fnx * p->fny * p->fnz;
  for (int64_t C = 0; C < (int64_t)np * len; ++C) ph[C] = -1.0f;
  for (int64_t C = 0; C < len; ++C)
    if ((double)phi[C] > LS && alpha[C] >= 1 && alpha[C] <= np) ph[C + (alpha[C] - 1) * len] = phi[C];
}

/* move_frame + copy_frame: interior k <- k+1, the top interior layer 2*phi[top] -
 * phi[top-1], archive and lost area as oracle_move_frame. */
void oracle_dense_move_frame(const cupf_apt_params* p, float* ph, float* z, const int32_t* alpha,
                             int32_t* alpha_full, int32_t* loss_area, int move_count) {
  const int fnx = p->fnx, fny = p->fny, fnz = p->fnz, np = p->num_theta;
  const int64_t plane = (int64_t)fnx * fny, len = plane * fnz;
  for (int64_t c = 0; c < plane; ++c) {
    int32_t a = alpha[plane + c];
    alpha_full[(int64_t)move_count * plane + plane + c] = a;
    if (a >= 1 && a <= p->num_theta) loss_area[a - 1] += 1;
  }
  float* top = (float*)malloc(sizeof(float) * (size_t)plane);
  for (int g = 0; g < np; ++g) {
    for (int64_t c = 0; c < plane; ++c) {
      int64_t C = g * len + (fnz - 2) * plane + c;
      top[c] = 2.0f * ph[C] - ph[C - plane];
    }
    for (int k = 1; k < fnz - 1; ++k)
      for (int j = 1; j < fny - 1; ++j)
        for (int i = 1; i < fnx - 1; ++i) {
          int64_t C = g * len + k * plane + (int64_t)j * fnx + i;
          ph[C] = (k < fnz - 2) ? ph[C + plane] : top[(int64_t)j * fnx + i];
        }
  }
  free(top);
  float ztop = 2.0f * z[fnz - 2] - z[fnz - 3];
  for (int k = 1; k < fnz - 2; ++k) z[k] = z[k + 1];
  z[fnz - 2] = ztop;
}
