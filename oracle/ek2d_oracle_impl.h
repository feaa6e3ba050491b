/* ek2d_oracle_impl.h — body of the 2D Echebarria–Karma oracle, included by
 * ek2d_oracle.c once per arithmetic type.  TEST INFRASTRUCTURE ONLY.
 *
 * Before inclusion: REAL (double or float), SUF (function-name suffix),
 * TANH / SQRT (math of REAL), REF_TIME (1: time, y and the integrated pulling
 * distance in float as the reference's host code keeps them; 0: in double).
 *
 * Each function restates the reference kernel named beside it
 * (cuPF 2DdendriteMPI/line_model/PF.cu), in the reference's per-cell form:
 * every edge flux is evaluated from the cell's own side, with the reference's
 * operand order. */

#define CAT_(a, b) a##b
#define CAT(a, b) CAT_(a, b)
#define FN(name) CAT(name, SUF)

typedef struct {
  REAL k, hi, Dl, eps, sqrt2, lamd, dt, cosa, sina, a_s, epsilon, a_12, U0, noise_amp;
} FN(ek_consts_);

static FN(ek_consts_) FN(ek_consts)(const cupf_ek2d_params* p) {
  FN(ek_consts_) c;
  c.k = p->k;
  c.hi = p->hi;
  c.Dl = p->Dl_tilde;
  c.eps = p->eps;
  c.sqrt2 = p->sqrt2;
  c.lamd = p->lamd;
  c.dt = p->dt;
  c.cosa = p->cosa;
  c.sina = p->sina;
  c.a_s = p->a_s;
  c.epsilon = p->epsilon;
  c.a_12 = p->a_12;
  c.U0 = p->U0;
  c.noise_amp = (REAL)(p->dt_sqrt * p->hi * p->eta);
  return c;
}

/* atheta (PF.cu:119-131) */
static REAL FN(atheta)(const FN(ek_consts_) * c, REAL ux, REAL uz) {
  REAL ux2 = c->cosa * ux + c->sina * uz;
  ux2 = ux2 * ux2;
  REAL uz2 = -c->sina * ux + c->cosa * uz;
  uz2 = uz2 * uz2;
  const REAL m = ux2 + uz2, m2 = m * m;
  if (m > c->eps) return c->a_s * ((REAL)1 + c->epsilon * (ux2 * ux2 + uz2 * uz2) / m2);
  return (REAL)1;
}

/* aptheta (PF.cu:135-146) */
static REAL FN(aptheta)(const FN(ek_consts_) * c, REAL ux, REAL uz) {
  const REAL uxr = c->cosa * ux + c->sina * uz, ux2 = uxr * uxr;
  const REAL uzr = -c->sina * ux + c->cosa * uz, uz2 = uzr * uzr;
  const REAL m = ux2 + uz2, m2 = m * m;
  if (m > c->eps) return -c->a_12 * uxr * uzr * (ux2 - uz2) / m2;
  return (REAL)0;
}

/* set_BC (PF.cu:35-73): rows 0 / fny-1 mirror rows 2 / fny-3, then columns
 * 0 / fnx-1 copy columns fnx-2 / 1 (so corners take both). */
void FN(ek2d_oracle_bc)(REAL* f, int fnx, int fny) {
  for (int i = 0; i < fnx; ++i) {
    f[i] = f[i + 2 * (int64_t)fnx];
    f[i + (int64_t)(fny - 1) * fnx] = f[i + (int64_t)(fny - 3) * fnx];
  }
  for (int j = 0; j < fny; ++j) {
    f[(int64_t)j * fnx] = f[(int64_t)j * fnx + fnx - 2];
    f[(int64_t)j * fnx + fnx - 1] = f[(int64_t)j * fnx + 1];
  }
}

/* One step over the interior: merge_PF (PF.cu:379-610; U then psi) when
 * prestep == 0, rhs_psi (PF.cu:150-280; psi only, U unchanged) when 1.
 * Inputs must carry their boundary values.  Up of row j = (y[j]/W0 - intR)/lT.
 * Noise (eta != 0) draws Philox4x32-10 keyed (seed, 0x5EED) at counter
 * (i, j, step, 'NOIS') in place of the reference's curand state. */
void FN(ek2d_oracle_step)(const cupf_ek2d_params* p, const REAL* ps, const REAL* ph, const REAL* U,
                          const REAL* D, REAL* ps_n, REAL* ph_n, REAL* U_n, REAL* D_n, const REAL* y,
                          REAL intR, REAL lT, int prestep, uint32_t step) {
  const FN(ek_consts_) c0 = FN(ek_consts)(p);
  const FN(ek_consts_)* c = &c0;
  const int fnx = p->nx + 2, fny = p->ny + 3;
#pragma omp parallel for schedule(static)
  for (int j = 1; j < fny - 1; ++j) {
    const REAL Up = (y[j] / (REAL)p->W0 - intR) / lT;
    for (int i = 1; i < fnx - 1; ++i) {
      const int64_t C = (int64_t)j * fnx + i, R = C + 1, L = C - 1, T = C + fnx, B = C - fnx;
      const REAL psipjp = (ps[C] + ps[R] + ps[T] + ps[T + 1]) * (REAL)0.25;
      const REAL psipjm = (ps[C] + ps[R] + ps[B] + ps[B + 1]) * (REAL)0.25;
      const REAL psimjp = (ps[C] + ps[L] + ps[T - 1] + ps[T]) * (REAL)0.25;
      const REAL psimjm = (ps[C] + ps[L] + ps[B - 1] + ps[B]) * (REAL)0.25;
      const REAL phipjp = (ph[C] + ph[R] + ph[T] + ph[T + 1]) * (REAL)0.25;
      const REAL phipjm = (ph[C] + ph[R] + ph[B] + ph[B + 1]) * (REAL)0.25;
      const REAL phimjp = (ph[C] + ph[L] + ph[T - 1] + ph[T]) * (REAL)0.25;
      const REAL phimjm = (ph[C] + ph[L] + ph[B - 1] + ph[B]) * (REAL)0.25;
      REAL A, Ap, phx, phz, psx, psz;
      /* right edge */
      phx = ph[R] - ph[C];
      phz = phipjp - phipjm;
      psx = ps[R] - ps[C];
      psz = psipjp - psipjm;
      A = FN(atheta)(c, phx, phz);
      Ap = FN(aptheta)(c, phx, phz);
      const REAL JR = A * (A * psx - Ap * psz);
      REAL n2 = phx * phx + phz * phz;
      const REAL nR = (n2 > c->eps) ? phx / SQRT(n2) : (REAL)0;
      /* left edge */
      phx = ph[C] - ph[L];
      phz = phimjp - phimjm;
      psx = ps[C] - ps[L];
      psz = psimjp - psimjm;
      A = FN(atheta)(c, phx, phz);
      Ap = FN(aptheta)(c, phx, phz);
      const REAL JL = A * (A * psx - Ap * psz);
      n2 = phx * phx + phz * phz;
      const REAL nL = (n2 > c->eps) ? phx / SQRT(n2) : (REAL)0;
      /* top edge */
      phx = phipjp - phimjp;
      phz = ph[T] - ph[C];
      psx = psipjp - psimjp;
      psz = ps[T] - ps[C];
      A = FN(atheta)(c, phx, phz);
      Ap = FN(aptheta)(c, phx, phz);
      const REAL JT = A * (A * psz + Ap * psx);
      n2 = phx * phx + phz * phz;
      const REAL nT = (n2 > c->eps) ? phz / SQRT(n2) : (REAL)0;
      /* bottom edge */
      phx = phipjm - phimjm;
      phz = ph[C] - ph[B];
      psx = psipjm - psimjm;
      psz = ps[C] - ps[B];
      A = FN(atheta)(c, phx, phz);
      Ap = FN(aptheta)(c, phx, phz);
      const REAL JB = A * (A * psz + Ap * psx);
      n2 = phx * phx + phz * phz;
      const REAL nB = (n2 > c->eps) ? phz / SQRT(n2) : (REAL)0;

      REAL Unew = U[C];
      if (!prestep) {
        /* U equation (PF.cu:460-556) */
        const REAL omk = (REAL)1 - c->k;
#define JAT(X) ((REAL)0.5 * ((REAL)1 + omk * U[X]) * ((REAL)1 - ph[X] * ph[X]) * D[X])
        const REAL jat = JAT(C);
        const REAL hd = c->hi * c->Dl * (REAL)0.5;
        const REAL UR = hd * ((REAL)2 - ph[C] - ph[R]) * (U[R] - U[C]) + (REAL)0.5 * (jat + JAT(R)) * nR;
        const REAL UL = hd * ((REAL)2 - ph[C] - ph[L]) * (U[C] - U[L]) + (REAL)0.5 * (jat + JAT(L)) * nL;
        const REAL UT = hd * ((REAL)2 - ph[C] - ph[T]) * (U[T] - U[C]) + (REAL)0.5 * (jat + JAT(T)) * nT;
        const REAL UB = hd * ((REAL)2 - ph[C] - ph[B]) * (U[C] - U[B]) + (REAL)0.5 * (jat + JAT(B)) * nB;
#undef JAT
        const REAL rhsU = ((UR - UL) + (UT - UB)) * c->hi + c->sqrt2 * jat;
        const REAL tauU = ((REAL)1 + c->k) - ((REAL)1 - c->k) * ph[C];
        Unew = U[C] + c->dt * (rhsU / tauU);
      }
      /* psi equation (PF.cu:563-598) */
      const REAL phxn = (ph[R] - ph[L]) * (REAL)0.5, phzn = (ph[T] - ph[B]) * (REAL)0.5;
      const REAL psxn = (ps[R] - ps[L]) * (REAL)0.5, pszn = (ps[T] - ps[B]) * (REAL)0.5;
      REAL A2 = FN(atheta)(c, phxn, phzn);
      A2 = A2 * A2;
      const REAL gradps2 = psxn * psxn + pszn * pszn;
      const REAL extra = -c->sqrt2 * A2 * ph[C] * gradps2;
      const REAL rhs = ((JR - JL) + (JT - JB) + extra) * c->hi * c->hi + c->sqrt2 * ph[C] -
                       c->lamd * ((REAL)1 - ph[C] * ph[C]) * c->sqrt2 * (Unew + Up);
      const REAL tp = (REAL)1 - ((REAL)1 - c->k) * Up;
      const REAL tau = (tp >= c->k) ? tp * A2 : c->k * A2;
      const REAL dps = rhs / tau;
      REAL noise = (REAL)0;
      if (c->noise_amp != (REAL)0 && (double)ph[C] > -0.995 && (double)ph[C] < 0.995) {
        uint32_t r[4];
        oracle_philox((uint32_t)i, (uint32_t)j, step, 0x4E4F4953u, (uint32_t)p->seed_val, 0x5EEDu, r);
        noise = c->noise_amp * ((REAL)ek2d_uniform01(r[0]) - (REAL)0.5);
      }
      ps_n[C] = ps[C] + c->dt * dps + noise;
      ph_n[C] = TANH(ps_n[C] / c->sqrt2);
      U_n[C] = Unew;
      D_n[C] = dps;
    }
  }
}

/* Row sums of phi over all fnx columns (ave_x, PF.cu:612-620), in double. */
void FN(ek2d_oracle_row_sums)(const REAL* ph, int fnx, int fny, double* out) {
  for (int j = 0; j < fny; ++j) {
    double s = 0.0;
    for (int i = 0; i < fnx; ++i) s += (double)ph[(int64_t)j * fnx + i];
    out[j] = s;
  }
}

/* One-row frame move (move_frame + copy_frame, PF.cu:625-668) of psi, phi, U
 * and the row coordinates: row j takes row j+1 for j < fny-2; row fny-2 is
 * extrapolated linearly (U there is U0).  dpsi is not moved. */
void FN(ek2d_oracle_shift)(const cupf_ek2d_params* p, REAL* ps, REAL* ph, REAL* U, REAL* y) {
  const int fnx = p->nx + 2, fny = p->ny + 3;
  for (int i = 1; i < fnx - 1; ++i) {
    const REAL pa = ps[(int64_t)(fny - 2) * fnx + i], pb = ps[(int64_t)(fny - 3) * fnx + i];
    const REAL qa = ph[(int64_t)(fny - 2) * fnx + i], qb = ph[(int64_t)(fny - 3) * fnx + i];
    for (int j = 1; j < fny - 2; ++j) {
      ps[(int64_t)j * fnx + i] = ps[(int64_t)(j + 1) * fnx + i];
      ph[(int64_t)j * fnx + i] = ph[(int64_t)(j + 1) * fnx + i];
      U[(int64_t)j * fnx + i] = U[(int64_t)(j + 1) * fnx + i];
    }
    ps[(int64_t)(fny - 2) * fnx + i] = (REAL)2 * pa - pb;
    ph[(int64_t)(fny - 2) * fnx + i] = (REAL)2 * qa - qb;
    U[(int64_t)(fny - 2) * fnx + i] = (REAL)p->U0;
  }
  const REAL ya = y[fny - 2], yb = y[fny - 3];
  for (int j = 1; j < fny - 2; ++j) y[j] = y[j + 1];
  y[fny - 2] = (REAL)2 * ya - yb;
}

/* R and G of the tables at t, linear within the interval that holds t (varGR,
 * PF.cu:685-697); the last interval past the end. */
static void FN(ek2d_table)(int Nt, const float* t_mac, const float* Gt, const float* Rt, REAL t,
                           REAL* R, REAL* G) {
  const REAL Dt = (REAL)t_mac[1] - (REAL)t_mac[0];
  const REAL x = (t - (REAL)t_mac[0]) / Dt;
  int kt = (int)x;
  REAL d = x - (REAL)kt;
  if (kt > Nt - 2) {
    d += (REAL)(kt - (Nt - 2));
    kt = Nt - 2;
  }
  *R = ((REAL)1 - d) * (REAL)Rt[kt] + d * (REAL)Rt[kt + 1];
  *G = ((REAL)1 - d) * (REAL)Gt[kt] + d * (REAL)Gt[kt + 1];
}

/* The time loop of setup() (PF.cu:742-820): optional psi-only pre-step, then
 * nsteps fused steps, each after varGR, with the tip search and frame move
 * after every multiple of tipp steps.  State arrays (reference layout) are
 * updated in place; y holds the fny row coordinates; st carries the step count,
 * frame shifts, tip row, time, pulling distance and thermal length across
 * calls (zero it before the first). */
int FN(ek2d_oracle_run)(const cupf_ek2d_params* p, int Nt, const float* t_mac, const float* Gt,
                        const float* Rt, REAL* ps, REAL* ph, REAL* U, REAL* D, REAL* y, int prestep,
                        int nsteps, cupf_ek2d_info* st) {
  const int fnx = p->nx + 2, fny = p->ny + 3;
  const size_t n = (size_t)fnx * fny;
  REAL* b = (REAL*)malloc(4 * n * sizeof(REAL));
  double* rows = (double*)malloc((size_t)fny * sizeof(double));
  if (!b || !rows) {
    free(b);
    free(rows);
    return -1;
  }
  REAL *bps = b, *bph = b + n, *bU = b + 2 * n, *bD = b + 3 * n;
  const REAL W0 = p->W0, tau0 = p->tau0, dt = p->dt;
  REAL intR = (REAL)st->intR;
  if (st->tip_thres == 0) st->tip_thres = (int)((1.0 - (double)p->blank) * fny);
  if (st->cur_tip == 0) st->cur_tip = 1;
  if (prestep) {
    const REAL lT = ((REAL)p->c_infm * ((REAL)1 / (REAL)p->k - (REAL)1) / (REAL)Gt[0]) / W0;
    FN(ek2d_oracle_bc)(ps, fnx, fny);
    FN(ek2d_oracle_bc)(ph, fnx, fny);
    FN(ek2d_oracle_bc)(U, fnx, fny);
    FN(ek2d_oracle_bc)(D, fnx, fny);
    FN(ek2d_oracle_step)(p, ps, ph, U, D, bps, bph, bU, bD, y, (REAL)0, lT, 1, 0u);
    memcpy(ps, bps, n * sizeof(REAL));
    memcpy(ph, bph, n * sizeof(REAL));
    memcpy(D, bD, n * sizeof(REAL));
    intR = (REAL)0;
    st->lT_tilde = (double)lT;
  }
  for (int s = 0; s < nsteps; ++s) {
    const int64_t m = st->steps + 1;
#if REF_TIME
    const REAL t = (REAL)m * dt * tau0;
#else
    const REAL t = (REAL)m * (REAL)dt * (REAL)tau0;
#endif
    REAL R, G;
    FN(ek2d_table)(Nt, t_mac, Gt, Rt, t, &R, &G);
    intR += (R * tau0 / W0) * dt;
    const REAL lT = ((REAL)p->c_infm * ((REAL)1 / (REAL)p->k - (REAL)1) / G) / W0;
    FN(ek2d_oracle_bc)(ps, fnx, fny);
    FN(ek2d_oracle_bc)(ph, fnx, fny);
    FN(ek2d_oracle_bc)(U, fnx, fny);
    FN(ek2d_oracle_bc)(D, fnx, fny);
    FN(ek2d_oracle_step)(p, ps, ph, U, D, bps, bph, bU, bD, y, intR, lT, 0, (uint32_t)m);
    memcpy(ps, bps, n * sizeof(REAL));
    memcpy(ph, bph, n * sizeof(REAL));
    memcpy(U, bU, n * sizeof(REAL));
    memcpy(D, bD, n * sizeof(REAL));
    st->steps = m;
    st->t = (double)t;
    st->lT_tilde = (double)lT;
    if (m % p->tipp == 0) {
      FN(ek2d_oracle_bc)(ph, fnx, fny);
      FN(ek2d_oracle_row_sums)(ph, fnx, fny, rows);
      while (rows[st->cur_tip] / fnx > (double)p->ls && st->cur_tip < fny - 1) st->cur_tip += 1;
      while (st->cur_tip >= st->tip_thres) {
        FN(ek2d_oracle_shift)(p, ps, ph, U, y);
        st->shifts += 1;
        st->cur_tip -= 1;
      }
    }
  }
  FN(ek2d_oracle_bc)(ps, fnx, fny);
  FN(ek2d_oracle_bc)(ph, fnx, fny);
  FN(ek2d_oracle_bc)(U, fnx, fny);
  FN(ek2d_oracle_bc)(D, fnx, fny);
  st->intR = (double)intR;
  free(b);
  free(rows);
  return 0;
}

#undef FN
#undef CAT
#undef CAT_
