/*
 * cupf_ek2d.h — C ABI of the B200 2D Echebarria–Karma directional-solidification
 * step (psi/U "line model" with a frozen thermal gradient).
 *
 * The reference (cuPF, 2DdendriteMPI/line_model) runs this model from
 * main.cpp + PF.cu: main reads `input_file` and the macro tables of a folder
 * (t.txt, Gt.txt, Rt.txt, y.txt, psi.txt, U.txt), builds the initial psi/U from
 * the 1-D profiles, and setup() runs the time loop: set_BC, the host update
 * varGR of the integrated pulling distance and thermal length, and the fused
 * kernel merge_PF (U then psi) twice per iteration, with a tip search and a
 * moving frame every TIPP steps.  Each entry point below replaces one part of
 * that code; the citation on each names it (paths relative to the cuPF
 * repository).
 *
 * Conventions are those of cupf.h (status codes, cupf_last_error, host
 * pointers).  "Reference layout" is the reference's 2D array:
 *     index = i + j*fnx,  fnx = nx+2, fny = ny+3        (main.cpp:222-223,232)
 * with one halo column on each side (x periodic) and one halo row at the bottom
 * and top (y mirrored about rows 1 and fny-2).
 *
 * State kept on the device: the phase field, U and dpsi (the last dpsi/dt, read
 * by the anti-trapping current of the next U update).  FP32 (the reference's
 * precision) and FP64 (a device transcription in double, the reference for
 * split-precision error at sizes the CPU oracle cannot run) store psi and
 * recompute phi = tanh(psi/sqrt2) wherever it is read, as the reference's
 * merge_PF stores it right after computing psi (PF.cu:596).  FP16 and BF16
 * (split precision, all arithmetic FP32) hold psi to |psi| <= 50 W0 (a signed
 * distance, it would otherwise reach thousands of W0, beyond what 16 bits
 * resolve) and store it as psi (FP16) or as phi's distance to the nearest bulk
 * value (BF16), U as its offset from U0, and dpsi; the phase field and U are
 * stored with stochastic rounding.  Time, the integrated pulling distance, the frame's y
 * coordinates and the row sums of the tip search are FP64 for every storage.
 */
#ifndef CUPF_EK2D_H_
#define CUPF_EK2D_H_

#include <stdint.h>

#include "cupf.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Extra storage precision of this model (beside CUPF_PREC_FP32/BF16/FP16). */
#define CUPF_PREC_FP64 3

/* Parameters.  Names and meanings follow the reference's GlobalConstants
 * (line_model/include_struct.h:1-43) as filled by main.cpp:82-205; the derived
 * fields are computed by cupf_ek2d_derive exactly as main.cpp:158-185 does. */
typedef struct cupf_ek2d_params {
  int32_t nx, ny;       /* interior size: fnx = nx+2 columns, fny = ny+3 rows */
  int32_t Mt;           /* time steps of the run (even), from the last t_mac */
  int32_t seed_val;     /* noise seed (Philox key) */
  int32_t tipp;         /* steps between tip searches (PF.cu:11, TIPP = 100) */
  int32_t noi_period;   /* read from the input file; unused by the step */
  int32_t reserved_i[2];
  /* input file (main.cpp:104-137) */
  float G, R, delta, k, c_infm, Dl, d0, W0, c_infty, eps, alpha0, dx, asp_ratio, lxd, eta,
      U0, cfl;
  /* derived (main.cpp:158-185) */
  float lT, lamd, tau0, R_tilde, Dl_tilde, lT_tilde, dt, lyd, hi, cosa, sina, sqrt2, a_s,
      epsilon, a_12, dt_sqrt;
  float blank;          /* fraction of rows kept ahead of the tip (PF.cu:12, BLANK) */
  float ls;             /* solid threshold of the tip search (PF.cu:10, LS = -0.995) */
  double y0;            /* y of row 1 in um: y_mac[0] (main.cpp:244-246) */
  double reserved_d[3];
} cupf_ek2d_params;

/* Fill the derived fields of p (lT .. dt_sqrt, nx, ny, Mt, blank, ls, tipp)
 * from the input-file fields and the last macro time t_last (s), as
 * main.cpp:158-185 (nx = (int)(lxd/(dx*W0)), ny = (int)(asp_ratio*nx),
 * Mt = even part of (int)(t_last/tau0/dt)). */
cupf_status cupf_ek2d_derive(cupf_ek2d_params* p, float t_last);

/* Parse an input file in the reference's `key = value` form (main.cpp:37-52,
 * 95-151: every line is scanned for each key; Ny, Nt and ztip0 are returned
 * separately).  Keys that are absent leave their fields unchanged. */
cupf_status cupf_ek2d_parse_input(const char* path, cupf_ek2d_params* p, int32_t* mac_Ny,
                                  int32_t* mac_Nt, float* ztip0);

typedef struct cupf_ek2d_handle cupf_ek2d_handle;

/* Allocate a simulation on `device` with the given storage precision
 * (CUPF_PREC_FP32, _BF16, _FP16 or CUPF_PREC_FP64).  Replaces the cudaMalloc /
 * cudaMemcpyToSymbol part of setup() (PF.cu:706-741). */
cupf_status cupf_ek2d_create(const cupf_ek2d_params* p, int32_t precision, int32_t device,
                             cupf_ek2d_handle** out);
cupf_status cupf_ek2d_destroy(cupf_ek2d_handle* h);

/* Time tables of the pulling speed R (um/s) and gradient G (K/um) on a uniform
 * time grid t_mac (s), Nt >= 2 entries (main.cpp:191-193; read by varGR,
 * PF.cu:685-697).  Times past the last entry use the last interval. */
cupf_status cupf_ek2d_set_thermal(cupf_ek2d_handle* h, int32_t Nt, const float* t_mac,
                                  const float* Gt, const float* Rt);

/* Load psi and U (reference layout, fnx*fny floats each; dpsi may be NULL for
 * zeros).  Halo cells are refilled from the interior (set_BC, PF.cu:35-73).
 * Resets the step count, time, pulling distance, tip row (1) and frame shifts. */
cupf_status cupf_ek2d_set_state(cupf_ek2d_handle* h, const float* psi, const float* U,
                                const float* dpsi);

/* The psi-only update setup() makes before its loop (rhs_psi at PF.cu:745,
 * with U left as it is, pulling distance 0 and the first table gradient). */
cupf_status cupf_ek2d_prestep(cupf_ek2d_handle* h);

/* nsteps fused U-then-psi steps (merge_PF, PF.cu:379-610, with varGR before
 * each, PF.cu:794,805).  After every step whose count is a multiple of tipp the
 * tip search and moving frame run (tip_mvf, move_frame, copy_frame;
 * PF.cu:612-683, 811-818). */
cupf_status cupf_ek2d_step(cupf_ek2d_handle* h, int32_t nsteps);

/* Copy the state out (reference layout, halos included; any pointer may be
 * NULL).  phi = tanh(psi/sqrt2). */
cupf_status cupf_ek2d_get_state(cupf_ek2d_handle* h, float* psi, float* phi, float* U,
                                float* dpsi);

/* The same in double (for the FP64 storage; other storages are widened). */
cupf_status cupf_ek2d_get_state_f64(cupf_ek2d_handle* h, double* psi, double* phi, double* U,
                                    double* dpsi);

/* y coordinate of every row (fny doubles, um), moved with the frame. */
cupf_status cupf_ek2d_get_y(cupf_ek2d_handle* h, double* y);

typedef struct cupf_ek2d_info {
  int64_t steps;        /* merge steps done since set_state */
  int64_t shifts;       /* rows the frame has moved */
  int32_t cur_tip;      /* tip row of the last search (PF.cu:750, 671) */
  int32_t tip_thres;    /* (int)((1-blank)*fny) */
  double t;             /* physical time of the last step, s */
  double intR;          /* integrated pulling distance / W0 */
  double lT_tilde;      /* thermal length / W0 of the last step */
} cupf_ek2d_info;
cupf_status cupf_ek2d_info_get(cupf_ek2d_handle* h, cupf_ek2d_info* info);

/* Mean of phi over each row, halo columns included (ave_x, PF.cu:612-620;
 * fny doubles). */
cupf_status cupf_ek2d_row_means(cupf_ek2d_handle* h, double* meanx);

/* Device time of nsteps steps (CUDA events around the launches, ms). */
cupf_status cupf_ek2d_time_steps(cupf_ek2d_handle* h, int32_t nsteps, float* ms);

/* The handle's cudaStream_t. */
cupf_status cupf_ek2d_stream(cupf_ek2d_handle* h, void** stream);

#ifdef __cplusplus
}
#endif

#endif /* CUPF_EK2D_H_ */
