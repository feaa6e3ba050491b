/*
 * cupf_dense.h — the full (non-APT) phase-field mode of the B200 library: one
 * phi field per grain (NUM_PF = number of grains), selected in the reference by
 * the driver's -a flag (3DgrainMPI/DesignSettingData.cpp:46-47, main.cpp:39-47).
 *
 * Replaces the dense solver of the reference, PhaseField::cudaSetup / evolve
 * (3DgrainMPI/PhaseField.cu:430-632) and its kernels set_minus1, collect_PF,
 * ini_PF, set_BC_3D, rhs_psi, move_frame, copy_frame, ave_x + tip_mvf
 * (PhaseField.cu:51-57, 60-88, 91-107, 111-166, 168-301, 316-346, 348-363,
 * 366-399).  Device layout as the reference's: phi[grain][z][y][x] in float.
 *
 * What the step computes is the reference's rhs_psi for every grain and cell:
 * mirror boundaries on all six faces (set_BC_3D ignores the -b digits), the
 * full-PF rotation of kine_ani (PhaseField.cu:32-50, not the APT one), the line
 * undercooling G*(z - R*1e6*t - 2) with R = Rmax in m/s (PhaseField.cu:277), and
 * the repulsion sum over every other grain.  A grain whose phi is exactly -1 at
 * all seven stencil points stays exactly -1 and adds exactly zero to every
 * repulsion sum, so the library evaluates only the grains that differ from -1
 * somewhere in a cell's stencil (per-cell lists of those grains, which each step
 * writes for the next, see cupf_dense_set_tuning) and leaves the others at -1:
 * the same floats as evaluating all of them, with traffic proportional to the
 * grains present near each cell rather than to the number of grains.
 *
 * Status codes, precision and parameter structs are those of cupf.h.  All calls
 * on one handle are ordered on the handle's CUDA stream; handles are independent.
 */
#ifndef CUPF_DENSE_H
#define CUPF_DENSE_H

#include "cupf.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct cupf_dense_handle cupf_dense_handle;

/* Allocate the two phi buffers (num_theta * fnx*fny*fnz floats each) and the
 * per-cell lists, upload coordinates and orientations.  NUM_PF is num_theta
 * (PhaseField::cudaSetup sets params.NUM_PF = params.num_theta, PhaseField.cu:440);
 * p->num_pf, the bc digits and thermalType are ignored, as the reference's dense
 * kernels ignore them.  R: the pulling speed Rmax of the forcing folder (m/s),
 * the cP.R of PhaseField.cu:277.  in->sint / in->cost have 2*num_theta+1 entries.
 * Replaces PhaseField::cudaSetup (3DgrainMPI/PhaseField.cu:430-493). */
cupf_status cupf_dense_create(const cupf_apt_params* p, const cupf_apt_inputs* in, float R,
                              int device, cupf_dense_handle** out);

/* Free everything.  Replaces ~PhaseField (PhaseField.cu:402-427). */
cupf_status cupf_dense_destroy(cupf_dense_handle* h);

/* set_minus1 on both buffers, ini_PF on both (grain alpha-1 takes phi where
 * phi > LS = -0.995), argmax phi field to -1, argmax alpha field = alpha, argmax
 * index buffer to 0 (its cudaSetup memset), boundary fill of both buffers; the
 * step counter restarts at 0.  phi, alpha: fnx*fny*fnz, reference layout.
 * Replaces PhaseField.cu:457, 464-466 (argmax buffers) and :545-553 of evolve. */
cupf_status cupf_dense_init_from_argmax(cupf_dense_handle* h, const float* phi,
                                        const int32_t* alpha);

/* The pre-loop update at t = 0 (rhs_psi with nt = t = 0 from the current buffer
 * into the other, PhaseField.cu:555-556).  Does not advance the step counter. */
cupf_status cupf_dense_prestep(cupf_dense_handle* h);

/* nsteps explicit steps; step n (1-based since init) runs at t = n*dt*tau0 in
 * float, as evolve forms (2*kt+1)*dt*tau0 and (2*kt+2)*dt*tau0.  Each step is the
 * boundary fill of the buffer read and rhs_psi into the other buffer
 * (PhaseField.cu:563-566, 600-605). */
cupf_status cupf_dense_step(cupf_dense_handle* h, int32_t nsteps);

cupf_status cupf_dense_steps_done(cupf_dense_handle* h, int64_t* steps);

/* collect_PF on the current buffer (after its boundary fill): per cell, the
 * argmax over grains starting from the previous call's argmax (a grain replaces
 * it only when strictly larger: ties keep the earlier winner); where the max is
 * above LS, phi_out[C] = max and alpha_out[C] = grain + 1, elsewhere the argmax
 * fields keep their values.  clear != 0 zeroes the alpha field first (the
 * cudaMemset of evolve's QoI branch, PhaseField.cu:573, 616).  Either output may
 * be NULL.  Replaces collect_PF + cudaMemcpy (PhaseField.cu:60-88, 574-575). */
cupf_status cupf_dense_collect(cupf_dense_handle* h, int32_t clear, float* phi_out,
                               int32_t* alpha_out);

/* Current buffer after its boundary fill (num_theta * fnx*fny*fnz floats), and
 * its replacement (the boundary is filled on the next step).  steps_done sets the
 * step counter. */
cupf_status cupf_dense_get_slots(cupf_dense_handle* h, float* ph);
cupf_status cupf_dense_set_slots(cupf_dense_handle* h, const float* ph, int64_t steps_done);

/* Moving-domain check and shift (evolve's TIPP branch, PhaseField.cu:584-601):
 * tip_mvf over all grains (per-layer mean of phi, summed in double in a fixed
 * order where the reference adds float atomics), then while *tip_front >=
 * tip_thres: collect_PF, move_frame (interior layers k <- k+1, the new top layer
 * extrapolated as 2*phi[top] - phi[top-1], z shifted and extrapolated, the
 * bottom interior alpha layer archived into alpha_full[move_count] and counted
 * into loss_area) and copy_frame; then the boundary fill.  *moved receives the
 * number of layers shifted.  Replaces tip_mvf + move_frame + copy_frame
 * (PhaseField.cu:316-346, 348-363, 366-399). */
cupf_status cupf_dense_move_domain(cupf_dense_handle* h, int32_t* tip_front, int32_t tip_thres,
                                   int32_t* move_count, int32_t* moved);

/* Archive of evicted alpha layers (fnx*fny*fnz_f ints) and per-grain lost area
 * (num_theta ints); either may be NULL.  The D2H copies of evolve
 * (PhaseField.cu:576, 621). */
cupf_status cupf_dense_get_archive(cupf_dense_handle* h, int32_t fnz_f, int32_t* alpha_full,
                                   int32_t* loss_area);
cupf_status cupf_dense_get_z(cupf_dense_handle* h, float* z);

cupf_status cupf_dense_sync(cupf_dense_handle* h, int32_t timeout_ms);

/* Device time of nsteps steps (CUDA events on the handle's stream). */
cupf_status cupf_dense_time_steps(cupf_dense_handle* h, int32_t nsteps, float* ms);

/* Capacity of the per-cell lists of grains that differ from -1 (1..16, default
 * 16).  A cell whose stencil meets a longer list is evaluated from the full phi
 * buffer instead (same result, slower); *overflow_cells, when not NULL, receives
 * how many cells took that path in the last step.  No reference counterpart
 * (the reference evaluates every grain of every cell, PhaseField.cu:168-301). */
cupf_status cupf_dense_set_tuning(cupf_dense_handle* h, int32_t list_cap);
cupf_status cupf_dense_overflow_cells(cupf_dense_handle* h, int64_t* overflow_cells);

#ifdef __cplusplus
}
#endif

#endif /* CUPF_DENSE_H */
