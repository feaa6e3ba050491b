/*
 * cupf.h — C ABI of the B200 APT (active parameter tracking) multi-grain
 * phase-field step.
 *
 * The reference (cuPF, 3DgrainMPI) drives its device step from the C++ class
 * APTPhaseField.  Every entry point below replaces one device-side method or
 * kernel-launch group of that class; the citation on each names the reference
 * code it stands in for (paths are relative to the cuPF repository).
 *
 * Conventions
 *   - Plain C: no C++ or torch types cross this boundary.  Every call returns a
 *     cupf_status; cupf_last_error() returns a message for the calling thread.
 *   - Host pointers unless a name ends in "_dev".
 *   - "Reference layout" means the reference's SoA slot layout:
 *       index = i + j*fnx + k*fnx*fny + slot*fnx*fny*fnz     (devicefunc.cu_inl:24-29)
 *     with fnx = nx+1+2 (one halo cell per side), NUM_PF slots per cell,
 *     phi as float32 and grain ids as int32 (-1 = empty slot).
 *   - A handle owns its device memory and one CUDA stream.  Calls on different
 *     handles may run from different host threads; calls on one handle must
 *     not overlap.
 */
#ifndef CUPF_H_
#define CUPF_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CUPF_ABI_VERSION 1
#define CUPF_MAX_PF 16

typedef enum cupf_status {
  CUPF_OK = 0,
  CUPF_ERR_INVALID = 1,     /* bad argument or unsupported size */
  CUPF_ERR_CUDA = 2,        /* a CUDA runtime/driver call failed */
  CUPF_ERR_OOM = 3,         /* device allocation failed */
  CUPF_ERR_UNSUPPORTED = 4, /* option not built into this library */
  CUPF_ERR_TIMEOUT = 5,     /* host-side watchdog deadline passed */
  CUPF_ERR_IO = 6,          /* file could not be read or written */
  CUPF_ERR_STATE = 7        /* call out of order (e.g. step before init) */
} cupf_status;

/* Storage precision of the phi slots.  FP32 is the reference's own storage;
 * BF16 / FP16 store phi in 16 bits and grain ids in int16 while all stencil
 * arithmetic stays FP32 (the split-precision variant). */
typedef enum cupf_precision {
  CUPF_PREC_FP32 = 0,
  CUPF_PREC_BF16 = 1,
  CUPF_PREC_FP16 = 2
} cupf_precision;

/* Parameter block read by the APT step.  Field names and meanings follow the
 * reference's GlobalConstants (params.h:10-56) as filled by
 * PhaseField::parseInputParams / cpuSetup (PhaseFieldCpu.cpp:17-374). */
typedef struct cupf_apt_params {
  int32_t fnx, fny, fnz;  /* points per axis, halo included */
  int32_t num_pf;         /* NUM_PF, active slots per cell (1..CUPF_MAX_PF) */
  int32_t num_theta;      /* NG: grain orientations in sint/cost */
  int32_t bcX, bcY, bcZ;  /* 0 = no-flux (mirror about 1 / fn-2), 1 = periodic */
  int32_t thermalType;    /* 0 none, 1 line, 2 cylinder, 3 cone, 4 paraboloid table,
                             5 analytic paraboloid melt pool (no counterpart in the
                             reference: a beam at x0 + V 1e6 t moving in +x along
                             y = lyd/2, z = z0 + lzd; pool radius r0 sqrt(1 - xi/mp_len)
                             at xi behind it, a hemisphere of radius r0 ahead;
                             T = -G dist - UC 1e6 t) */
  int32_t Nx, Ny, Nz, Nt; /* macro thermal grid (thermalType 4, nucleation) */
  float kin_delta;        /* kinetic anisotropy strength */
  float eps;              /* |grad phi|^2 threshold in kine_ani */
  float G;                /* thermal gradient, K/um */
  float z0;               /* interface height, um */
  float underCoolingRate; /* UC, K/us */
  float underCoolingRate0;
  float L_cp;
  float hi;               /* 1/dx */
  float lamd;             /* coupling constant lambda */
  float dt;               /* dimensionless time step */
  float tau0;             /* time scale, s */
  float lyd, lzd;         /* domain lengths, um */
  float r0, x0, angle, V, mp_len, order;
  float dx, W0;
  /* nucleation (used only by the nucleation entry points) */
  float undcool_mean, undcool_std, nuc_Nmax, nuc_Nmax0, nuc_rad, sqrt2;
  int32_t pts_cell;
  int32_t seed;
  int32_t haloWidth;      /* must be 1 */
  int32_t reserved[5];
} cupf_apt_params;

/* Thermal and orientation inputs (the reference's ThermalInputData,
 * ThermalInputData.h:8-24, plus the coordinate arrays of PDE, cuPDE.h:18-23).
 * Host arrays; copied to the device by cupf_apt_create. */
typedef struct cupf_apt_inputs {
  const float* x;       /* [fnx] */
  const float* y;       /* [fny] */
  const float* z;       /* [fnz] */
  const float* sint;    /* [2*num_theta+1] sinf(theta) */
  const float* cost;    /* [2*num_theta+1] cosf(theta) */
  const float* X_mac;   /* [Nx]   (thermalType 4 / nucleation; else NULL) */
  const float* Y_mac;   /* [Ny] */
  const float* Z_mac;   /* [Nz] */
  const float* t_mac;   /* [Nt] */
  const float* psi_mac; /* [Nx*Ny*Nz] */
  const float* T_3D;    /* [Nx*Ny*Nz*Nt] (nucleation only; may be NULL) */
} cupf_apt_inputs;

typedef struct cupf_apt_handle cupf_apt_handle;

/* Message describing the last failure on the calling thread ("" if none). */
const char* cupf_last_error(void);
int cupf_abi_version(void);
/* sizeof of the ABI structs as compiled into the library: which = 0 for
 * cupf_apt_params, 1 for cupf_apt_inputs (lets bindings check their mirror). */
size_t cupf_struct_size(int which);

/* Allocate device state and upload parameters and thermal inputs.
 * Replaces APTPhaseField::cudaSetup (3DgrainMPI/APTPhaseField.cu:569-637).
 * device: CUDA ordinal.  precision: storage type of the phi slots. */
cupf_status cupf_apt_create(const cupf_apt_params* p, const cupf_apt_inputs* in,
                            int device, cupf_precision precision,
                            cupf_apt_handle** out);

/* Free all device memory of the handle.  Replaces ~APTPhaseField
 * (3DgrainMPI/APTPhaseField.cu:540-566). */
cupf_status cupf_apt_destroy(cupf_apt_handle* h);

/* Initialise both slot buffers from the argmax fields phi[length], alpha[length]
 * (reference layout, length = fnx*fny*fnz): every slot = (-1, -1), then slot 0 =
 * (phi, alpha) where phi > LS (-0.995).  Resets the step counter and time.
 * Replaces set_minus1 x2 + APTini_PF x2 + setBC x2 in APTPhaseField::evolve
 * (3DgrainMPI/APTPhaseField.cu:727-728, 771-772, 817-818; PhaseField.cu:51-57). */
cupf_status cupf_apt_init_from_argmax(cupf_apt_handle* h, const float* phi,
                                      const int32_t* alpha);

/* Load a full slot state (reference layout, num_pf*length entries) into the
 * "old" buffer, i.e. the buffer the next step reads.  kt_half is the number of
 * explicit steps already taken (sets the time of the next step). */
cupf_status cupf_apt_set_slots(cupf_apt_handle* h, const float* ph,
                               const int32_t* ids, int64_t steps_done);

/* Export the current slot state in reference layout with the halo filled by the
 * boundary rule (what APTsetBC3D leaves in PFs_old / active_args_old).
 * Replaces the D2H copies of APTPhaseField::getLineQoIs
 * (3DgrainMPI/APTPhaseField.cu:666-667) preceded by setBC (:700-707). */
cupf_status cupf_apt_get_slots(cupf_apt_handle* h, float* ph, int32_t* ids);

/* Advance nsteps explicit Euler steps.  Each step reads the current buffer,
 * applies the boundary rule to its halo, and writes the other buffer; the time
 * of step n (1-based, counted from the last init) is t = n*dt*tau0 in float,
 * as the reference forms (2*kt+1)*dt*tau0 and (2*kt+2)*dt*tau0.
 * Replaces the APTsetBC3D + APTrhs_psi launches of APTPhaseField::evolve
 * (3DgrainMPI/APTPhaseField.cu:861-864, 880, 919-920; kernels :93-174, :178-354).
 * use_initial_undercooling selects the reference's liquid-start temperature
 * (Tinterp = -underCoolingRate0*1e6*t, :280-283). */
cupf_status cupf_apt_step(cupf_apt_handle* h, int32_t nsteps,
                          int32_t use_initial_undercooling);

/* Number of explicit steps taken since the last init / set_slots. */
cupf_status cupf_apt_steps_done(cupf_apt_handle* h, int64_t* steps);

/* Per-cell argmax over the slots of the current buffer: where the max phi is
 * above LS, phi_out[C] = max and alpha_out[C] = its grain id (first slot wins
 * ties); elsewhere the cell keeps the value it had in the device argmax buffer,
 * which cupf_apt_collect clears to (phi 0, alpha 0) first when clear != 0.
 * Either output may be NULL.  Replaces APTcollect_PF + cudaMemcpy
 * (3DgrainMPI/APTPhaseField.cu:55-75, 820-822, 907-909). */
cupf_status cupf_apt_collect(cupf_apt_handle* h, int32_t clear, float* phi_out,
                             int32_t* alpha_out);

/* Voxel count of every grain id 1..num_grains over the interior cells of the
 * argmax map computed by the last cupf_apt_collect (alpha > 0 only), FP64-free
 * integer reduction on the device.  counts has num_grains+1 entries; counts[0]
 * receives the number of interior cells with alpha <= 0 or alpha > num_grains.
 * The per-grain volumes of QOI::calculateQoIs (3DgrainMPI/QOI.cpp:198-231). */
cupf_status cupf_apt_grain_volumes(cupf_apt_handle* h, int32_t num_grains,
                                   int64_t* counts);

/* FP64 interface quantities of the current state, over interior cells, from
 * the per-cell maximum of phi over the slots (m):
 *   out[0] = sum (1+m)/2            solid volume in cells
 *   out[1] = sum |grad m|/2         interface area in cell faces (central differences)
 *   out[2] = out[0] / (interior cells per layer)   mean interface height in cells
 * Reduced in double in a fixed order (deterministic).  Supplies the volume and
 * interface measures the split-precision error is measured on; the reference has
 * no counterpart (its QoIs are integer voxel counts, QOI.cpp:38-231). */
cupf_status cupf_apt_qoi_sums(cupf_apt_handle* h, double* out);

/* ---------------------------------------------------------------- nucleation
 * Coarse cells of (2*pts_cell+1)^3 fine cells (cnx = (fnx-3)/(2*pts_cell+1), ...)
 * each hold a status (1 = solid or already nucleated).
 * cupf_apt_nucl_init: status from slot 0 at each coarse cell's centre, indexed
 *   without the halo offset exactly as init_nucl_status does
 *   (3DgrainMPI/APTPhaseField.cu:420-444, 733-745).
 * cupf_apt_nucleate: one add_nucl pass on the current state (:459-536, called
 *   after the odd step of each evolve iteration, :866-870): a liquid coarse cell
 *   nucleates with the reference's Gaussian probability (:446-455; undercooling
 *   from the liquid-start rate when use_initial_undercooling, else from the 4-D
 *   T_3D table), using time t = (steps done)*dt*tau0 and interval 2*dt*tau0.  The
 *   draw is Philox4x32-10 keyed on (seed, coarse cell, step) instead of curand;
 *   a nucleus is the (2*pts_cell+1)^3 tanh sphere in slot 0 with a new grain id
 *   num_theta + 1 + (draw mod id_space), id_space = 2^30 (FP32) or
 *   32767 - num_theta (16-bit storage).  *total (may be NULL) receives the
 *   number of nuclei so far.
 * cupf_apt_nucl_reset: every status to 0 (the reference's reset before the
 *   liquid-start phase, :781). */
cupf_status cupf_apt_nucl_init(cupf_apt_handle* h);
cupf_status cupf_apt_nucleate(cupf_apt_handle* h, int32_t use_initial_undercooling,
                              int32_t* total);
cupf_status cupf_apt_nucl_reset(cupf_apt_handle* h);

/* Candidate cells of the 3D junction search (QOI3D::searchJunctionsOnImage,
 * QOI.cpp:233-311), on the device, over the argmax map of the last
 * cupf_apt_collect: solid cells whose 19-point neighbourhood has no liquid cell,
 * exactly four grain ids and no id more than ten times.  Writes up to `cap`
 * cell indices (reference layout) in ascending order and the number of
 * candidates to *count (which can exceed cap: call again with more room).
 * `distinct` (may be NULL; (fnx-2)*(fny-2)*(fnz-2) bytes, interior cells in
 * (k, j, i) order) receives each cell's number of distinct neighbourhood values,
 * which the host needs to list each junction's grain ids in the reference's
 * order.  Building the records of the candidate cells only
 * (cupf_host_junctions_3d_cells) gives the records of the full host scan. */
cupf_status cupf_apt_junction_candidates(cupf_apt_handle* h, int64_t* cells, int64_t cap,
                                         int64_t* count, uint8_t* distinct);

/* Candidate cells of the line-configuration junction search
 * (QOILine::searchJunctionsOnImage, QOI.cpp:103-160), on device `device`.
 * `layers` (host memory) holds `nlayers` x-y layers of fnx*fny int32 argmax
 * values each (reference layout), one per sampled frame: the layer at that
 * frame's tip height.  Candidates are interior cells whose 3x3 in-plane
 * neighbourhood holds at least three distinct values and none more than five
 * times.  Writes up to `cap` of their indices in the stacked layers
 * (layer*fnx*fny + j*fnx + i), in ascending order, and their number to *count
 * (which can exceed cap: call again with more room).  Building the records of
 * the candidate cells only (cupf_host_line_junctions_cells) gives the records
 * of the full host scan.  Needs no handle (the APT and the full-PF drivers both
 * call it); allocates its scratch for the call, on the calling thread's
 * per-thread stream, and returns when the result is on the host. */
cupf_status cupf_line_junction_candidates(int32_t device, int32_t fnx, int32_t fny,
                                          const int32_t* layers, int32_t nlayers, int64_t* cells,
                                          int64_t cap, int64_t* count);

/* Allocation-free per-grain voxel counts (no counterpart in the reference).
 * For callers that cannot let a library allocate device memory: codes that give
 * all device memory to their own pool allocator at start-up, and services whose
 * device footprint must stay fixed after start-up.  Same result as
 * cupf_apt_grain_volumes (voxel count of every grain id 1..num_grains over the
 * interior cells of an argmax map, counts[0] = interior cells with no such id),
 * but the caller passes the argmax map alpha_dev (reference layout,
 * fnx*fny*fnz int32, already in device memory) and a host array counts of
 * num_grains+1 entries, and the call allocates nothing: its scratch is a fixed
 * device array of CUPF_NOALLOC_MAX_GRAINS+1 counts and first-occurrence
 * indices (1 MiB) that every GPU loading the library holds until the process
 * exits.  num_grains above CUPF_NOALLOC_MAX_GRAINS is rejected
 * (CUPF_ERR_INVALID).  Work is queued on `stream` (a cudaStream_t, NULL for
 * the default stream) on the current device, and the call returns after the
 * counts are in host memory (the call is synchronous).  The first call on a
 * device looks up the scratch address (cudaGetSymbolAddress).  Every call
 * shares the one scratch array and clears it first, so
 * calls whose GPU work overlaps (different streams or threads on one device)
 * race and must be serialised by the caller. */
#define CUPF_NOALLOC_MAX_GRAINS 65535
cupf_status cupf_grain_volumes_noalloc(const int32_t* alpha_dev, int32_t fnx, int32_t fny,
                                       int32_t fnz, int32_t num_grains, int64_t* counts,
                                       void* stream);

/* Moving-domain check and shift (line configuration).  Computes the per-layer
 * mean of phi over all slots and cells, advances *tip_front while the mean is
 * above LS, and while *tip_front >= tip_thres shifts the window down one layer:
 * archives the bottom interior alpha layer into alpha_full[move_count] (device
 * archive of fnz_f layers), adds its cells to loss_area, sets the new top
 * interior layer to (-1, -1) and shifts z.  Ends with the boundary fill and a
 * fresh argmax.  *moved receives the number of layers shifted.
 * Replaces APTPhaseField::moveDomain + tip_mvf + APTmove_frame + APTcopy_frame
 * (3DgrainMPI/APTPhaseField.cu:678-697, 357-410; PhaseField.cu:366-399). */
cupf_status cupf_apt_move_domain(cupf_apt_handle* h, int32_t* tip_front,
                                 int32_t tip_thres, int32_t* move_count,
                                 int32_t* moved);

/* Read back the archive of evicted alpha layers (fnx*fny*fnz_f ints) and the
 * per-grain lost area (num_theta ints); either pointer may be NULL.
 * The D2H copies of APTPhaseField::getLineQoIs / evolve
 * (3DgrainMPI/APTPhaseField.cu:668, 912). */
cupf_status cupf_apt_get_archive(cupf_apt_handle* h, int32_t fnz_f,
                                 int32_t* alpha_full, int32_t* loss_area);

/* Current z coordinates (fnz floats), shifted by cupf_apt_move_domain. */
cupf_status cupf_apt_get_z(cupf_apt_handle* h, float* z);

/* Wait for all work queued on the handle's stream, failing with
 * CUPF_ERR_TIMEOUT after timeout_ms milliseconds (<= 0: wait forever). */
cupf_status cupf_apt_sync(cupf_apt_handle* h, int32_t timeout_ms);

/* Time nsteps steps with CUDA events on the handle's stream (warm state, no
 * host copies).  *ms receives the elapsed device time. */
cupf_status cupf_apt_time_steps(cupf_apt_handle* h, int32_t nsteps, float* ms);

/* Raw stream of the handle (a cudaStream_t), for callers that order their own
 * work after the solver's. */
void* cupf_apt_stream(cupf_apt_handle* h);

/* Launch shape of the step kernel: z_chunk = interior planes per CTA work item
 * (the column tile is fixed at 32 x 8).  No reference counterpart (the
 * reference marches every column over the whole height, APTPhaseField.cu:190).
 * Without this call (or the CUPF_ZC environment variable) the library picks the
 * chunk whenever a state is loaded (init_from_argmax, set_slots) from the
 * planes that hold grain ids; after it, the given chunk stays. */
cupf_status cupf_apt_set_tuning(cupf_apt_handle* h, int32_t z_chunk);

/* Column-tile height of the step's work items (no counterpart in the reference,
 * whose kernel uses 32x4 thread blocks): 8 (the default) or 4 rows of 32 cells.
 * Results are identical for both; only the speed differs (the server picks per
 * grid shape by timing both with the z chunk).  Resets the quiet-item flags. */
cupf_status cupf_apt_set_tile(cupf_apt_handle* h, int32_t tile_y);

/* Quiet work items (on by default).  The step keeps, per work item and buffer, a
 * flag that every slot of the item's cells holds the empty pair (id -1, phi -1),
 * and leaves an item alone when its cells in the buffer it writes are already
 * empty and its cells and their face neighbours in the buffer it reads are too:
 * every cell of such an
 * item would be written empty again (APTrhs_psi on a cell whose 7 stencil
 * points hold no id, APTPhaseField.cu:198-233), so results are identical with
 * and without it.  enable = 0 computes every item (the reference's full sweep).
 * Init, set_slots and set_tuning reset the flags; a nucleation pass marks the
 * items its nuclei reach, and a domain shift moves the flags with the planes. */
cupf_status cupf_apt_set_skip_quiet(cupf_apt_handle* h, int32_t enable);

/* Bound of the step kernel's waits for its plane loads, in SM clock cycles (no
 * counterpart in the reference, which checks no CUDA error).  0 restores the
 * default of 2^31 cycles (about one second).  A wait that runs out makes the
 * step stop loading, wait (with the default bound) for the loads in flight,
 * record an error word and finish; the next synchronising call returns
 * CUPF_ERR_TIMEOUT, and the state is undefined until init_from_argmax or
 * set_slots, which clear the error word.  A short bound is meant for tests of
 * that path. */
cupf_status cupf_apt_set_wait_limit(cupf_apt_handle* h, int64_t cycles);

/* Merge overflows since the last call (hazard H1 of the reference's merge,
 * APTPhaseField.cu:222-231: a stencil holding more than NUM_PF distinct ids):
 * counts[0] = entries written to local_phs[s][NUM_PF], which aliases the next
 * point's slot 0 (s < 6, reproduced), counts[1] = entries past the array at the
 * last point (s == 6, dropped).  Resets both. */
cupf_status cupf_apt_merge_overflows(cupf_apt_handle* h, uint64_t* counts);

/* Cells of the work items the step computed (not left alone as quiet) since the
 * previous call, summed over steps; the counter restarts at 0. */
cupf_status cupf_apt_active_cells(cupf_apt_handle* h, uint64_t* cells);

/* ---------------------------------------------------------------- serving
 * Continuous batching of independent simulations on one GPU.  No reference
 * counterpart: the reference runs one simulation per process (main.cpp:15-77).
 * Requests of any grid size queue FIFO; cupf_server_pump retires finished
 * simulations (argmax map, per-grain volumes and FP64 interface sums copied to
 * host memory), admits queued ones while a slot and HBM within the budget are
 * free, and advances every resident simulation steps_per_round steps in one
 * persistent batched kernel per step, replayed from a captured CUDA graph.
 * A request's results are identical whether it runs alone or batched. */
typedef struct cupf_server cupf_server;

typedef struct cupf_server_config {
  int32_t device;
  int32_t precision;        /* cupf_precision, shared by every request */
  int32_t num_pf;           /* NUM_PF, shared by every request */
  int32_t max_active;       /* resident simulations at most */
  int32_t steps_per_round;  /* steps per graph replay (one pump) */
  int32_t autotune;         /* 1: pick the tile height and z chunk of each grid shape by timing */
  int64_t hbm_budget_bytes; /* device memory for requests; 0 = free memory - 2 GiB.
                               Requests' buffers come from a stream-ordered pool that
                               keeps what retired requests free for later admissions:
                               up to this much stays held until cupf_server_destroy */
  int32_t tile_y;           /* column-tile height: 0 = the autotuner's pick (8 without
                               autotune), or 4 / 8 for every request */
} cupf_server_config;

cupf_status cupf_server_create(const cupf_server_config* cfg, cupf_server** out);
cupf_status cupf_server_destroy(cupf_server* s);

/* Queue a simulation: parameters and inputs as for cupf_apt_create, initial
 * argmax fields as for cupf_apt_init_from_argmax (all copied, the fields into
 * page-locked host buffers the server recycles between requests, up to 4 GiB),
 * nsteps explicit steps (line / cylinder thermal types).  *request_id
 * identifies it. */
cupf_status cupf_server_submit(cupf_server* s, const cupf_apt_params* p,
                               const cupf_apt_inputs* in, const float* phi,
                               const int32_t* alpha, int64_t nsteps, int64_t* request_id);

/* Device time of the rounds waited for so far (CUDA events around each round's
 * graph launch, ms) and the number of rounds launched.  Either pointer may be
 * NULL. */
cupf_status cupf_server_stats(cupf_server* s, double* busy_ms, int64_t* rounds);

/* One scheduling round (see above).  It first waits for the previous round's
 * steps, retires and admits, then launches this round's steps and returns
 * without waiting for them, so the caller's own work between rounds overlaps
 * the device.  Counts are those after admission.  Any output pointer may be
 * NULL. */
cupf_status cupf_server_pump(cupf_server* s, int32_t* n_running, int32_t* n_pending,
                             int32_t* n_done);

/* State of a request (0 pending, 1 running, 2 done, 3 failed) and, when done,
 * its results: argmax grain map (length ints, as cupf_apt_collect with clear),
 * voxel counts per grain id 0..num_grains (as cupf_apt_grain_volumes), the three
 * FP64 sums of cupf_apt_qoi_sums, and the host clock (seconds) at submit,
 * admission and completion.  Output pointers may be NULL. */
cupf_status cupf_server_result(cupf_server* s, int64_t id, int32_t* status, int32_t* alpha_out,
                               int64_t* volumes_out, int32_t num_grains, double* qoi_out,
                               double* times_out);

/* Forget a finished (or still queued) request and its host results. */
cupf_status cupf_server_release(cupf_server* s, int64_t id);

/* Tile shape of a request's work items: the column-tile height (8 or 4) and the
 * z chunk the autotuner (or the configuration) picked for its grid shape; 0 and
 * 0 until it is admitted.  Either output pointer may be NULL. */
cupf_status cupf_server_request_tile(cupf_server* s, int64_t id, int32_t* tile_y,
                                     int32_t* z_chunk);

/* Column-tile height of requests admitted from now on: 0 = the autotuner's pick
 * (8 without autotune), 4 or 8 fixed (as cupf_server_config::tile_y).  Forgets
 * the earlier picks; resident requests keep theirs. */
cupf_status cupf_server_set_tile(cupf_server* s, int32_t tile_y);

#ifdef __cplusplus
}
#endif

#endif /* CUPF_H_ */
