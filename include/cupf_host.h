/*
 * cupf_host.h — C entry points into the host side of the APT driver (the C++
 * classes in cupf_b200/host), for bindings and tests.  Each mirrors one host
 * routine of the reference driver; maps use the reference layout
 * (index i + j*fnx + k*fnx*fny).
 */
#ifndef CUPF_HOST_H_
#define CUPF_HOST_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* QOI::calculateQoIs (3DgrainMPI/QOI.cpp:198-231): grains with alpha > 0 over the
 * interior, in order of first occurrence; returns their count (or -1 if cap is
 * too small) and fills grain_ids[] / volumes[]. */
int cupf_host_grain_volumes(int fnx, int fny, int fnz, const int32_t* alpha, int32_t* grain_ids,
                            int32_t* volumes, int cap);

/* QOI::calculateLineQoIs (QOI.cpp:38-101) for one frame; *cur_tip in/out.
 * total_area / extra_area receive num_theta entries each. */
int cupf_host_line_qois(int fnx, int fny, int fnz, int num_theta, int* cur_tip,
                        const int32_t* alpha, const int32_t* loss_area, int move_count,
                        int32_t* tip_y, int32_t* total_area, int32_t* extra_area);

/* QOI::sampleHeights (QOI.cpp:162-185); *cur_tip in/out. */
int cupf_host_sample_heights(int* cur_tip, const int32_t* alpha, int fnx, int fny, int fnz);

/* QOI3D::searchJunctionsOnImage (QOI.cpp:233-311) after calculateQoIs; writes up to
 * cap ints of node records (i, j, k, max_occur, 4 grain ids, -1 padding) and
 * returns the record length used (40 * active grains * 9). */
int cupf_host_junctions_3d(int fnx, int fny, int fnz, const int32_t* alpha, int32_t* nodes, int cap);

/* The same records from the device's junction candidates: `cells` (ascending)
 * and `distinct` as cupf_apt_junction_candidates returns them. */
int cupf_host_junctions_3d_cells(int fnx, int fny, int fnz, const int32_t* alpha,
                                 const int64_t* cells, int64_t ncells, const uint8_t* distinct,
                                 int32_t* nodes, int cap);

/* QOILine::searchJunctionsOnImage (QOI.cpp:103-160) on a full line-configuration
 * map alpha (fnx*fny per layer) whose frame kt (0..nts) has its tip layer at
 * tip_y[kt], with num_nodes the input's NN: writes up to cap ints of node
 * records ((nts+1) frames x 5*NN records x 8 ints: i, j, max_occur, up to 5
 * grain ids, -1 padding) and, when cross is not NULL, up to cross_cap ints of
 * the frames' cross sections; returns the record length used, or -1. */
int cupf_host_line_junctions(int fnx, int fny, int nts, int num_nodes, const int32_t* tip_y,
                             const int32_t* alpha, int32_t* nodes, int cap, int32_t* cross,
                             int64_t cross_cap);

/* The same records from the device's candidates: `cells` (ascending) as
 * cupf_line_junction_candidates returns them for the frames' tip layers. */
int cupf_host_line_junctions_cells(int fnx, int fny, int nts, int num_nodes, const int32_t* tip_y,
                                   const int32_t* alpha, const int64_t* cells, int64_t ncells,
                                   int32_t* nodes, int cap, int32_t* cross, int64_t cross_cap);

/* Seeded 2D Voronoi substrate of nxp x nyp macro pixels (a line run's alpha.txt
 * holds (nx+1) x (ny+1) of them) with num_grains grains, for forcing folders
 * made without the reference's Python generator (graph_datastruct.py:194-271,
 * whose output format it keeps).  alpha (nxp*nyp, rows of constant y) gets each
 * pixel's grain id 1..num_grains: the nearest of num_grains seeded points, with
 * minimum-image distances when periodic is nonzero.  theta (2*num_grains+1)
 * gets [0, theta_x[1..NG], theta_z[1..NG]] from a Gaussian random vector per
 * grain (theta_x = atan2(u_y,u_x) mod pi, theta_z = atan2(|u_xy|,u_z) mod pi, as
 * graph_datastruct.py:256-269).  Same seed, same output.  Returns 0, or -1 on a
 * bad argument. */
int cupf_host_voronoi_substrate(int nxp, int nyp, int num_grains, uint64_t seed, int periodic,
                                int32_t* alpha, float* theta);

/* Grain orientations given as unit quaternions (w, x, y, z per grain, normalised
 * here) in the reference's two-angle form: theta (2*num_grains+1) gets
 * [0, theta_x[1..NG], theta_z[1..NG]], the azimuth and polar angle (mod pi, as
 * graph_datastruct.py:256-269) of each grain's crystal [001] axis in the lab
 * frame, which the step's rotation (APTPhaseField.cu:41-46) sends to the crystal
 * z axis.  The rotation about that axis has no parameter in the two-angle model
 * and is dropped.  Returns 0, or -1 on a bad argument or a zero quaternion.
 * The drivers read quaternions.txt (4*NG values) when theta.txt is absent. */
int cupf_host_quaternions_to_angles(int num_grains, const double* q, float* theta);

/* Writes alpha.txt ("%d" per line), theta.txt ("%1.4e" per line) and NG.txt
 * into an existing folder, as the reference's input scripts save them
 * (input_file.py:148-152).  Returns 0, or -1 on a bad argument or write. */
int cupf_host_write_substrate(const char* folder, int nxp, int nyp, const int32_t* alpha,
                              int num_grains, const float* theta);

/* h5write_1d of a whole file (3DgrainMPI/PhaseFieldCpu.cpp:584-613, as OutputQoIs /
 * OutputField use it): writes n 1-D datasets into the root group of a new HDF5
 * file at path (superblock version 0, contiguous little-endian data).  Dataset
 * i is named names[i] and holds counts[i] elements of kind kinds[i] ('i' signed
 * integer of 1, 2, 4 or 8 bytes, 'f' IEEE float of 4 or 8 bytes; elem_bytes[i])
 * read from data[i].  At most 1024 datasets; a repeated name keeps the last.
 * Returns 0, or -1 on a bad argument or a failed write. */
int cupf_host_h5_write(const char* path, int n, const char* const* names, const char* kinds,
                       const int32_t* elem_bytes, const int64_t* counts, const void* const* data);

/* getParam (helper.cpp:44-74); returns 1 if the key was set. */
int cupf_host_get_param_float(const char* line, const char* key, float* value);
int cupf_host_get_param_int(const char* line, const char* key, int32_t* value);

/* DesignSettingData::getOptions (DesignSettingData.cpp:14-80).
 * out: [useLineConfig, includeNucleation, pureNucleation, useAPT, save3DField,
 *       mpiDim, seedValue, bcX, bcY, bcZ]; strings are copied with cap bytes. */
int cupf_host_get_options(int argc, char** argv, int32_t* out, char* input_file, char* folder,
                          char* outdir, int cap);

/* parseInputParams + cpuSetup + initField (PhaseFieldCpu.cpp:17-459) on an input
 * file and forcing folder.  flags bit 0 = line configuration, bit 1 = pure
 * nucleation.  On success fills dims[0..3] = fnx, fny, fnz, num_theta and
 * fparams[0..7] = dt, tau0, lamd, hi, G, underCoolingRate, z0, kin_delta; and
 * copies phi / alpha (length entries each) when the pointers are not NULL and
 * length_cap is large enough.  Returns 0, or -1 with a message in err. */
int cupf_host_setup(const char* input_file, const char* folder, int bcX, int bcY, int bcZ,
                    int flags, int32_t* dims, float* fparams, float* phi, int32_t* alpha,
                    int64_t length_cap, char* err, int err_cap);

/* The same set-up with the state the reference's PhaseField holds after it
 * (PhaseFieldCpu.cpp:17-459): flags bit 2 = nucleation (includeNucleation).
 * dims[0..7] = fnx, fny, fnz, num_theta, Mt, nts, thermalType, fnz_f;
 * fparams[0..19] = dt, tau0, lamd, hi, G, underCoolingRate, z0, kin_delta, lxd,
 * lyd, lzd, R, V, top, r0, x0, cfl, underCoolingRate0, W0, dx.  x / y / z /
 * z_full receive fnx / fny / fnz / fnz_f coordinates; phi, psi, alpha (fnx*fny*fnz)
 * and sint, cost (2*num_theta+1) are copied when cap is large enough; any
 * output may be NULL.  Returns 0, 1 when cap was too small for the arrays, or
 * -1 with a message in err. */
int cupf_host_setup_state(const char* input_file, const char* folder, int bcX, int bcY, int bcZ,
                          int flags, int32_t* dims, float* fparams, float* x, float* y, float* z,
                          float* z_full, float* phi, float* psi, int32_t* alpha, float* sint,
                          float* cost, int64_t cap, char* err, int err_cap);

/* 2D Echebarria–Karma line model (cupf_ek2d.h).  The params type is declared
 * there; these take a pointer to it. */
struct cupf_ek2d_params;

/* Coordinates and initial fields of 2DdendriteMPI/line_model/main.cpp:225-271:
 * x (fnx), y (fny), psi/phi/U (fnx*fny, reference layout, halos zero) from the
 * 1-D profiles y_mac/psi_mac/U_mac of Ny points.  Any output may be NULL. */
int cupf_host_ek2d_initial_fields(const struct cupf_ek2d_params* p, int Ny, const float* y_mac,
                                  const float* psi_mac, const float* U_mac, float* x, float* y,
                                  float* psi, float* phi, float* U);

/* Seeded front perturbation (no counterpart in the reference): `sites`
 * Gaussian bumps evenly spaced in x, each adding amp*(2u-1) to psi (u from
 * Philox keyed on the site and seed_val); phi is recomputed. */
int cupf_host_ek2d_perturb(const struct cupf_ek2d_params* p, int sites, float amp, float* psi,
                           float* phi);

/* Quantities of interest of one phi frame (FP64): out[0] tip height (highest
 * phi = 0 crossing, um), out[1] mean column front height (um), out[2] primary
 * spacing (um, 0 without cells), out[3] its wavenumber index, out[4] the row
 * whose solid fraction is nearest 1/2 (-1 if none).  y holds the fny row
 * coordinates, dxd the cell size in um. */
int cupf_host_ek2d_qois(const float* phi, int fnx, int fny, const double* y, double dxd,
                        double* out);

#ifdef __cplusplus
}
#endif

#endif /* CUPF_HOST_H_ */
