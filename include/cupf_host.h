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

#ifdef __cplusplus
}
#endif

#endif /* CUPF_HOST_H_ */
