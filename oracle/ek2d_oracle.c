/* ek2d_oracle.c — TEST INFRASTRUCTURE ONLY: CPU oracle of the 2D
 * Echebarria–Karma line model (cuPF 2DdendriteMPI/line_model/PF.cu and the
 * time loop of its setup()).  Used by tests/, smoke() and bench.py's CPU
 * baseline as the checker; the library never calls it.
 *
 * Two builds of one body (ek2d_oracle_impl.h):
 *   *_f64  double arithmetic, time and coordinates: the FP64 oracle against
 *          which split-precision results state their error;
 *   *_f32  float arithmetic with the reference's float time, y and pulling
 *          distance: checked against the reference's own kernels on the GPU
 *          (within a tolerance, since the GPU build contracts a*b+c into fused
 *          multiply-adds where this build, compiled with -ffp-contract=off,
 *          does not).
 * The noise term draws from Philox4x32-10 (oracle_philox in apt_oracle.c), as
 * the library does; the reference's curand stream is not reproduced. */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/cupf_ek2d.h"

void oracle_philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1,
                   uint32_t* out);

/* Uniform in (0, 1] from the top 24 bits, as the library's uniform01. */
static float ek2d_uniform01(uint32_t x) { return (float)((x >> 8) + 1u) * (1.0f / 16777216.0f); }

#define REAL double
#define SUF _f64
#define TANH tanh
#define SQRT sqrt
#define REF_TIME 0
#include "ek2d_oracle_impl.h"
#undef REAL
#undef SUF
#undef TANH
#undef SQRT
#undef REF_TIME

#define REAL float
#define SUF _f32
#define TANH tanhf
#define SQRT sqrtf
#define REF_TIME 1
#include "ek2d_oracle_impl.h"
#undef REAL
#undef SUF
#undef TANH
#undef SQRT
#undef REF_TIME
