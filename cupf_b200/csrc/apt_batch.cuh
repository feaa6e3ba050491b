// apt_batch.cuh — one launch advances every active simulation of a server by
// one step (continuous batching).
//
// Each simulation keeps its own pair buffers, tensor maps, parameters, step
// counter and ping-pong index in device memory (BatchSim), so a captured CUDA
// graph of K (step, finish) launch pairs can be replayed without host updates.
// The step kernel is persistent: CTAs pull (simulation, column tile, z chunk)
// work items from an atomic counter until the list is exhausted, and run the
// same per-item code as the single-simulation kernel (step_item), so a
// simulation's arithmetic and results do not depend on what else is batched
// with it.
#pragma once

#include "apt_step.cuh"

namespace cupf {

struct BatchSim {
  StepArgs a;          // in / out / t are filled per step from the fields below
  void* buf[2];
  uint8_t* quiet[2];   // quiet-item flags of each buffer (StepArgs::quiet_in/out)
  long long steps;     // explicit steps done
  long long target;    // steps requested
  int cur;             // buffer holding the current state
  int active;          // 1 while steps < target
  int use_iuc;
  int pad;
};

// TY: the column-tile height of every simulation in the launch (the server
// launches one kernel per tile height present in a round).
template <int NP, class S, int TY>
__global__ void __launch_bounds__(tile_threads<TY>(), step_min_blocks<NP, S, TY>())
    apt_batch_step_kernel(BatchSim* sims, const CUtensorMap* tmaps, const int4* items, int nitems,
                          int* work, const int* err) {
  extern __shared__ __align__(128) unsigned char smem[];
  CtaSmem<NP, S, TY> sm(smem);
  sm.init();
  int qbase = 0;
  for (;;) {
    const int it = next_work_item(work, nitems, sm.s_item, err);
    if (it < 0) break;
    const int4 w = items[it];  // simulation, txi, tyi, zci
    const BatchSim* sd = sims + w.x;
    if (!sd->active) continue;
    StepArgs a = sd->a;
    const int cur = sd->cur;
    a.in = sd->buf[cur];
    a.out = sd->buf[cur ^ 1];
    a.quiet_in = sd->quiet[cur];
    a.quiet_out = sd->quiet[cur ^ 1];
    a.use_iuc = sd->use_iuc;
    // t of step n (1-based) = (float)n * dt * tau0, as the single-simulation path
    a.t = __fmul_rn(__fmul_rn((float)(sd->steps + 1), a.dt), a.tau0);
    a.t64 = __dmul_rn(__dmul_rn((double)(sd->steps + 1), (double)a.dt), (double)a.tau0);
    a.sr_key = (uint32_t)(sd->steps + 1);
    if (a.quiet_out && item_quiet<TY>(a, w.y, w.z, w.w)) continue;
    step_item<NP, S, TY>(tmaps + 2 * w.x + cur, a, w.y, w.z, w.w, sm, qbase);
  }
  sm.drain();
}

// After every simulation's step: flip its buffers, count the step and retire
// it at its target.
static __global__ void batch_finish_kernel(BatchSim* sims, int nsims) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nsims && sims[i].active) {
    sims[i].cur ^= 1;
    sims[i].steps += 1;
    if (sims[i].steps >= sims[i].target) sims[i].active = 0;
  }
}

}  // namespace cupf
