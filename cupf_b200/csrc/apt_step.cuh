// apt_step.cuh — the fused APT step kernel for sm_100a.
//
// One launch = one explicit step of the reference's APTsetBC3D + APTrhs_psi
// pair (3DgrainMPI/APTPhaseField.cu:93-174, 178-354): boundary fill, neighbour
// grain-id gather with the first-seen merge, per-slot anisotropic update.
//
// Work decomposition: a CTA owns a TX x TY column tile of interior (x, y) cells
// (TX = 32, one warp per tile row; TY = 8 or 4, a template parameter the host
// picks per simulation, the server by timing) and a z chunk of ZC planes; one
// thread per (x, y) column marches z.  Planes of
// the input pair buffer (all NUM_PF slots, tile plus one-cell halo) stream into
// shared memory through a ring of S stages filled by TMA
// (cp.async.bulk.tensor.4d, one 4-D box {TX+2, TY+2, 1, NP} per plane) and
// completed on per-stage mbarriers.  Computing plane k needs planes k-1, k, k+1
// resident; planes k+2, k+3 are in flight.
//
// Boundary fill: plane indices 0 and fnz-1 are loaded from their mapped source
// planes (TMA coordinate remap), and the x/y halo cells are read from HBM,
// where they hold their mapped interior source: the step writes every cell it
// computes also into the halo cells that map to it, and every other writer of
// the pair buffers (initialisation, import, nucleation, domain shift) is
// followed by a fill of the halo.  Halo edges and corners, which no 7-point
// stencil reads, are not maintained by the step.
//
// After a plane lands, each cell of its tile gets a slot-occupancy bit mask
// (bit p set when slot p holds an id).  The merge then visits only occupied
// slots of the 7 stencil points, in the reference's order (D,B,L,C,R,T,U) x
// slot, and records for every stencil point which source slot feeds which
// output slot (4-bit codes), so the per-slot update reads exactly the values
// the reference's local_phs array would hold, including its aliasing write on
// merge overflow (local_phs[s][NUM_PF] == local_phs[s+1][0]).
#pragma once

#include "apt_storage.cuh"
#include "apt_update.cuh"

namespace cupf {

constexpr int TX = 32;
constexpr int STAGES = 5;

// Column-tile heights the step is built for (the box height is TY + 2 cells; the
// box width is the storage format's kBW).
constexpr bool tile_height_built(int ty) { return ty == 8 || ty == 4; }
template <int TY>
constexpr int tile_threads() {
  return TX * TY;
}

template <int NP, class S, int TY>
struct StepSmem {
  static constexpr int BW = S::kBW;
  static constexpr int BH = TY + 2;
  static constexpr int BCELLS = BW * BH;
  static constexpr int kBoxBytes = NP * BCELLS * S::kBytes;      // bytes one TMA plane load delivers
  static constexpr int kStageBytes = (kBoxBytes + 127) & ~127;  // stage stride (TMA dst: 128 B aligned)
  static constexpr int kStagePairs = kStageBytes / S::kBytes;
  static constexpr int kMaskOff = STAGES * kStageBytes;
  // 16-bit pairs in 32x8 tiles: the centre plane's phi values decoded once per
  // plane into FP32 (slot-major like a stage, plus one row of -1 that the absent
  // code NP points at), read by the five stencil points in that plane.  Three
  // CTAs per SM still fit; for 32x4 tiles the extra row would cost one.
  static constexpr bool kDecode = S::kBytes == 4 && TY == 8;
  static constexpr int kDecOff = (kMaskOff + STAGES * BCELLS * 2 + 15) & ~15;
  static constexpr int kDecBytes = kDecode ? (NP + 1) * BCELLS * 4 : 0;
  static constexpr int kBarOff = (kDecOff + kDecBytes + 7) & ~7;
  // + abort word, issued count, item index, one occupancy flag per stage
  static constexpr int kBytes = kBarOff + STAGES * 8 + 16 + STAGES * 4;
};

// Per-slot update loop shape of a storage format: rolled for the 16-bit pairs,
// unrolled over NUM_PF for FP32 (each measured faster for its format).
template <class S>
struct RolledSlots {
  static constexpr bool value = S::kBytes == 4;
};

template <int NP>
using CodeMap = typename std::conditional<(NP <= 8), uint32_t, unsigned long long>::type;

// Replace 4-bit field j of a code map with v (one bfi for 32-bit maps).
__device__ __forceinline__ uint32_t nib_insert(uint32_t c, uint32_t v, int j) {
  uint32_t r;
  asm("bfi.b32 %0, %1, %2, %3, 4;" : "=r"(r) : "r"(v), "r"(c), "r"(4 * j));
  return r;
}
__device__ __forceinline__ unsigned long long nib_insert(unsigned long long c, uint32_t v, int j) {
  const int sh = 4 * j;
  return (c & ~(0xFull << sh)) | ((unsigned long long)v << sh);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ bool mbar_test_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Wait for a stage with a bounded spin: by default about one second of SM
// clock (kWaitCycles), then give up and report (the caller records an error and
// carries on so that every thread still reaches every barrier).  A try_wait may
// itself suspend the thread for a hardware-chosen interval, so a bound shorter
// than kShortWait is kept with non-blocking probes only.
constexpr long long kWaitCycles = 1ll << 31;
constexpr long long kShortWait = 1ll << 20;
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity,
                                                  long long limit = kWaitCycles) {
  if (limit < kShortWait) {
    const long long t0 = clock64();
    do {
      if (mbar_test_wait(bar, parity)) return true;
    } while (clock64() - t0 <= limit);
    return false;
  }
  if (mbar_try_wait(bar, parity)) return true;
  long long t0 = clock64();
  while (!mbar_try_wait(bar, parity)) {
    if (clock64() - t0 > limit) return false;
  }
  return true;
}

__device__ __forceinline__ void tma_load_plane(void* dst, const CUtensorMap* map, uint64_t* bar,
                                               int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_u32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(z), "r"(0), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Per-CTA shared-memory state, carved from the dynamic allocation.
template <int NP, class S, int TY>
struct CtaSmem {
  using P = typename S::T;
  using Smem = StepSmem<NP, S, TY>;
  P* stages;
  uint16_t* masks;
  float* dec;     // decoded centre plane (Smem::kDecode)
  uint64_t* bars;
  int* s_abort;   // global plane sequence number of the first failed wait, + 1
  int* s_issued;  // plane sequence numbers issued so far (written by thread 0)
  int* s_item;    // work item handed to the CTA (batched kernel)
  int* s_occ;     // per stage: some cell of the landed plane holds an id
  __device__ explicit CtaSmem(unsigned char* smem) {
    stages = reinterpret_cast<P*>(smem);
    masks = reinterpret_cast<uint16_t*>(smem + Smem::kMaskOff);
    dec = reinterpret_cast<float*>(smem + Smem::kDecOff);
    bars = reinterpret_cast<uint64_t*>(smem + Smem::kBarOff);
    s_abort = reinterpret_cast<int*>(smem + Smem::kBarOff + STAGES * 8);
    s_issued = s_abort + 1;
    s_item = s_abort + 2;
    s_occ = s_abort + 4;
  }
  __device__ void init() {
    if (threadIdx.x == 0) {
      for (int s = 0; s < STAGES; ++s) mbar_init(&bars[s], 1);
      *s_abort = 0;
      *s_issued = 0;
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (Smem::kDecode)
      for (int c = threadIdx.x; c < Smem::BCELLS; c += blockDim.x) dec[NP * Smem::BCELLS + c] = -1.0f;
    __syncthreads();
  }
  // After a timed-out wait no further loads are issued; before the CTA exits
  // (and its shared memory is reused) wait, bounded by the default limit
  // whatever the launch's own, for those in flight.
  __device__ void drain() {
    __syncthreads();
    if (threadIdx.x == 0 && *s_abort) {
      for (int q = *s_abort - 1; q < *s_issued; ++q)
        mbar_wait_bounded(&bars[q % STAGES], (uint32_t)((q / STAGES) & 1));
    }
  }
};

// One work item: the column tile (txi, tyi) over the z chunk zci of one
// simulation.  qbase is the CTA's running plane sequence number: plane q of
// this item is sequence number qbase + q, which fixes its stage (mod STAGES)
// and the mbarrier phase parity; every issued plane is waited exactly once, in
// order, so the phases stay consistent across items.
template <int NP, class S, int TY>
__device__ __forceinline__ void step_item(const CUtensorMap* tmap, const StepArgs& a, int txi,
                                          int tyi, int zci, CtaSmem<NP, S, TY>& sm, int& qbase) {
  using Map = CodeMap<NP>;
  static_assert(NP <= 8, "slot codes are 4-bit fields of one 32-bit word");
  using Smem = StepSmem<NP, S, TY>;
  constexpr int NTHREADS = tile_threads<TY>();
  using P = typename S::T;
  constexpr int BW = Smem::BW;
  constexpr int BCELLS = Smem::BCELLS;
  constexpr bool kDec = Smem::kDecode;
  // code of an absent source slot: NP (the decoded plane's row of -1) where the
  // centre plane is decoded, else 0xF; 0xE marks the aliased overflow value
  constexpr uint32_t kAbsent = kDec ? (uint32_t)NP : 0xFu;
  // offsets of the centre plane's stencil points B, L, C, R, T from the cell
  constexpr int ctr_off[7] = {0, -BW, -1, 0, 1, BW, 0};
  P* stages = sm.stages;
  uint16_t* masks = sm.masks;
  uint64_t* bars = sm.bars;
  int* s_abort = sm.s_abort;
  int* s_issued = sm.s_issued;
  P* gout = static_cast<P*>(a.out);

  const int tid = threadIdx.x;
  const int tx = tid % TX, ty = tid / TX;
  const int x0 = 1 + TX * txi;  // first interior x of the tile
  const int y0 = 1 + TY * tyi;
  const int k_begin = 1 + a.zc * zci;
  const int k_end = min(k_begin + a.zc, a.fnz - 1);
  const int nplanes = k_end - k_begin + 2;  // planes k_begin-1 .. k_end
  const long long ss = a.slot_stride;
  const long long plane_pairs = (long long)a.xp * a.fny;
  const int q0 = qbase;

  auto issue = [&](int q) {  // plane index q -> logical z = k_begin - 1 + q
    const int g = q0 + q;
    const int s = g % STAGES;
    const int zl = k_begin - 1 + q;
    const int zp = bc_map(zl, a.fnz, a.bcZ);
    if (kDec) sm.s_occ[s] = 0;
    mbar_arrive_expect_tx(&bars[s], Smem::kBoxBytes);
    tma_load_plane(stages + (size_t)s * Smem::kStagePairs, tmap, &bars[s], x0 - 1, y0 - 1, zp);
    *s_issued = g + 1;
  };

  // the previous item (if any) is done with every stage before they refill
  __syncthreads();
  if (tid == 0 && !*s_abort) {
    fence_proxy_async();
    const int npre = min(STAGES, nplanes);
    for (int q = 0; q < npre; ++q) issue(q);
  }

  // Wait for plane q and compute the occupancy masks of its cells.
  auto land = [&](int q) {
    const int g = q0 + q;
    const int s = g % STAGES;
    const uint32_t parity = (uint32_t)((g / STAGES) & 1);
    if (!*s_abort && !mbar_wait_bounded(&bars[s], parity, a.wait_limit)) {
      atomicCAS(s_abort, 0, g + 1);
      atomicExch(a.err, ERR_TMA_TIMEOUT);
    }
    const P* st = stages + (size_t)s * Smem::kStagePairs;
    uint32_t any = 0;
    for (int c = tid; c < BCELLS; c += NTHREADS) {
      uint32_t m = 0;
#pragma unroll
      for (int p = 0; p < NP; ++p) m |= (uint32_t)(S::id(st[p * BCELLS + c]) != -1) << p;
      masks[s * BCELLS + c] = (uint16_t)m;
      any |= m;
    }
    if (kDec && any) sm.s_occ[s] = 1;
  };

  land(0);
  land(1);
  // bit 0: this thread wrote a slot other than the exact empty pair (an occupied
  // slot, or one whose id was just dropped: it keeps its last phi) or left one
  // unwritten; bits 1 and 2: the same in the item's bottom and top plane
  uint32_t live = 0;
  // merge overflows of this thread's cells (StepArgs::overflows), aliased ones
  // in the low 16 bits and dropped ones in the high 16 (at most 7 NP per cell
  // and plane), summed per warp at the end of the item
  uint32_t n_ovf = 0;

  const int gx = x0 + tx, gy = y0 + ty;
  const bool valid = gx <= a.fnx - 2 && gy <= a.fny - 2;
  const int c = (ty + 1) * BW + (tx + 1);
  // offsets (in pairs, 0 = none) from this cell to the x/y halo cells whose
  // boundary map sources it (APTsetBC3D, APTPhaseField.cu:93-174)
  const int hdx0 = bc_map(0, a.fnx, a.bcX) == gx ? -gx : 0;
  const int hdx1 = bc_map(a.fnx - 1, a.fnx, a.bcX) == gx ? a.fnx - 1 - gx : 0;
  const int hdy0 = bc_map(0, a.fny, a.bcY) == gy ? -gy * a.xp : 0;
  const int hdy1 = bc_map(a.fny - 1, a.fny, a.bcY) == gy ? (a.fny - 1 - gy) * a.xp : 0;
  const bool halo_any = (hdx0 | hdx1 | hdy0 | hdy1) != 0;
  // the line profile and the liquid-start undercooling depend on z only: one
  // evaluation per plane instead of one per cell
  const bool plane_T = a.use_iuc || a.thermalType == 0 || a.thermalType == 1;
  const float kLS = __uint_as_float(kLSFloatBits);
  const float kDrop = __uint_as_float(kDropFloatBits);
  const KineConst kc = kine_const(a.kin_delta);

  for (int k = k_begin; k < k_end; ++k) {
    const int qk = k - k_begin + 1;
    float Up_plane = 0.0f;
    if (plane_T) {
      float T;
      tinterp(a, 0, 0, k, &T);
      Up_plane = __fdiv_rn(T, a.L_cp);
    }
    land(qk + 1);
    __syncthreads();
    if (tid == 0 && qk >= 2 && qk - 2 + STAGES < nplanes && !*s_abort) {
      fence_proxy_async();
      issue(qk - 2 + STAGES);
    }
    const int sD = (q0 + qk - 1) % STAGES, sC = (q0 + qk) % STAGES, sU = (q0 + qk + 1) % STAGES;
    // decode the centre plane's phi once (a plane without ids needs none: every
    // code into it is then absent); every thread has finished the previous
    // plane, the last reader of the decoded values, at the barrier above
    if constexpr (kDec) {
      if (sm.s_occ[sC]) {
        // four pairs per thread and pass (a stage and the decoded plane start on
        // 16-byte boundaries; NP * BCELLS is a multiple of 4)
        static_assert((NP * BCELLS) % 4 == 0, "vector decode");
        const uint4* st = reinterpret_cast<const uint4*>(stages + (size_t)sC * Smem::kStagePairs);
        float4* d4 = reinterpret_cast<float4*>(sm.dec);
        for (int e = tid; e < NP * BCELLS / 4; e += NTHREADS) {
          const uint4 w = st[e];
          d4[e] = make_float4(S::phi(w.x), S::phi(w.y), S::phi(w.z), S::phi(w.w));
        }
        __syncthreads();
      }
    }
    if (!valid) continue;

    const P* pD = stages + (size_t)sD * Smem::kStagePairs + c;
    const P* pC = stages + (size_t)sC * Smem::kStagePairs + c;
    const P* pU = stages + (size_t)sU * Smem::kStagePairs + c;
    const P* pts[7] = {pD, pC - BW, pC - 1, pC, pC + 1, pC + BW, pU};
    uint32_t mk[7];
    mk[0] = masks[sD * BCELLS + c];
    mk[1] = masks[sC * BCELLS + c - BW];
    mk[2] = masks[sC * BCELLS + c - 1];
    mk[3] = masks[sC * BCELLS + c];
    mk[4] = masks[sC * BCELLS + c + 1];
    mk[5] = masks[sC * BCELLS + c + BW];
    mk[6] = masks[sU * BCELLS + c];

    P* outp = gout + (long long)k * plane_pairs + (long long)gy * a.xp + gx;
    // write pair v to output slot j of this cell and to the halo cells it sources
    auto put = [&](int j, P v) {
      P* o = outp + j * ss;
      *o = v;
      if (halo_any) {
        if (hdx0) o[hdx0] = v;
        if (hdx1) o[hdx1] = v;
        if (hdy0) o[hdy0] = v;
        if (hdy1) o[hdy1] = v;
      }
    };
    bool clive = false;
    const uint32_t any = mk[0] | mk[1] | mk[2] | mk[3] | mk[4] | mk[5] | mk[6];
    if (any == 0) {
      const P empty = S::empty();
#pragma unroll
      for (int p = 0; p < NP; ++p) put(p, empty);
      continue;
    }

    // ---- merge: first-seen order over (D,B,L,C,R,T,U) x slot
    int L[NP];
#pragma unroll
    for (int q = 0; q < NP; ++q) L[q] = -1;
    int n = 0;
    Map code[7];
    float alias[7];
#pragma unroll
    for (int s = 0; s < 7; ++s) {
      code[s] = kDec ? (Map)(0x11111111u * kAbsent) : ~(Map)0;
      alias[s] = -1.0f;
    }
    bool has_alias = false;  // some point's slot 0 holds an aliased overflow value
    // General visit of stencil point s: each occupied slot's id is looked up in
    // the list and appended when new (APTPhaseField.cu:211-233).
    auto merge_point = [&](int s) {
      uint32_t m = mk[s];
      while (m) {
        const int p = __ffs(m) - 1;
        m &= m - 1;
        const P pr = pts[s][p * BCELLS];
        const int id = S::id(pr);
        int j = n;
#pragma unroll
        for (int q = NP - 1; q >= 0; --q)
          if (L[q] == id) j = q;
        if (j == n) {
          if (n < NP) {
#pragma unroll
            for (int q = 0; q < NP; ++q)
              if (q == n) L[q] = id;
            ++n;
          } else {
            // local_phs[s][NUM_PF] aliases local_phs[s+1][0]; past the array at s == 6
            if (s < 6) {
              code[s + 1] = nib_insert(code[s + 1], 0xEu, 0);
              alias[s + 1] = S::phi(pr);
              has_alias = true;
            }
            n_ovf += s < 6 ? 1u : 0x10000u;
            continue;
          }
        }
        code[s] = nib_insert(code[s], (uint32_t)p, j);
      }
    };
    // A point whose every occupied slot q holds the id already at list position
    // q maps q to q and adds nothing to the list: the general visit finds each of
    // its ids at q (the list holds distinct ids).  The centre and the point above
    // nearly always satisfy this, because every cell's slot order is the
    // first-seen order of its own neighbourhood, which starts with the column.
    auto identity_point = [&](int s) -> bool {
      const uint32_t m = mk[s];
      bool ok = true;
      Map occ = 0;
#pragma unroll
      for (int q = 0; q < NP; ++q)
        if ((m >> q) & 1u) {
          ok = ok && (S::id(pts[s][q * BCELLS]) == L[q]);
          occ |= (Map)0xF << (4 * q);
        }
      if (ok) code[s] = (code[s] & ~occ) | ((Map)0x76543210u & occ);
      return ok;
    };
    // The point below comes first: the list is empty, so its slot p can only meet
    // the ids of its own lower slots (n <= p, and the list cannot overflow).
    {
      const uint32_t m = mk[0];
#pragma unroll
      for (int p = 0; p < NP; ++p) {
        if (!((m >> p) & 1u)) continue;
        const int id = S::id(pts[0][p * BCELLS]);
        int j = n;
#pragma unroll
        for (int q = p - 1; q >= 0; --q)
          if (L[q] == id) j = q;
        if (j == n) {
#pragma unroll
          for (int q = 0; q <= p; ++q)
            if (q == n) L[q] = id;
          ++n;
        }
        code[0] = nib_insert(code[0], (uint32_t)p, j);
      }
    }
    merge_point(1);
    merge_point(2);
    if (!identity_point(3)) merge_point(3);
    merge_point(4);
    merge_point(5);
    if (!identity_point(6)) merge_point(6);

    // Value of output slot j at stencil point s: kAbsent = absent (-1), 0xE = the
    // aliased overflow value, which only ever lands in slot 0 (kAlias false: the
    // caller knows no point of the cell has one).  The five points of the centre
    // plane read the decoded plane where there is one.
    auto fetch = [&](int s, int j, auto alias_tag) -> float {
      constexpr bool kAlias = decltype(alias_tag)::value;
      const uint32_t cd = (uint32_t)(code[s] >> (4 * j)) & 0xF;
      const bool al = kAlias && j == 0 && cd == 0xEu;
      if (kDec && s >= 1 && s <= 5) {
        // the index stays inside the decoded plane for the alias code too
        const float v = sm.dec[(al ? kAbsent : cd) * BCELLS + c + ctr_off[s]];
        return al ? alias[s] : v;
      }
      if (al) return alias[s];
      if (cd == kAbsent) return -1.0f;
      return S::phi(pts[s][cd * BCELLS]);
    };
    using WithAlias = std::integral_constant<bool, true>;
    using NoAlias = std::integral_constant<bool, false>;

    // phi + 1 at the centre for every slot (the repulsion sum's terms); the loops
    // over slots stop at n, so a warp runs only as many iterations as its
    // fullest cell
    float phc1[NP];
#pragma unroll
    for (int q = 0; q < NP; ++q) phc1[q] = 0.0f;
#pragma unroll
    for (int q = 0; q < NP; ++q) {
      if (q >= n) break;
      phc1[q] = __fadd_rn(fetch(3, q, WithAlias{}), 1.0f);
    }

    // rounding bits of this cell and step: keyed on the cell's reference-layout
    // index and the step number, so a simulation rounds the same alone or batched
    uint32_t cell_key = 0;
    if (S::kStochastic)
      cell_key = mix32((uint32_t)(gx + a.fnx * (gy + a.fny * k)) ^ mix32(a.sr_key));

    float Up = Up_plane;
    bool upd = true;
    if (!plane_T) {
      float T;
      upd = tinterp(a, gx, gy, k, &T);
      Up = __fdiv_rn(T, a.L_cp);
    }

    // New value of output slot j < n holding grain `id`.
    auto update_slot = [&](int j, int id, auto alias_tag) -> P {
      // orientation of the grain (APTPhaseField.cu:259-273): loads issued before
      // the stencil values are gathered so their latency overlaps; ids are >= 0
      // here (cupf_apt_set_slots rejects other negative ids) and the clamp only
      // keeps a corrupted id from reading outside the tables
      int tid2 = id;
      if (id > a.num_theta)  // id % num_theta + 1
        tid2 = id - (int)div_invariant((uint32_t)id, a.nt_magic, a.nt_sh1, a.nt_sh2) * a.num_theta + 1;
      const bool tab_ok = (unsigned)tid2 <= (unsigned)a.num_theta;
      const int ti = tab_ok ? tid2 : 0;
      const float4 t_o = __ldg(a.orient + ti);  // {sint[ti], cost[ti], sint[ti+NG], cost[ti+NG]}
      float ph7[7];
#pragma unroll
      for (int s = 0; s < 7; ++s) ph7[s] = fetch(s, j, alias_tag);
      float sina = 0.0f, cosa = 1.0f, sinb = 0.0f, cosb = 1.0f;
      if (ph7[3] > kLS && tab_ok) {  // (double)phC > LS
        sina = t_o.x;
        cosa = t_o.y;
        sinb = t_o.z;
        cosb = t_o.w;
      }
      // repulsion sum over the other slots (APTPhaseField.cu:328-335): the
      // reference accumulates r += 0.25 (phi+1)(phi+1) with the product fused,
      // r' = RN(0.25 q q + r).  Kept four times larger, R = 4 r, the same sum is
      // R' = RN(q q + R) = 4 RN(0.25 q q + r) exactly (scaling by a power of two
      // commutes with rounding; every term is far from the subnormal range), so
      // one fused multiply-add per term and one multiply at the end give the
      // reference's bits.
      static_assert(Contract::REP == 1, "the scaled sum restates the fused form only");
      float rsum = 0.0f;
#pragma unroll
      for (int q = 0; q < NP; ++q) {
        if (q >= n) break;
        if (q != j) rsum = __fmaf_rn(phc1[q], phc1[q], rsum);
      }
      const float repul = __fmul_rn(0.25f, rsum);
      const float nv = slot_update(a, kc, ph7, sina, cosa, sinb, cosb, repul, Up);
      const int oid = (nv < kDrop) ? -1 : id;  // (double)nv < -0.9999
      // slot j's rounding bits: the cell's hashed key times a distinct odd
      // constant per slot (a bijection of a uniform 32-bit value, one multiply)
      if (S::kStochastic) return S::make_sr(nv, oid, cell_key * ((uint32_t)(2 * j + 1) * 0x9E3779B9u));
      return S::make(nv, oid);
    };
    if constexpr (RolledSlots<S>::value) {
      static_assert(S::kBytes == 4, "the packed id queue holds 16-bit ids");
      // 16-bit pairs: one loop body run to the cell's slot count (the smaller code
      // and register footprint measured faster at three CTAs per SM)
#pragma unroll
      for (int j = 0; j < NP; ++j)
        if (j >= n) put(j, S::empty());
      if (upd) {
        auto slots = [&](auto alias_tag) {
          // the list's ids (16-bit in these formats) packed two to a word and
          // shifted down one id per slot: slot j's id is always the low half
          uint32_t w[(NP + 1) / 2];
#pragma unroll
          for (int q = 0; q < (NP + 1) / 2; ++q)
            w[q] = __byte_perm((uint32_t)L[2 * q], 2 * q + 1 < NP ? (uint32_t)L[2 * q + 1] : 0u, 0x5410);
#pragma unroll 1
          for (int j = 0; j < n; ++j) {
            const int id = (int)(short)(w[0] & 0xFFFFu);
#pragma unroll
            for (int q = 0; q < (NP + 1) / 2 - 1; ++q) w[q] = __funnelshift_r(w[q], w[q + 1], 16);
            w[(NP + 1) / 2 - 1] >>= 16;
            const P v = update_slot(j, id, alias_tag);
            clive |= !S::is_empty(v);
            put(j, v);
          }
        };
        // merge overflows are rare: a warp none of whose cells has an aliased
        // value runs the loop without the alias checks
        if (__any_sync(__activemask(), has_alias))
          slots(WithAlias{});
        else
          slots(NoAlias{});
      } else {
        clive = true;
      }
    } else {
#pragma unroll
      for (int j = 0; j < NP; ++j) {
        if (j >= n) {
          put(j, S::empty());
        } else if (upd) {
          const P v = update_slot(j, L[j], WithAlias{});
          clive |= !S::is_empty(v);
          put(j, v);
        } else {
          clive = true;  // the reference leaves the slot unwritten
        }
      }
    }
    if (clive) live |= 1u | (k == k_begin ? 2u : 0u) | (k == k_end - 1 ? 4u : 0u);
  }

  // record which of the item's output, its bottom plane and its top plane hold
  // only exact empty pairs (flag bits 0, 1, 2)
  const int busy = __syncthreads_or(live & 1u), busy_lo = __syncthreads_or(live & 2u),
            busy_hi = __syncthreads_or(live & 4u);
  if (tid == 0 && a.quiet_out)
    a.quiet_out[(zci * a.nty + tyi) * a.ntx + txi] =
        (uint8_t)((busy ? 0 : 1) | (busy_lo ? 0 : 2) | (busy_hi ? 0 : 4));
  if (a.overflows) {
    const uint32_t wa = __reduce_add_sync(0xffffffffu, n_ovf & 0xFFFFu);
    const uint32_t wd = __reduce_add_sync(0xffffffffu, n_ovf >> 16);
    if ((tid & 31) == 0 && (wa | wd)) {
      atomicAdd(a.overflows, (unsigned long long)wa);
      atomicAdd(a.overflows + 1, (unsigned long long)wd);
    }
  }
  if (tid == 0 && a.active_cells) {
    const int wx = min(TX, a.fnx - 1 - x0), wy = min(TY, a.fny - 1 - y0);
    atomicAdd(a.active_cells, (unsigned long long)(wx * wy * (k_end - k_begin)));
  }

  qbase = q0 + nplanes;
}

// True when the step may leave work item (txi, tyi, zci) alone: its cells in
// the output buffer already hold only exact empty pairs (id -1, phi -1), and its
// cells and the face-neighbour cells its 7-point stencil reads in the input
// buffer hold no id.  Those neighbours are the whole items across the x and y
// faces (or the items the boundary map sends a halo cell to), and across the z
// faces the top plane of the item below and the bottom plane of the item above
// (flag bits 2 and 1; a halo plane maps to an arbitrary plane, so there the
// whole item's bit 0).  Every cell of such an item would be written as the empty
// pair again.
template <int TY>
__device__ __forceinline__ bool item_quiet(const StepArgs& a, int txi, int tyi, int zci) {
  const int per = a.ntx * a.nty;
  const int it = zci * per + tyi * a.ntx + txi;
  if (!(a.quiet_out[it] & 1) || !(a.quiet_in[it] & 1)) return false;
  auto q = [&](int tx, int ty, int zc, int bit) {
    return (a.quiet_in[zc * per + ty * a.ntx + tx] & bit) != 0;
  };
  const int x0 = 1 + TX * txi, x1 = min(x0 + TX - 1, a.fnx - 2);
  const int y0 = 1 + TY * tyi, y1 = min(y0 + TY - 1, a.fny - 2);
  const int k0 = 1 + a.zc * zci, k1 = min(k0 + a.zc, a.fnz - 1);
  const int xl = bc_map(x0 - 1, a.fnx, a.bcX), xr = bc_map(x1 + 1, a.fnx, a.bcX);
  const int yl = bc_map(y0 - 1, a.fny, a.bcY), yr = bc_map(y1 + 1, a.fny, a.bcY);
  const bool below = k0 - 1 >= 1
                         ? q(txi, tyi, zci - 1, 4)
                         : q(txi, tyi, (bc_map(k0 - 1, a.fnz, a.bcZ) - 1) / a.zc, 1);
  const bool above = k1 <= a.fnz - 2 ? q(txi, tyi, zci + 1, 2)
                                     : q(txi, tyi, (bc_map(k1, a.fnz, a.bcZ) - 1) / a.zc, 1);
  return below && above && q((xl - 1) / TX, tyi, zci, 1) && q((xr - 1) / TX, tyi, zci, 1) &&
         q(txi, (yl - 1) / TY, zci, 1) && q(txi, (yr - 1) / TY, zci, 1);
}

// Hand the CTA its next work item from the launch's atomic counter (-1 when
// none is left).  After its last fetch each CTA counts itself done; the last one
// resets both words, so the next launch (or graph replay) starts from zero.
__device__ __forceinline__ int next_work_item(int* work, int nitems, int* s_item,
                                              const int* err) {
  __syncthreads();  // every thread has read the previous index
  if (threadIdx.x == 0) {
    int it = atomicAdd(work, 1);
    // a CTA that gave up on a load set the error word: take no further items
    // (read with the ticket, once per item, not per plane)
    if (*(volatile const int*)err != 0) it = nitems;
    if (it >= nitems) {
      it = -1;
      __threadfence();
      if (atomicAdd(work + 1, 1) == (int)gridDim.x - 1) {
        atomicExch(work, 0);
        atomicExch(work + 1, 0);
      }
    }
    *s_item = it;
  }
  __syncthreads();
  return *s_item;
}

// One launch = one step of one simulation.  Persistent CTAs pull work items
// (column tile x z chunk) from an atomic counter, z-chunk-major so the chunks
// nearest the bottom (the solid, where cells carry the most grain ids in a
// directional-solidification run) start first and the light liquid chunks fill
// in behind them.
// Resident CTAs per SM the step is compiled for.  32x8 tiles: three where three
// CTAs' shared memory fits (16-bit pairs, or FP32 up to NUM_PF = 5), else two.
// 32x4 tiles: twice that (the same registers per thread), or as many as their
// shared memory fits on one SM (228 KB) when fewer.
template <int NP, class S, int TY>
constexpr int step_min_blocks() {
  constexpr int tall = StepSmem<NP, S, 8>::kBytes <= 74 * 1024 ? 3 : 2;
  constexpr int by_smem = (228 * 1024) / StepSmem<NP, S, TY>::kBytes;
  return TY == 8 ? tall : (2 * tall < by_smem ? 2 * tall : by_smem);
}

template <int NP, class S, int TY>
__global__ void __launch_bounds__(tile_threads<TY>(), step_min_blocks<NP, S, TY>())
    apt_step_kernel(const __grid_constant__ CUtensorMap tmap, const StepArgs a) {
  extern __shared__ __align__(128) unsigned char smem[];
  CtaSmem<NP, S, TY> sm(smem);
  sm.init();
  const int per_chunk = a.ntx * a.nty;
  const int nitems = per_chunk * a.nzc;
  int qbase = 0;
  for (;;) {
    const int it = next_work_item(a.work, nitems, sm.s_item, a.err);
    if (it < 0) break;
    const int zci = it / per_chunk;
    const int r = it - zci * per_chunk;
    if (a.quiet_out && item_quiet<TY>(a, r % a.ntx, r / a.ntx, zci)) continue;
    step_item<NP, S, TY>(&tmap, a, r % a.ntx, r / a.ntx, zci, sm, qbase);
  }
  sm.drain();
}

}  // namespace cupf
