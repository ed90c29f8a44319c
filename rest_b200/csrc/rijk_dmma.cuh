// CTA-level FP64 tensor-core (DMMA, mma.m8n8k4.f64) contraction over 32x32
// operand slots staged by bulk copies.
//
// A CTA computes a (MT*32) x (NT*32) block of  sum_kt  A_kt * B_kt  where each
// k-step kt contributes MT A-slots (32 rows x 32 k) and NT B-slots (32 k x 32
// cols).  A schedule object says, for every (kt, slot), which 32x32 block of
// global memory to stage and in which orientation:
//
//   SlotSrc{ptr, ld, trans}: the block S[r][c] = ptr[r + ld*c] (column-major,
//   32 columns of 32 contiguous doubles).  For an A-slot, A[m][k] = S[m][k]
//   when trans == 0 and S[k][m] when trans == 1; for a B-slot, B[k][n] = S[k][n]
//   when trans == 0 and S[n][k] when trans == 1.  ptr == nullptr stages zeros.
//
// Staging: warp 0 issues one 256-byte cp.async.bulk per slot column into a
// slot with leading dimension 36 doubles (36 = 4 mod 16 makes the m8n8k4
// fragment loads bank-conflict free in both orientations), all completing on
// the stage's mbarrier.  STAGES stages are in flight; every wait is bounded.
#pragma once
#include "rijk_common.cuh"

namespace rijk {

struct SlotSrc {
  const double* ptr;
  int64_t ld;
  int trans;
};

template <int MT_, int NT_, int WM_, int WN_, int STAGES_>
struct DmmaCfg {
  static constexpr int MT = MT_, NT = NT_, WM = WM_, WN = WN_, STAGES = STAGES_;
  static constexpr int BM = MT * TS, BN = NT * TS;
  static constexpr int WARPS = WM * WN, THREADS = WARPS * 32;
  static constexpr int WTM = BM / WM, WTN = BN / WN;  // warp tile
  static constexpr int FM = WTM / 8, FN = WTN / 8;    // m8n8 fragments per warp
  static constexpr int SLOTS = MT + NT;
  static constexpr int STAGE_DOUBLES = SLOTS * SLOT_DOUBLES;
  static constexpr uint32_t STAGE_BYTES = SLOTS * TS * TS * 8;  // bytes landed per stage
  static constexpr size_t SMEM_BYTES = (size_t)STAGES * STAGE_DOUBLES * 8 + 64;
  static_assert(BM % WM == 0 && BN % WN == 0, "warp grid");
  static_assert(WTM % 8 == 0 && WTN % 8 == 0, "warp tile");
  static_assert(TS % WTM == 0 || WTM % TS == 0, "warp rows vs slot");
  static_assert(TS % WTN == 0 || WTN % TS == 0, "warp cols vs slot");
};

template <class Cfg, class Sched>
__device__ __forceinline__ void dmma_issue_stage(const Sched& sc, int kt, double* stage, uint64_t* bar) {
  const int lane = threadIdx.x & 31;
  if (lane == 0) mbar_arrive_expect_tx(bar, Cfg::STAGE_BYTES);
  __syncwarp();
#pragma unroll
  for (int s = 0; s < Cfg::SLOTS; ++s) {
    const SlotSrc src = (s < Cfg::MT) ? sc.a(kt, s) : sc.b(kt, s - Cfg::MT);
    const double* g = src.ptr ? src.ptr + (int64_t)lane * src.ld : g_zero_tile + lane * TS;
    bulk_g2s(stage + s * SLOT_DOUBLES + lane * SLD, g, TS * 8, bar);
  }
}

// Runs the k-loop of one CTA tile; acc[fm][fn][2] holds, for this thread, the
// elements (m = warp_m0 + 8 fm + lane/4, n = warp_n0 + 8 fn + 2 (lane%4) + j).
// Returns false if a stage wait timed out (the device error flag is then set).
template <class Cfg, class Sched>
__device__ __forceinline__ bool dmma_mainloop(const Sched& sc, int ktiles, double* smem, uint64_t* bars,
                                              double (&acc)[Cfg::FM][Cfg::FN][2], int* err) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int warp_m0 = (warp / Cfg::WN) * Cfg::WTM;
  const int warp_n0 = (warp % Cfg::WN) * Cfg::WTN;

#pragma unroll
  for (int i = 0; i < Cfg::FM; ++i)
#pragma unroll
    for (int j = 0; j < Cfg::FN; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

  if (tid == 0) {
    for (int s = 0; s < Cfg::STAGES; ++s) mbar_init(&bars[s], 1);
    mbar_fence_init();
  }
  __syncthreads();

  if (warp == 0) {
    for (int s = 0; s < Cfg::STAGES && s < ktiles; ++s)
      dmma_issue_stage<Cfg>(sc, s, smem + s * Cfg::STAGE_DOUBLES, &bars[s]);
  }

  for (int kt = 0; kt < ktiles; ++kt) {
    const int st = kt % Cfg::STAGES;
    const uint32_t parity = (uint32_t)((kt / Cfg::STAGES) & 1);
    const bool ok = mbar_wait_bounded(&bars[st], parity, err);
    if (!__syncthreads_and(ok)) {
      // Give the copies still in flight (stages kt+1 .. kt+STAGES-1) a bounded
      // time to land before the CTA's shared memory is released.
      if (tid == 0)
        for (int k2 = kt + 1; k2 < ktiles && k2 < kt + Cfg::STAGES; ++k2)
          mbar_wait_bounded(&bars[k2 % Cfg::STAGES], (uint32_t)((k2 / Cfg::STAGES) & 1), nullptr);
      __syncthreads();
      return false;
    }
    const double* sbase = smem + st * Cfg::STAGE_DOUBLES;

    // Per-fragment slot offsets and k strides for this k-step.
    int aoff[Cfg::FM], ask[Cfg::FM], boff[Cfg::FN], bsk[Cfg::FN];
#pragma unroll
    for (int fm = 0; fm < Cfg::FM; ++fm) {
      const int m = warp_m0 + fm * 8 + (lane >> 2);
      const int slot = m / TS, r = m % TS;
      const int tr = sc.a(kt, slot).trans;
      const int sm = tr ? SLD : 1, sk = tr ? 1 : SLD;
      aoff[fm] = slot * SLOT_DOUBLES + r * sm + (lane & 3) * sk;
      ask[fm] = 4 * sk;
    }
#pragma unroll
    for (int fn = 0; fn < Cfg::FN; ++fn) {
      const int n = warp_n0 + fn * 8 + (lane >> 2);
      const int slot = n / TS, c = n % TS;
      const int tr = sc.b(kt, slot).trans;
      const int sn = tr ? 1 : SLD, sk = tr ? SLD : 1;
      boff[fn] = (Cfg::MT + slot) * SLOT_DOUBLES + c * sn + (lane & 3) * sk;
      bsk[fn] = 4 * sk;
    }

#pragma unroll
    for (int kk = 0; kk < TS / 4; ++kk) {
      double af[Cfg::FM], bf[Cfg::FN];
#pragma unroll
      for (int fm = 0; fm < Cfg::FM; ++fm) af[fm] = sbase[aoff[fm] + kk * ask[fm]];
#pragma unroll
      for (int fn = 0; fn < Cfg::FN; ++fn) bf[fn] = sbase[boff[fn] + kk * bsk[fn]];
#pragma unroll
      for (int fm = 0; fm < Cfg::FM; ++fm)
#pragma unroll
        for (int fn = 0; fn < Cfg::FN; ++fn) dmma_m8n8k4(acc[fm][fn][0], acc[fm][fn][1], af[fm], bf[fn]);
    }
    __syncthreads();  // every warp is done reading stage st
    if (warp == 0 && kt + Cfg::STAGES < ktiles)
      dmma_issue_stage<Cfg>(sc, kt + Cfg::STAGES, smem + st * Cfg::STAGE_DOUBLES, &bars[st]);
  }
  return true;
}

// Visits every accumulator element of this thread with its CTA-local (m, n).
template <class Cfg, class F>
__device__ __forceinline__ void dmma_for_each(const double (&acc)[Cfg::FM][Cfg::FN][2], F&& f) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int warp_m0 = (warp / Cfg::WN) * Cfg::WTM;
  const int warp_n0 = (warp % Cfg::WN) * Cfg::WTN;
#pragma unroll
  for (int fm = 0; fm < Cfg::FM; ++fm)
#pragma unroll
    for (int fn = 0; fn < Cfg::FN; ++fn) {
      const int m = warp_m0 + fm * 8 + (lane >> 2);
      const int n = warp_n0 + fn * 8 + 2 * (lane & 3);
      f(m, n, acc[fm][fn][0], acc[fm][fn][1]);
    }
}

}  // namespace rijk
