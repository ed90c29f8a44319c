// CTA-level FP64 tensor-core (DMMA, mma.m8n8k4.f64) contraction over 32x32
// operand slots staged by bulk copies, with a dedicated producer warp.
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
//   kvalid(kt) is the number of k columns of step kt that count; the slot's
//   columns beyond it are ignored (skipped k4 steps, and zeros in place of the
//   slot's contents in a partial k4 step), so they may hold anything finite
//   or not.
//
// Warp roles: warps 0 .. WM*WN-1 compute, the last warp produces.  The producer
// waits until a stage is released (empty mbarrier, one arrival per consumer
// warp), writes the stage's orientation flags, arms the full mbarrier with the
// stage's byte count and issues one 256-byte cp.async.bulk per slot column (one
// per lane) into a slot with leading dimension 36 doubles (36 = 4 mod 16 makes
// the m8n8k4 fragment loads bank-conflict free in both orientations).
// Consumers wait on full, run the DMMAs, and release the stage.  No CTA-wide
// barrier runs inside the k-loop; every wait is bounded.
#pragma once
#include "rijk_common.cuh"

namespace rijk {

struct SlotSrc {
  const double* ptr;
  int64_t ld;
  int trans;
};

template <int MT_, int NT_, int WM_, int WN_, int STAGES_, bool CPASYNC_ = false>
struct DmmaCfg {
  static constexpr int MT = MT_, NT = NT_, WM = WM_, WN = WN_, STAGES = STAGES_;
  static constexpr bool CPASYNC = CPASYNC_;  // cp.async staging instead of the bulk-copy producer
  static constexpr int BM = MT * TS, BN = NT * TS;
  static constexpr int CWARPS = WM * WN;                  // consumer warps
  static constexpr int THREADS = (CWARPS + (CPASYNC ? 0 : 1)) * 32;  // + producer warp
  static constexpr int WTM = BM / WM, WTN = BN / WN;      // warp tile
  static constexpr int FM = WTM / 8, FN = WTN / 8;        // m8n8 fragments per warp
  static constexpr int SLOTS = MT + NT;
  static constexpr int STAGE_DOUBLES = SLOTS * SLOT_DOUBLES;
  static constexpr uint32_t STAGE_BYTES = SLOTS * TS * TS * 8;  // bytes landed per stage
  // slots | full[STAGES] | empty[STAGES] | flags[STAGES][SLOTS]
  static constexpr size_t BAR_OFFSET = (size_t)STAGES * STAGE_DOUBLES * 8;
  static constexpr size_t FLAG_OFFSET = BAR_OFFSET + 2 * STAGES * 8;
  static constexpr size_t SMEM_BYTES = FLAG_OFFSET + ((STAGES * SLOTS + 15) / 16) * 16;
  static_assert(BM % WM == 0 && BN % WN == 0, "warp grid");
  static_assert(WTM % 8 == 0 && WTN % 8 == 0, "warp tile");
  static_assert(TS % WTM == 0 || WTM % TS == 0, "warp rows vs slot");
  static_assert(TS % WTN == 0 || WTN % TS == 0, "warp cols vs slot");
};

struct DefaultKValid {
  __device__ int operator()(int) const { return TS; }
};

template <class Cfg>
struct DmmaSmem {
  double* slots;
  uint64_t* full;
  uint64_t* empty;
  uint8_t* flags;
  __device__ explicit DmmaSmem(void* base) {
    char* b = static_cast<char*>(base);
    slots = reinterpret_cast<double*>(b);
    full = reinterpret_cast<uint64_t*>(b + Cfg::BAR_OFFSET);
    empty = full + Cfg::STAGES;
    flags = reinterpret_cast<uint8_t*>(b + Cfg::FLAG_OFFSET);
  }
};

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Producer warp: stages every k-step.  Returns false on a timed-out wait.
template <class Cfg, class Sched>
__device__ __forceinline__ bool dmma_produce(const Sched& sc, int ktiles, DmmaSmem<Cfg>& sm, int* err) {
  const int lane = threadIdx.x & 31;
  for (int kt = 0; kt < ktiles; ++kt) {
    const int st = kt % Cfg::STAGES;
    if (kt >= Cfg::STAGES) {
      const uint32_t parity = (uint32_t)(((kt / Cfg::STAGES) - 1) & 1);
      if (!mbar_wait_bounded(&sm.empty[st], parity, err)) return false;
    }
    if (lane == 0) {
#pragma unroll 1
      for (int s = 0; s < Cfg::SLOTS; ++s) {
        const SlotSrc src = (s < Cfg::MT) ? sc.a(kt, s) : sc.b(kt, s - Cfg::MT);
        sm.flags[st * Cfg::SLOTS + s] = (uint8_t)src.trans;
      }
      mbar_arrive_expect_tx(&sm.full[st], Cfg::STAGE_BYTES);
    }
    __syncwarp();
    double* stage = sm.slots + st * Cfg::STAGE_DOUBLES;
#pragma unroll 1
    for (int s = 0; s < Cfg::SLOTS; ++s) {
      const SlotSrc src = (s < Cfg::MT) ? sc.a(kt, s) : sc.b(kt, s - Cfg::MT);
      const double* g = src.ptr ? src.ptr + (int64_t)lane * src.ld : g_zero_tile + lane * TS;
      bulk_g2s(stage + s * SLOT_DOUBLES + lane * SLD, g, TS * 8, &sm.full[st]);
    }
  }
  return true;
}

// Consumer warps: acc[fm][fn][2] holds, for this thread, the elements
// (m = warp_m0 + 8 fm + lane/4, n = warp_n0 + 8 fn + 2 (lane%4) + j).
// Fragments at or beyond (mvalid, nvalid) (CTA-local) are known to be zero
// and are skipped.  Returns false if a stage wait timed out.
template <class Cfg, class KValid>
__device__ __forceinline__ bool dmma_consume(int ktiles, DmmaSmem<Cfg>& sm, double (&acc)[Cfg::FM][Cfg::FN][2],
                                             int mvalid, int nvalid, const KValid& kvalid, int* err) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int warp_m0 = (warp / Cfg::WN) * Cfg::WTM;
  const int warp_n0 = (warp % Cfg::WN) * Cfg::WTN;
  const int fm_lim = max(0, min(Cfg::FM, (mvalid - warp_m0 + 7) / 8));
  const int fn_lim = max(0, min(Cfg::FN, (nvalid - warp_n0 + 7) / 8));
  const bool idle = fm_lim == 0 || fn_lim == 0;
  for (int kt = 0; kt < ktiles; ++kt) {
    const int st = kt % Cfg::STAGES;
    const uint32_t parity = (uint32_t)((kt / Cfg::STAGES) & 1);
    if (!mbar_wait_bounded(&sm.full[st], parity, err)) return false;
    if (!idle) {
      const double* sbase = sm.slots + st * Cfg::STAGE_DOUBLES;
      const uint8_t* fl = sm.flags + st * Cfg::SLOTS;
      // One (base, m/n stride, k stride) per slot this warp touches: fragment
      // fm lies in relative slot fm / FPS at row (fm % FPS) * 8 inside it.
      constexpr int APS = Cfg::WTM >= TS ? Cfg::WTM / TS : 1;  // A slots per warp
      constexpr int BPS = Cfg::WTN >= TS ? Cfg::WTN / TS : 1;  // B slots per warp
      constexpr int FPA = Cfg::FM / APS, FPB = Cfg::FN / BPS;  // fragments per slot
      int abase[APS], amst[APS], akst[APS], bbase[BPS], bnst[BPS], bkst[BPS];
#pragma unroll
      for (int j = 0; j < APS; ++j) {
        const int m = warp_m0 + j * TS;
        const int slot = m / TS, r = m % TS + (lane >> 2);
        const int tr = fl[slot];
        amst[j] = tr ? SLD : 1;
        akst[j] = tr ? 1 : SLD;
        abase[j] = slot * SLOT_DOUBLES + r * amst[j] + (lane & 3) * akst[j];
      }
#pragma unroll
      for (int j = 0; j < BPS; ++j) {
        const int c0 = warp_n0 + j * TS;
        const int slot = c0 / TS, c = c0 % TS + (lane >> 2);
        const int tr = fl[Cfg::MT + slot];
        bnst[j] = tr ? 1 : SLD;
        bkst[j] = tr ? SLD : 1;
        bbase[j] = (Cfg::MT + slot) * SLOT_DOUBLES + c * bnst[j] + (lane & 3) * bkst[j];
      }
      const int kvl = kvalid(kt);
      const int kk_lim = (kvl + 3) / 4;
      if (kvl == TS && fm_lim == Cfg::FM && fn_lim == Cfg::FN) {
        // Common case: straight-line code, so the compiler can load the
        // fragments of step kk+1 while the DMMAs of step kk issue.
#pragma unroll
        for (int kk = 0; kk < TS / 4; ++kk) {
          double af[Cfg::FM], bf[Cfg::FN];
#pragma unroll
          for (int fm = 0; fm < Cfg::FM; ++fm) {
            const int j = fm / FPA, i = fm % FPA;
            af[fm] = sbase[abase[j] + (i * 8) * amst[j] + (kk * 4) * akst[j]];
          }
#pragma unroll
          for (int fn = 0; fn < Cfg::FN; ++fn) {
            const int j = fn / FPB, i = fn % FPB;
            bf[fn] = sbase[bbase[j] + (i * 8) * bnst[j] + (kk * 4) * bkst[j]];
          }
#pragma unroll
          for (int fm = 0; fm < Cfg::FM; ++fm)
#pragma unroll
            for (int fn = 0; fn < Cfg::FN; ++fn) dmma_m8n8k4(acc[fm][fn][0], acc[fm][fn][1], af[fm], bf[fn]);
        }
      } else {
        // Edge tiles: skip the k4 steps and fragments that only hold padding;
        // k columns at or beyond kvalid of the last k4 step read as zero (a
        // slot may hold other data there, not only zero padding).
#pragma unroll 1
        for (int kk = 0; kk < kk_lim; ++kk) {
          double af[Cfg::FM], bf[Cfg::FN];
          const bool kin = kk * 4 + (lane & 3) < kvl;
#pragma unroll
          for (int fm = 0; fm < Cfg::FM; ++fm) {
            const int j = fm / FPA, i = fm % FPA;
            af[fm] = (fm < fm_lim && kin) ? sbase[abase[j] + (i * 8) * amst[j] + (kk * 4) * akst[j]] : 0.0;
          }
#pragma unroll
          for (int fn = 0; fn < Cfg::FN; ++fn) {
            const int j = fn / FPB, i = fn % FPB;
            bf[fn] = (fn < fn_lim && kin) ? sbase[bbase[j] + (i * 8) * bnst[j] + (kk * 4) * bkst[j]] : 0.0;
          }
#pragma unroll
          for (int fm = 0; fm < Cfg::FM; ++fm)
#pragma unroll
            for (int fn = 0; fn < Cfg::FN; ++fn)
              if (fm < fm_lim && fn < fn_lim) dmma_m8n8k4(acc[fm][fn][0], acc[fm][fn][1], af[fm], bf[fn]);
        }
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&sm.empty[st]);
  }
  return true;
}

// ---------------------------------------------------------------------------
// Remainder columns (cp.async scheme, 4-warp 64 x 64 CTAs).  When the B
// operand's valid columns end XF * 8 or fewer columns past a multiple of 64,
// the CTAs of the last full column block also compute those columns, so that
// no CTA streams the A operand for a nearly empty output tile.  Per k-step the
// 32 x (8 XF) block of B is staged into the padding words of the stage's slots
// (element (k, n) of it at slot n / 4, column 4 (k / 4) + n % 4, word 32 + k % 4:
// 16-byte runs of two k, and conflict-free fragment loads), and warp (wm, wn)
// multiplies it by the A fragments of rows wm * 32 + wn * 16 .. + 15, which it
// holds already: two extra DMMAs per k4 step and extra fragment.
// ---------------------------------------------------------------------------
template <int XF>
struct ExtraCols {
  double acc[2][XF > 0 ? XF : 1][2];  // rows (wn * 2 + e) * 8 + lane / 4 of the warp tile
  bool on = false;                    // this CTA computes the remainder columns
};

// Per-lane offset (in doubles, inside a stage) of extra fragment j for k4 step 0.
__device__ __forceinline__ int extra_off(int j, int lane) {
  const int l4 = lane >> 2;
  return (2 * j + (l4 >> 2)) * SLOT_DOUBLES + (l4 & 3) * SLD + 32 + (lane & 3);
}

template <int XF>
__device__ __forceinline__ void extra_k4(const double* __restrict__ sbase, int kk, int lane, double a0, double a1,
                                         bool v0, bool v1, bool kin, ExtraCols<XF>& x) {
#pragma unroll
  for (int j = 0; j < XF; ++j) {
    const double b = kin ? sbase[extra_off(j, lane) + kk * 4 * SLD] : 0.0;
    if (v0) dmma_m8n8k4(x.acc[0][j][0], x.acc[0][j][1], a0, b);
    if (v1) dmma_m8n8k4(x.acc[1][j][0], x.acc[1][j][1], a1, b);
  }
}

// ---------------------------------------------------------------------------
// Second staging scheme, selected per CTA shape (Cfg::STAGES < 0 never; the
// template flag below): every thread copies 16-byte chunks with cp.async into
// the same padded slots, cp.async groups track the stages, one CTA barrier per
// k-step protects stage reuse.  No producer warp: all WM*WN warps compute, the
// extra warp of Cfg::THREADS only helps copying.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(smem_dst)), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

template <class Cfg, int XF = 0, class Sched>
__device__ __forceinline__ void cpa_issue_stage(const Sched& sc, int kt, double* stage, uint8_t* flags,
                                                bool extra = false) {
  // 512 16-byte chunks per slot: chunk = column c (0..31) x row pair r2 (0..15).
  // Thread t copies chunks t + THREADS j: with THREADS a multiple of 16 they
  // share the row pair t % 16 and step THREADS / 16 columns, so one base
  // address per slot and constant strides cover them.
  constexpr int CHUNKS = 512;
  static_assert(Cfg::THREADS % 16 == 0 && CHUNKS % Cfg::THREADS == 0, "chunk split");
  constexpr int NJ = CHUNKS / Cfg::THREADS, CSTEP = Cfg::THREADS / 16;
  const int c0 = threadIdx.x >> 4, r = (threadIdx.x & 15) * 2;
#pragma unroll
  for (int s = 0; s < Cfg::SLOTS; ++s) {
    const SlotSrc src = (s < Cfg::MT) ? sc.a(kt, s) : sc.b(kt, s - Cfg::MT);
    if (threadIdx.x == 0) flags[s] = (uint8_t)src.trans;
    const double* base = src.ptr ? src.ptr : g_zero_tile;
    const int64_t ld = src.ptr ? src.ld : TS;
    const double* g = base + (int64_t)c0 * ld + r;
    const int64_t gstep = (int64_t)CSTEP * ld;
    double* d = stage + s * SLOT_DOUBLES + c0 * SLD + r;
#pragma unroll
    for (int j = 0; j < NJ; ++j) cp_async16(d + j * CSTEP * SLD, g + j * gstep);
  }
  if constexpr (XF > 0) {
    static_assert(Cfg::THREADS == 128 && 2 * XF <= Cfg::SLOTS, "remainder staging");
    if (extra) {
      // 16-byte chunk id = column nn (0 .. 8 XF - 1) x row pair r2 (k = 2 r2, 2 r2 + 1)
      const SlotSrc xs = sc.x(kt);
#pragma unroll
      for (int i = 0; i < XF; ++i) {
        const int id = threadIdx.x + 128 * i;
        const int nn = id >> 4, r2 = id & 15;
        const double* g = xs.ptr + (int64_t)nn * xs.ld + 2 * r2;
        double* d = stage + (nn >> 2) * SLOT_DOUBLES + (4 * (r2 >> 1) + (nn & 3)) * SLD + 32 + 2 * (r2 & 1);
        cp_async16(d, g);
      }
    }
  }
}

// One full k-tile (32 k) of a warp whose A slots (consecutive, from slot_a) all
// have orientation TA and whose B slots (consecutive, from slot_b) all have
// orientation TB: every fragment address is the warp's base plus an immediate.
// PARTIAL: only fragments fm < fm_lim, fn < fn_lim are loaded and multiplied
// (the warp's tile straddles the valid rows or columns); the k-tile is full.
template <class Cfg, bool TA, bool TB, bool PARTIAL = false, int XF = 0>
__device__ __forceinline__ void dmma_ktile_fixed(const double* __restrict__ sbase, int slot_a, int slot_b, int lane,
                                                 double (&acc)[Cfg::FM][Cfg::FN][2], int fm_lim = Cfg::FM,
                                                 int fn_lim = Cfg::FN, ExtraCols<XF>* x = nullptr, int wn = 0) {
  constexpr int AMST = TA ? SLD : 1, AKST = TA ? 1 : SLD;
  constexpr int BNST = TB ? 1 : SLD, BKST = TB ? SLD : 1;
  constexpr int APS = Cfg::WTM >= TS ? Cfg::WTM / TS : 1;
  constexpr int BPS = Cfg::WTN >= TS ? Cfg::WTN / TS : 1;
  constexpr int FPA = Cfg::FM / APS, FPB = Cfg::FN / BPS;
  const double* sa = sbase + slot_a * SLOT_DOUBLES + (lane >> 2) * AMST + (lane & 3) * AKST;
  const double* sb = sbase + (Cfg::MT + slot_b) * SLOT_DOUBLES + (lane >> 2) * BNST + (lane & 3) * BKST;
#pragma unroll
  for (int kk = 0; kk < TS / 4; ++kk) {
    double af[Cfg::FM], bf[Cfg::FN];
#pragma unroll
    for (int fm = 0; fm < Cfg::FM; ++fm)
      if (!PARTIAL || fm < fm_lim) af[fm] = sa[(fm / FPA) * SLOT_DOUBLES + ((fm % FPA) * 8) * AMST + (kk * 4) * AKST];
#pragma unroll
    for (int fn = 0; fn < Cfg::FN; ++fn)
      if (!PARTIAL || fn < fn_lim) bf[fn] = sb[(fn / FPB) * SLOT_DOUBLES + ((fn % FPB) * 8) * BNST + (kk * 4) * BKST];
#pragma unroll
    for (int fm = 0; fm < Cfg::FM; ++fm)
#pragma unroll
      for (int fn = 0; fn < Cfg::FN; ++fn)
        if (!PARTIAL || (fm < fm_lim && fn < fn_lim)) dmma_m8n8k4(acc[fm][fn][0], acc[fm][fn][1], af[fm], bf[fn]);
    if constexpr (XF > 0) {
      if (x->on) {
        const double a0 = wn ? af[2] : af[0], a1 = wn ? af[3] : af[1];
        extra_k4<XF>(sbase, kk, lane, a0, a1, !PARTIAL || 2 * wn < fm_lim, !PARTIAL || 2 * wn + 1 < fm_lim, true,
                     *x);
      }
    }
  }
}

template <class Cfg, int XF = 0, class Sched, class KValid>
__device__ __forceinline__ bool dmma_mainloop_cpasync(const Sched& sc, int ktiles, void* smem_base,
                                                      double (&acc)[Cfg::FM][Cfg::FN][2], int mvalid, int nvalid,
                                                      const KValid& kvalid, ExtraCols<XF>* x = nullptr) {
  DmmaSmem<Cfg> sm(smem_base);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < Cfg::FM; ++i)
#pragma unroll
    for (int j = 0; j < Cfg::FN; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
  bool xon = false;
  if constexpr (XF > 0) {
    xon = x->on;
#pragma unroll
    for (int e = 0; e < 2; ++e)
#pragma unroll
      for (int j = 0; j < XF; ++j) x->acc[e][j][0] = x->acc[e][j][1] = 0.0;
  }
  constexpr int S = Cfg::STAGES;
#pragma unroll
  for (int s = 0; s < S - 1; ++s) {
    if (s < ktiles)
      cpa_issue_stage<Cfg, XF>(sc, s, sm.slots + s * Cfg::STAGE_DOUBLES, sm.flags + s * Cfg::SLOTS, xon);
    cp_async_commit();
  }
  const bool compute = warp < Cfg::CWARPS;
  const int warp_m0 = (warp / Cfg::WN) * Cfg::WTM;
  const int warp_n0 = (warp % Cfg::WN) * Cfg::WTN;
  const int fm_lim = compute ? max(0, min(Cfg::FM, (mvalid - warp_m0 + 7) / 8)) : 0;
  const int fn_lim = compute ? max(0, min(Cfg::FN, (nvalid - warp_n0 + 7) / 8)) : 0;
  const bool idle = fm_lim == 0 || fn_lim == 0;
  constexpr int APS = Cfg::WTM >= TS ? Cfg::WTM / TS : 1;
  constexpr int BPS = Cfg::WTN >= TS ? Cfg::WTN / TS : 1;
  constexpr int FPA = Cfg::FM / APS, FPB = Cfg::FN / BPS;
  for (int kt = 0; kt < ktiles; ++kt) {
    cp_async_wait<S - 2>();
    __syncthreads();  // stage kt landed for everyone; stage kt-1 is free
    {
      const int nk = kt + S - 1;
      const int ns = nk % S;
      if (nk < ktiles)
        cpa_issue_stage<Cfg, XF>(sc, nk, sm.slots + ns * Cfg::STAGE_DOUBLES, sm.flags + ns * Cfg::SLOTS, xon);
      cp_async_commit();
    }
    if (idle) continue;
    const int st = kt % S;
    const double* sbase = sm.slots + st * Cfg::STAGE_DOUBLES;
    const uint8_t* fl = sm.flags + st * Cfg::SLOTS;
    const int kvl = kvalid(kt);
    const int kk_lim = (kvl + 3) / 4;
    const bool full = kvl == TS && fm_lim == Cfg::FM && fn_lim == Cfg::FN;
    if constexpr (Cfg::WTM % TS == 0 && Cfg::WTN % TS == 0) {
      // the warp's A slots and B slots; orientations are warp-uniform per slot
      const int sa = warp_m0 / TS, sbs = warp_n0 / TS;
      const bool ta = fl[sa] != 0, tb = fl[Cfg::MT + sbs] != 0;
      bool uniform = true;
#pragma unroll
      for (int j = 1; j < APS; ++j) uniform = uniform && ((fl[sa + j] != 0) == ta);
#pragma unroll
      for (int j = 1; j < BPS; ++j) uniform = uniform && ((fl[Cfg::MT + sbs + j] != 0) == tb);
      const int wn = warp % Cfg::WN;
      if (full && uniform) {
        if (!ta && !tb)
          dmma_ktile_fixed<Cfg, false, false, false, XF>(sbase, sa, sbs, lane, acc, Cfg::FM, Cfg::FN, x, wn);
        else if (ta && !tb)
          dmma_ktile_fixed<Cfg, true, false, false, XF>(sbase, sa, sbs, lane, acc, Cfg::FM, Cfg::FN, x, wn);
        else if (!ta && tb)
          dmma_ktile_fixed<Cfg, false, true, false, XF>(sbase, sa, sbs, lane, acc, Cfg::FM, Cfg::FN, x, wn);
        else
          dmma_ktile_fixed<Cfg, true, true, false, XF>(sbase, sa, sbs, lane, acc, Cfg::FM, Cfg::FN, x, wn);
        continue;
      }
      if constexpr (Cfg::THREADS == 128 && Cfg::FM * Cfg::FN == 16 && 3 * Cfg::SMEM_BYTES <= 227 * 1024) {
        if (kvl == TS && uniform) {
          // full k-tile, warp tile straddling the valid rows or columns (the
          // 4-warp 64x64 shapes only: the variant costs registers)
          if (!ta && !tb)
            dmma_ktile_fixed<Cfg, false, false, true, XF>(sbase, sa, sbs, lane, acc, fm_lim, fn_lim, x, wn);
          else if (ta && !tb)
            dmma_ktile_fixed<Cfg, true, false, true, XF>(sbase, sa, sbs, lane, acc, fm_lim, fn_lim, x, wn);
          else if (!ta && tb)
            dmma_ktile_fixed<Cfg, false, true, true, XF>(sbase, sa, sbs, lane, acc, fm_lim, fn_lim, x, wn);
          else
            dmma_ktile_fixed<Cfg, true, true, true, XF>(sbase, sa, sbs, lane, acc, fm_lim, fn_lim, x, wn);
          continue;
        }
      }
    }
    // general path: per-slot fragment bases and strides from the orientation flags
    int abase[APS], amst[APS], akst[APS], bbase[BPS], bnst[BPS], bkst[BPS];
#pragma unroll
    for (int j = 0; j < APS; ++j) {
      const int m = warp_m0 + j * TS;
      const int slot = m / TS, r = m % TS + (lane >> 2);
      const int tr = fl[slot];
      amst[j] = tr ? SLD : 1;
      akst[j] = tr ? 1 : SLD;
      abase[j] = slot * SLOT_DOUBLES + r * amst[j] + (lane & 3) * akst[j];
    }
#pragma unroll
    for (int j = 0; j < BPS; ++j) {
      const int c0 = warp_n0 + j * TS;
      const int slot = c0 / TS, c = c0 % TS + (lane >> 2);
      const int tr = fl[Cfg::MT + slot];
      bnst[j] = tr ? 1 : SLD;
      bkst[j] = tr ? SLD : 1;
      bbase[j] = (Cfg::MT + slot) * SLOT_DOUBLES + c * bnst[j] + (lane & 3) * bkst[j];
    }
    if (full) {
#pragma unroll
      for (int kk = 0; kk < TS / 4; ++kk) {
        double af[Cfg::FM], bf[Cfg::FN];
#pragma unroll
        for (int fm = 0; fm < Cfg::FM; ++fm) {
          const int j = fm / FPA, i = fm % FPA;
          af[fm] = sbase[abase[j] + (i * 8) * amst[j] + (kk * 4) * akst[j]];
        }
#pragma unroll
        for (int fn = 0; fn < Cfg::FN; ++fn) {
          const int j = fn / FPB, i = fn % FPB;
          bf[fn] = sbase[bbase[j] + (i * 8) * bnst[j] + (kk * 4) * bkst[j]];
        }
#pragma unroll
        for (int fm = 0; fm < Cfg::FM; ++fm)
#pragma unroll
          for (int fn = 0; fn < Cfg::FN; ++fn) dmma_m8n8k4(acc[fm][fn][0], acc[fm][fn][1], af[fm], bf[fn]);
        if constexpr (XF > 0) {
          if (xon) {
            const int wn = warp % Cfg::WN;
            extra_k4<XF>(sbase, kk, lane, wn ? af[2] : af[0], wn ? af[3] : af[1], true, true, true, *x);
          }
        }
      }
    } else {
      // edge tile: as in dmma_consume, k at or beyond kvalid reads as zero
#pragma unroll 1
      for (int kk = 0; kk < kk_lim; ++kk) {
        double af[Cfg::FM], bf[Cfg::FN];
        const bool kin = kk * 4 + (lane & 3) < kvl;
#pragma unroll
        for (int fm = 0; fm < Cfg::FM; ++fm) {
          const int j = fm / FPA, i = fm % FPA;
          af[fm] = (fm < fm_lim && kin) ? sbase[abase[j] + (i * 8) * amst[j] + (kk * 4) * akst[j]] : 0.0;
        }
#pragma unroll
        for (int fn = 0; fn < Cfg::FN; ++fn) {
          const int j = fn / FPB, i = fn % FPB;
          bf[fn] = (fn < fn_lim && kin) ? sbase[bbase[j] + (i * 8) * bnst[j] + (kk * 4) * bkst[j]] : 0.0;
        }
#pragma unroll
        for (int fm = 0; fm < Cfg::FM; ++fm)
#pragma unroll
          for (int fn = 0; fn < Cfg::FN; ++fn)
            if (fm < fm_lim && fn < fn_lim) dmma_m8n8k4(acc[fm][fn][0], acc[fm][fn][1], af[fm], bf[fn]);
        if constexpr (XF > 0) {
          if (xon) {
            const int wn = warp % Cfg::WN;
            extra_k4<XF>(sbase, kk, lane, wn ? af[2] : af[0], wn ? af[3] : af[1], 2 * wn < fm_lim,
                         2 * wn + 1 < fm_lim, kin, *x);
          }
        }
      }
    }
  }
  cp_async_wait<0>();
  return compute;
}

// Whole CTA: set up the barriers, split into producer and consumers.  Only
// consumer threads return true (and hold results); the producer returns false.
// Cfg::CPASYNC selects the cp.async staging above instead.
template <class Cfg, class Sched, class KValid = DefaultKValid, int XF = 0>
__device__ __forceinline__ bool dmma_mainloop(const Sched& sc, int ktiles, void* smem_base,
                                              double (&acc)[Cfg::FM][Cfg::FN][2], int* err, int mvalid = 1 << 30,
                                              int nvalid = 1 << 30, const KValid& kvalid = KValid(),
                                              ExtraCols<XF>* x = nullptr) {
  if constexpr (Cfg::CPASYNC) {
    (void)err;
    return dmma_mainloop_cpasync<Cfg, XF>(sc, ktiles, smem_base, acc, mvalid, nvalid, kvalid, x);
  } else {
    static_assert(XF == 0, "remainder columns need the cp.async scheme");
  }
  DmmaSmem<Cfg> sm(smem_base);
  const int warp = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < Cfg::FM; ++i)
#pragma unroll
    for (int j = 0; j < Cfg::FN; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
  if (threadIdx.x == 0) {
    for (int s = 0; s < Cfg::STAGES; ++s) {
      mbar_init(&sm.full[s], 1);
      mbar_init(&sm.empty[s], Cfg::CWARPS);
    }
    mbar_fence_init();
  }
  __syncthreads();
  if (warp == Cfg::CWARPS) {
    dmma_produce<Cfg>(sc, ktiles, sm, err);
    return false;
  }
  return dmma_consume<Cfg>(ktiles, sm, acc, mvalid, nvalid, kvalid, err);
}

// Visits every accumulator element of this consumer thread with its CTA-local (m, n).
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
