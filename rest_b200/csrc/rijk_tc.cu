// Split-precision exchange build on the 5th-generation tensor cores (tcgen05).
//
// Every FP64 operand x is carried as two BF16 numbers, hi = bf16(x) and
// lo = bf16(x - hi), so that x = hi + lo to about 2^-17 relative.  A product
// a b is formed as a_hi b_hi + a_hi b_lo + a_lo b_hi (three tcgen05.mma of kind
// f16 accumulating into one FP32 accumulator in tensor memory); the dropped
// a_lo b_lo term is below 2^-16 relative.  The two contractions of the
// exchange build in the occupied-orbital form of REST's vk_upper_with_ri_v_sync
// (src/scf_io/mod.rs:2758-2834),
//     X_P = B_P V          (half-transform)
//     K   = sum_P X_P S X_P^T  (rank update, S = diag(+1.. , -1..))
// run this way; with V the occupied orbitals scaled by sqrt(occ) it is the
// plain exchange matrix, and with V the signed square-root factor of a
// density difference it is the exchange matrix of that difference (the
// incremental builds of the mixed-precision SCF).
//
// Operands live in HBM in the canonical K-major layout of tcgen05 without
// swizzle: 8-row x 16-byte "core matrices" (8 x 8 BF16), core matrix (r8, k8)
// of a (R x 64) block at byte offset (k8 * R/8 + r8) * 128, row r%8 of it at
// (r%8) * 16.  The descriptor's stride between core matrices along the rows is
// then 128 bytes (SBO) and along K is R/8 * 128 bytes (LBO).  Each pipeline
// stage is a handful of contiguous bulk copies (TMA engine, no multicast).
//
// The split tensor keeps only the upper 128 x 128 squares (I <= J) of each
// symmetric B_P, as the FP64 tensor keeps only its upper 32 x 32 tiles.  A
// square below the diagonal is read from its mirror: the same core matrices,
// seen with the rows and K exchanged, are the MN-major canonical layout (each
// core matrix is 8 K-rows of 16 bytes along M), which the MMA takes with the
// A-major bit of the instruction descriptor set.
//
// Kernel forms (make_tc_geom chooses): one SM per tile, or a cluster of two
// SMs running M = 256 MMAs (cta_group::2) whose copies complete on the first
// CTA's barrier.  The paired half-transform runs N = the used columns rounded
// up to 16 (V laid out at that width, in two halves); the rank updates skip the
// k-steps of X's padding columns.  J's scalars w_P = <V, X_P> can come out of
// the half-transform's epilogue (a separate instantiation).
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <mutex>

#include "rijk_common.cuh"
#include "rijk_internal.h"

namespace rijk {

namespace {

constexpr int TC_M = 128;   // rows per UMMA / per operand block
constexpr int TC_KB = 64;   // K per pipeline stage (4 UMMA k-steps of 16)
constexpr int BLOCK_ELEMS = TC_M * TC_KB;          // 8192 BF16 = 16 KB
constexpr uint32_t BLOCK_BYTES = BLOCK_ELEMS * 2;  // 16384

inline int64_t cdiv_t(int64_t a, int64_t b) { return (a + b - 1) / b; }

// element offset of (r, k) inside an (R x 64) K-major core-matrix block
__host__ __device__ __forceinline__ int core_off(int r, int k, int R) {
  return ((k >> 3) * (R >> 3) + (r >> 3)) * 64 + (r & 7) * 8 + (k & 7);
}

// ---- tcgen05 helpers -------------------------------------------------------
__device__ __forceinline__ uint64_t smem_desc(const void* p, uint32_t lbo, uint32_t sbo) {
  const uint64_t a = smem_u32(p);
  uint64_t d = 0;
  d |= (a >> 4) & 0x3FFFull;                   // start address
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;  // leading (K-direction) byte offset
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;  // stride (row-direction) byte offset
  d |= 1ull << 46;                             // descriptor version for tcgen05
  // base offset 0, lbo mode 0, layout type 0 (no swizzle)
  return d;
}

// kind::f16 instruction descriptor: BF16 A and B, FP32 D, both K-major.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, bool neg_b, bool a_mn_major = false) {
  return (1u << 4)                        // D format F32
         | (1u << 7)                      // A format BF16
         | (1u << 10)                     // B format BF16
         | ((neg_b ? 1u : 0u) << 14)      // negate B
         | ((a_mn_major ? 1u : 0u) << 15)  // A is MN-major (else K-major)
         | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void tc_mma(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                       uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tc_alloc(uint32_t* dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst_smem)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tc_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 32 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tc_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// One tiled tensor copy (TMA, this GPU's memory, no multicast) of a 3-D box.
__device__ __forceinline__ void tma_load_3d(void* smem_dst, const CUtensorMap* map, int x, int y, int z,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_u32(smem_dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void split_bf16(double x, __nv_bfloat16& hi, __nv_bfloat16& lo) {
  hi = __double2bfloat16(x);
  lo = __double2bfloat16(x - (double)__bfloat162float(hi));
}

// The same split of eight FP32 accumulator values, in FP32: bf16(v) rounds
// exactly as bf16((double)v) does, and v - hi is exact in FP32 (hi agrees with v
// in its leading bits), so hi and lo equal split_bf16((double)v) bit for bit
// while the conversions run as packed FP32 -> BF16 pairs instead of FP64.
__device__ __forceinline__ void split_bf16x8(const float* v, uint4& hi, uint4& lo) {
  __nv_bfloat162 h[4], l[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    h[q] = __floats2bfloat162_rn(v[2 * q], v[2 * q + 1]);
    const float2 hf = __bfloat1622float2(h[q]);
    l[q] = __floats2bfloat162_rn(v[2 * q] - hf.x, v[2 * q + 1] - hf.y);
  }
  hi = *reinterpret_cast<const uint4*>(h);
  lo = *reinterpret_cast<const uint4*>(l);
}

// ---- layout producers --------------------------------------------------------
// Square (I <= J) of B_P is number J (J + 1) / 2 + I, two (128 x 64) K-major
// blocks (K halves j = 0, 1): rows mu = 128 I + r, K kappa = 128 J + 64 j + k.
__host__ __device__ __forceinline__ int64_t sq_index(int64_t I, int64_t J) { return J * (J + 1) / 2 + I; }

// Bs[P][square][j] (hi and lo planes) from the FP64 tile-packed tensor; the
// diagonal squares hold both triangles, entries beyond n are zero.
__global__ void __launch_bounds__(256) k_split_tensor(const double* __restrict__ B, int64_t ldB, int64_t n, int nmb,
                                                      int64_t p0, int64_t np, __nv_bfloat16* __restrict__ hi,
                                                      __nv_bfloat16* __restrict__ lo) {
  const int64_t nsq = (int64_t)nmb * (nmb + 1) / 2;
  const int64_t per_p = nsq * 2 * BLOCK_ELEMS;
  const int64_t total = np * per_p;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t pl = e / per_p;
    const int64_t rem = e - pl * per_p;
    const int64_t blk = rem / BLOCK_ELEMS;
    const int o = (int)(rem - blk * BLOCK_ELEMS);
    const int64_t sq = blk >> 1;
    const int j = (int)(blk & 1);
    int64_t J = (int64_t)((sqrt(8.0 * (double)sq + 1.0) - 1.0) * 0.5);
    while (J * (J + 1) / 2 > sq) --J;
    while ((J + 1) * (J + 2) / 2 <= sq) ++J;
    const int64_t I = sq - J * (J + 1) / 2;
    // invert core_off for R = 128
    const int within = o & 63, core = o >> 6;
    const int r = ((core % (TC_M / 8)) << 3) | (within >> 3);
    const int k = ((core / (TC_M / 8)) << 3) | (within & 7);
    const int64_t mu = I * TC_M + r, ka = J * TC_M + j * TC_KB + k;
    double x = 0.0;
    if (mu < n && ka < n) {
      const int64_t ti = mu / TS, tj = ka / TS;
      const double* Bp = B + (p0 + pl) * ldB;
      x = ti <= tj ? Bp[tile_pair_index(ti, tj) * TILE_ELEMS + (mu % TS) + TS * (ka % TS)]
                   : Bp[tile_pair_index(tj, ti) * TILE_ELEMS + (ka % TS) + TS * (mu % TS)];
    }
    __nv_bfloat16 h, l;
    split_bf16(x, h, l);
    hi[e] = h;
    lo[e] = l;
  }
}

// Vs[kb] (hi, lo): columns of V (n x ncols, column-major, ld) as the B operand
// of the half-transform, N = npad rows (columns of V), K = kappa.  With
// halves = 2 each K block is two (npad/2 x 64) K-major blocks, columns
// [0, npad/2) then [npad/2, npad): the two CTAs of a paired launch copy one each.
__global__ void __launch_bounds__(256) k_split_cols(const double* __restrict__ V, int64_t ldv, int64_t n,
                                                    int ncols, int npad, int nkb, int halves,
                                                    __nv_bfloat16* __restrict__ hi, __nv_bfloat16* __restrict__ lo) {
  const int64_t per_kb = (int64_t)npad * TC_KB;
  const int64_t total = per_kb * nkb;
  const int rows = npad / halves;  // rows of one K-major block
  const int64_t per_half = (int64_t)rows * TC_KB;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int kb = (int)(e / per_kb);
    const int oo = (int)(e - kb * per_kb);
    const int half = (int)(oo / per_half), o = (int)(oo - half * per_half);
    const int within = o & 63, core = o >> 6;
    const int i = half * rows + (((core % (rows / 8)) << 3) | (within >> 3));
    const int k = ((core / (rows / 8)) << 3) | (within & 7);
    const int64_t ka = (int64_t)kb * TC_KB + k;
    const double x = (i < ncols && ka < n) ? V[ka + ldv * i] : 0.0;
    __nv_bfloat16 h, l;
    split_bf16(x, h, l);
    hi[e] = h;
    lo[e] = l;
  }
}

// ---- persistent half-transform ---------------------------------------------------
// One CTA per SM walks tiles (P, 128-row block) with stride gridDim.x.  Two FP32
// accumulators in tensor memory (2 x NPAD columns) alternate between tiles, so
// the epilogue of tile i (4 warps, TMEM -> BF16 split -> HBM) overlaps the MMAs
// of tile i+1.  Warp 0: producer, warp 1: MMA issuer, warps 2..5: epilogue
// (warp w reads TMEM lanes 32 (w % 4) .. 32 (w % 4) + 31).
// KS: K per pipeline stage (64, or 32 for twice as many stages in the same
// shared memory, i.e. a deeper look-ahead for the same bytes in flight).
template <int NPAD, int KS = TC_KB>
struct HalfTcP {
  static_assert(KS == 64 || KS == 32, "stage K");
  static constexpr uint32_t A_BYTES = TC_M * KS * 2;  // one plane's A tile per stage
  static constexpr uint32_t V_BYTES = NPAD * KS * 2;
  static constexpr uint32_t STAGE_BYTES = 2 * A_BYTES + 2 * V_BYTES;
  static constexpr size_t SMEM = 232448;  // whole per-CTA budget (one CTA per SM)
  static constexpr int STAGES = (int)((SMEM - 1024 - 256) / STAGE_BYTES) > 8 ? 8
                                                                            : (int)((SMEM - 1024 - 256) / STAGE_BYTES);
  static_assert(STAGES >= 2 && (size_t)STAGES * STAGE_BYTES + 1024 + 256 <= SMEM, "stage budget");
};

// K step kb of row block mb reads square (mb, kb / 2) when mb <= kb / 2, else
// the mirror square (kb / 2, mb) seen MN-major: its 16 groups of 8 rows mu
// (one 1 KB run of the 8 core matrices of K half kb % 2 each) land at 1 KB
// strides, so the MN-major descriptor has 128-byte K-group and 1 KB M-group
// strides.
// With use_tm the mirrored half is one tiled tensor copy per plane: the plane
// seen as rows of 1024 BF16 (one group of 8 rows of a square, all 16 of its K
// groups), as dims {256, 4, rows}; the box {256, 2, 16} at (0, 2 j, 16 square)
// is K half j of the square's 16 row groups, landing at 1 KB per group.
// WJ: with J's epilogue (wpart non-null).  A separate instantiation, because
// its loop over the accumulator's columns indexes v at run time, which puts v
// in local memory; without J, v stays in registers.  The J loop is unrolled 32
// (all its loads of V in flight at once) with its run-time bound: measured on
// the paired kernel at n = 1200, the fused split J/K build took 37.4 / 21.6 /
// 19.0 / 18.7 / 18.0 ms at unroll 1 / 4 / 8 / 16 / 32, while a version with the
// bound as a per-iteration predicate and four FMA chains took three times as
// long as unroll 8.
template <int NPAD, int KS, bool WJ>
__global__ void __launch_bounds__(192, 1)
    k_half_tc_persistent(const __nv_bfloat16* __restrict__ Bhi, const __nv_bfloat16* __restrict__ Blo, int nmb,
                         int nkb, const __nv_bfloat16* __restrict__ Vhi, const __nv_bfloat16* __restrict__ Vlo,
                         int nib, int64_t ntiles, __nv_bfloat16* __restrict__ Xhi, __nv_bfloat16* __restrict__ Xlo,
                         int* err, const __grid_constant__ CUtensorMap tm_hi, const __grid_constant__ CUtensorMap tm_lo,
                         int use_tm, int64_t p0, const double* __restrict__ Vd, int64_t ldv, int ncols, int nrows,
                         double* __restrict__ wpart) {
  const int64_t nsq = (int64_t)nmb * (nmb + 1) / 2;
  using C = HalfTcP<NPAD, KS>;
  constexpr int S = C::STAGES;
  constexpr int QK = TC_KB / KS;  // stages per 64-wide K block
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + S * C::STAGE_BYTES);
  uint64_t* empty = full + S;
  uint64_t* acc_full = empty + S;    // [2]
  uint64_t* acc_empty = acc_full + 2;  // [2]
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(acc_empty + 2);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t G = gridDim.x;
  const int64_t my_tiles = ntiles > blockIdx.x ? (ntiles - blockIdx.x + G - 1) / G : 0;

  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&acc_full[b], 1);
      mbar_init(&acc_empty[b], 4);
    }
    mbar_fence_init();
  }
  if (warp == 0) tc_alloc(tmem_slot, 2 * NPAD);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  bool ok = true;

  if (warp == 0) {
    // The whole warp stages: lane 0 waits for the slot and arms the barrier,
    // then the copies are issued one per lane (a mirrored square is 32 runs
    // of 1 KB, hi and lo).
    const int nks = nkb * QK;  // stages per tile
    for (int64_t lt = 0; lt < my_tiles && ok; ++lt) {
      const int64_t tile = blockIdx.x + lt * G;
      const int64_t pl = tile / nmb;
      const int mb = (int)(tile % nmb);
      for (int ksg = 0; ksg < nks && ok; ++ksg) {
        const int64_t g = lt * nks + ksg;
        const int s = (int)(g % S);
        if (lane == 0 && g >= S) ok = mbar_wait_bounded(&empty[s], (uint32_t)(((g / S) - 1) & 1), err);
        ok = __shfl_sync(0xffffffffu, ok, 0);
        if (!ok) break;
        uint8_t* st = smem + s * C::STAGE_BYTES;
        if (lane == 0) mbar_arrive_expect_tx(&full[s], C::STAGE_BYTES);
        __syncwarp();
        const int kb = ksg / QK, q = ksg % QK;  // 64-wide K block, and this stage's part of it
        const int Kb = kb >> 1, j = kb & 1;
        if (mb <= Kb) {
          // stage q of a K-major block: K groups [8 q KS/64 ..) are its first / second half
          const int64_t boff = ((pl * nsq + sq_index(mb, Kb)) * 2 + j) * BLOCK_ELEMS + (int64_t)q * (TC_M * KS);
          if (lane == 0) bulk_g2s(st, Bhi + boff, C::A_BYTES, &full[s]);
          if (lane == 1) bulk_g2s(st + C::A_BYTES, Blo + boff, C::A_BYTES, &full[s]);
        } else if (use_tm) {
          // mirrored square: K rows [64 j + KS q, +KS) of it are the 512-element
          // pieces y = (64 j + KS q) / 32 .. of each of its 16 K-group rows
          const int z = (int)(((p0 + pl) * nsq + sq_index(Kb, mb)) * 16);
          const int y = (64 * j + KS * q) / 32;
          if (lane == 0) tma_load_3d(st, &tm_hi, 0, y, z, &full[s]);
          if (lane == 1) tma_load_3d(st + C::A_BYTES, &tm_lo, 0, y, z, &full[s]);
        } else if (KS == TC_KB) {
          const int64_t sbase = (pl * nsq + sq_index(Kb, mb)) * 2 * BLOCK_ELEMS + (int64_t)(8 * j) * 64;
          const int run = lane & 15;  // M group of 8 rows: run `run` of 1 KB
          const int64_t src = sbase + (int64_t)(run >> 3) * BLOCK_ELEMS + (int64_t)((run & 7) * (TC_M / 8)) * 64;
          if (lane < 16)
            bulk_g2s(st + run * 1024, Bhi + src, 1024, &full[s]);
          else
            bulk_g2s(st + BLOCK_BYTES + run * 1024, Blo + src, 1024, &full[s]);
        }
        // V stage: K groups [KS q / 8, +KS / 8) of block kb, contiguous
        const int64_t voff = (int64_t)kb * NPAD * TC_KB + (int64_t)q * NPAD * KS;
        if (lane == 2) bulk_g2s(st + 2 * C::A_BYTES, Vhi + voff, C::V_BYTES, &full[s]);
        if (lane == 3) bulk_g2s(st + 2 * C::A_BYTES + C::V_BYTES, Vlo + voff, C::V_BYTES, &full[s]);
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      constexpr uint32_t idesc_k = idesc_bf16(TC_M, NPAD, false);
      constexpr uint32_t idesc_mn = idesc_bf16(TC_M, NPAD, false, true);
      const int nks = nkb * QK;
      for (int64_t lt = 0; lt < my_tiles && ok; ++lt) {
        const int b = (int)(lt & 1);
        const int mb = (int)((blockIdx.x + lt * G) % nmb);
        if (lt >= 2) ok = mbar_wait_bounded(&acc_empty[b], (uint32_t)(((lt / 2) - 1) & 1), err);
        if (!ok) break;
        tc_fence_after();
        const uint32_t d = tmem + (uint32_t)(b * NPAD);
        for (int ksg = 0; ksg < nks && ok; ++ksg) {
          const int64_t g = lt * nks + ksg;
          const int s = (int)(g % S);
          ok = mbar_wait_bounded(&full[s], (uint32_t)((g / S) & 1), err);
          if (!ok) break;
          tc_fence_after();
          const uint8_t* st = smem + s * C::STAGE_BYTES;
          const bool mirror = mb > ((ksg / QK) >> 1);
          const uint32_t idesc = mirror ? idesc_mn : idesc_k;
          // K-major: K groups 2 KB apart, row groups 128 B; MN-major mirror:
          // K groups 128 B apart (LBO), row groups KS * 16 B (SBO: one
          // 2 KB-strided K-group row of the square holds KS / 8 cores per stage)
          const uint32_t a_lbo = mirror ? 128u : (TC_M / 8) * 128u, a_sbo = mirror ? (uint32_t)(KS * 16) : 128u;
#pragma unroll
          for (int ks = 0; ks < KS / 16; ++ks) {
            const uint32_t ak = mirror ? 2 * ks * 128 : 2 * ks * (TC_M / 8) * 128, vk = 2 * ks * (NPAD / 8) * 128;
            const uint64_t dah = smem_desc(st + ak, a_lbo, a_sbo);
            const uint64_t dal = smem_desc(st + C::A_BYTES + ak, a_lbo, a_sbo);
            const uint64_t dvh = smem_desc(st + 2 * C::A_BYTES + vk, (NPAD / 8) * 128, 128);
            const uint64_t dvl = smem_desc(st + 2 * C::A_BYTES + C::V_BYTES + vk, (NPAD / 8) * 128, 128);
            const uint32_t acc0 = (ksg > 0 || ks > 0) ? 1u : 0u;
            tc_mma(d, dah, dvh, idesc, acc0);
            tc_mma(d, dah, dvl, idesc, 1u);
            tc_mma(d, dal, dvh, idesc, 1u);
          }
          tc_commit(&empty[s]);
        }
        tc_commit(&acc_full[b]);
      }
    }
  } else {
    // epilogue warps 2..5
    const int quad = warp & 3;
    const int m = quad * 32 + lane;
    for (int64_t lt = 0; lt < my_tiles; ++lt) {
      const int b = (int)(lt & 1);
      const bool got = mbar_wait_bounded(&acc_full[b], (uint32_t)((lt / 2) & 1), err);
      if (!__all_sync(0xffffffffu, got)) {
        ok = false;
        break;
      }
      tc_fence_after();
      const int64_t tile = blockIdx.x + lt * G;
      const int64_t pl = tile / nmb;
      const int mb = (int)(tile % nmb);
      const int64_t xbase = ((pl * nmb + mb) * (int64_t)nib) * BLOCK_ELEMS;
      // with wpart: this row's share of J's scalar <V, X_P> (V in FP64, X the
      // FP32 accumulator) for the aux row of the tile
      const int row = mb * TC_M + m;
      double jacc = 0.0;
#pragma unroll 1
      for (int c0 = 0; c0 < NPAD; c0 += 32) {
        float v[32];
        tc_ld32(tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)(b * NPAD + c0), v);
        if constexpr (WJ) {
          if (row < nrows) {
#pragma unroll 32
            for (int jj = 0; jj < 32 && c0 + jj < ncols; ++jj)
              jacc = fma((double)v[jj], Vd[(int64_t)(c0 + jj) * ldv + row], jacc);
          }
        }
        const int ib = c0 / TC_KB;
#pragma unroll
        for (int gq = 0; gq < 4; ++gq) {
          uint4 h, l;
          split_bf16x8(v + gq * 8, h, l);
          const int k = (c0 % TC_KB) + gq * 8;
          const int64_t off = xbase + (int64_t)ib * BLOCK_ELEMS + core_off(m, k, TC_M);
          *reinterpret_cast<uint4*>(Xhi + off) = h;
          *reinterpret_cast<uint4*>(Xlo + off) = l;
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&acc_empty[b]);
      if constexpr (WJ) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) jacc += __shfl_xor_sync(0xffffffffu, jacc, o);
        if (lane == 0) wpart[tile * 4 + quad] = jacc;
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tc_dealloc(tmem, 2 * NPAD);
}

// w[p0 + p] += sgn * (the 4 nmb warp shares of aux row p, in a fixed order);
// one warp per aux row.
__global__ void __launch_bounds__(256) k_tc_wreduce(const double* __restrict__ wpart, int64_t np, int per_row,
                                                    double sgn, int64_t p0, double* __restrict__ w) {
  const int lane = threadIdx.x & 31;
  for (int64_t pl = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; pl < np;
       pl += ((int64_t)gridDim.x * blockDim.x) >> 5) {
    double a = 0.0;
    for (int t = lane; t < per_row; t += 32) a += wpart[pl * per_row + t];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if (lane == 0) w[p0 + pl] += sgn * a;
  }
}

// ---- paired half-transform: one M = 256 MMA over two SMs (cta_group::2) -----------
// The persistent kernel above streams all of V (n_pad x npad, hi and lo) from
// L2 again for every 128-row tile: two thirds of each stage.  Here a cluster of
// two CTAs runs one tcgen05.mma.cta_group::2 with M = 256: CTA r supplies the A
// rows of aux row P0 + r (same row block mb, so both take the same mirrored or
// direct reading of the same square position) and half r of V's columns, and
// each CTA's tensor memory receives its own 128 rows x npad columns.  Per SM a
// stage is then A (32 KB) + half of V, and V crosses from L2 once per pair.
//
// Synchronisation (one MMA issuer, thread 32 of CTA 0):
//  * CTA 0's producer arms CTA 0's full[s] with the bytes of both CTAs' halves;
//    both CTAs' producers fill their own stage with tiled tensor copies of the
//    .cta_group::2 form whose completion lands on CTA 0's full[s] (no
//    multicast: each CTA reads only its own operands), so the issuer waits on
//    one local barrier per stage;
//  * the issuer's commits arrive on empty[s] and acc_full[b] of both CTAs
//    (commit multicast over the pair);
//  * the four epilogue warps of each CTA arrive on CTA 0's acc_empty[b]
//    (count 8) when they have read their rows of accumulator b.
// All waits are bounded by the context's budget; every thread reaches the final
// cluster barrier, after which the pair releases its tensor memory together.
template <int NPAD>
struct HalfTcPair {
  static constexpr int STAGES = NPAD == 256 ? 3 : NPAD == 128 ? 4 : 5;
  static constexpr uint32_t VH_BYTES = (NPAD / 2) * TC_KB * 2;  // one plane's half of V per stage
  static constexpr uint32_t STAGE_BYTES = 2 * BLOCK_BYTES + 2 * VH_BYTES;
  static constexpr size_t SMEM = 232448;
  static_assert((size_t)STAGES * STAGE_BYTES + 1024 + 512 <= SMEM, "stage budget");
};

__device__ __forceinline__ uint32_t cluster_ctarank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}

__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release;\n\tbarrier.cluster.wait.acquire;" ::: "memory");
}

// shared::cluster address of the same object in CTA `rank` of the cluster
__device__ __forceinline__ uint32_t cluster_addr(const void* p, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(smem_u32(p)), "r"(rank));
  return r;
}

__device__ __forceinline__ void mbar_arrive_cluster(uint32_t addr) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(addr) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait_cluster(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ bool mbar_wait_cluster_bounded(uint64_t* bar, uint32_t parity, int* err) {
  if (mbar_try_wait_cluster(bar, parity)) return true;
  const uint64_t t0 = globaltimer_ns();
  const uint64_t limit = wait_budget_ns(err);
  while (true) {
    if (mbar_try_wait_cluster(bar, parity)) return true;
    if (globaltimer_ns() - t0 > limit) {
      if (err) atomicCAS(err, DEV_OK, DEV_WAIT_TIMEOUT);
      return false;
    }
  }
}

__device__ __forceinline__ void tc2_alloc(uint32_t* dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst_smem)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tc2_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void tc2_mma(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                        uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// arrive (once the issuer's earlier MMAs complete) on `bar` in both CTAs of the pair
__device__ __forceinline__ void tc2_commit_pair(uint64_t* bar) {
  const uint16_t mask = 3;
  asm volatile("tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::
                   "r"(smem_u32(bar)),
               "h"(mask)
               : "memory");
}

// Tiled tensor copies (this GPU's memory, no multicast) into this CTA's shared
// memory whose completion is counted on the mbarrier at shared::cluster address
// `bar`, which may belong to the other CTA of the pair.
__device__ __forceinline__ void tma2_load_2d(void* smem_dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, "
      "%3}], [%4];" ::"r"(smem_u32(smem_dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void tma2_load_3d(void* smem_dst, const CUtensorMap* map, int x, int y, int z,
                                             uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, "
      "%3, %4}], [%5];" ::"r"(smem_u32(smem_dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(bar)
      : "memory");
}

// Operand maps of the paired kernel: direct blocks of a split plane as rows of
// 64 BF16 (box 64 x 128: one 16 KB block), the mirrored halves (mirror_map), and
// the halves of V as rows of 64 BF16 (box 64 x npad/2).
struct PairMaps {
  CUtensorMap dhi, dlo, mhi, mlo, vhi, vlo;
};

template <int NPAD, bool WJ>
__global__ void __launch_bounds__(192, 1)
    k_half_tc_pair(int nmb, int nkb, int nib, int nv, int64_t np, int64_t ntp, __nv_bfloat16* __restrict__ Xhi,
                   __nv_bfloat16* __restrict__ Xlo, int* err, const __grid_constant__ PairMaps maps, int64_t p0,
                   const double* __restrict__ Vd, int64_t ldv, int ncols, int nrows, double* __restrict__ wpart) {
  const int64_t nsq = (int64_t)nmb * (nmb + 1) / 2;
  using C = HalfTcPair<NPAD>;
  constexpr int S = C::STAGES;
  const int NH = nv / 2;  // V columns (B rows) per CTA; nv: the MMA's N, a multiple of 16 up to NPAD
  const uint32_t stage_tx = 2 * BLOCK_BYTES + 2 * (uint32_t)NH * TC_KB * 2;  // bytes one CTA lands per stage
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + S * C::STAGE_BYTES);  // used in CTA 0
  uint64_t* empty = full + S;
  uint64_t* acc_full = empty + S;      // [2]
  uint64_t* acc_empty = acc_full + 2;  // [2], used in CTA 0
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(acc_empty + 2);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = cluster_ctarank();
  const int64_t NPR = gridDim.x / 2, pair = blockIdx.x / 2;
  const int64_t my_tiles = ntp > pair ? (ntp - pair + NPR - 1) / NPR : 0;

  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&acc_full[b], 1);
      mbar_init(&acc_empty[b], 8);
    }
    mbar_fence_init();
  }
  if (warp == 0) tc2_alloc(tmem_slot, 2 * NPAD);
  tc_fence_before();
  cluster_sync_all();  // barriers initialised and tensor memory allocated in both CTAs
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  bool ok = true;

  if (warp == 0) {
    for (int64_t lt = 0; lt < my_tiles && ok; ++lt) {
      const int64_t tile = pair + lt * NPR;
      const int64_t P0 = 2 * (tile / nmb);
      const int mb = (int)(tile % nmb);
      const int64_t pl = P0 + (int64_t)rank < np ? P0 + (int64_t)rank : P0;  // a missing partner reads P0
      for (int kb = 0; kb < nkb && ok; ++kb) {
        const int64_t g = lt * nkb + kb;
        const int s = (int)(g % S);
        if (lane == 0 && g >= S) ok = mbar_wait_cluster_bounded(&empty[s], (uint32_t)(((g / S) - 1) & 1), err);
        ok = __shfl_sync(0xffffffffu, ok, 0);
        if (!ok) break;
        uint8_t* st = smem + s * C::STAGE_BYTES;
        const uint32_t fb = cluster_addr(&full[s], 0);
        if (lane == 0 && rank == 0) mbar_arrive_expect_tx(&full[s], 2 * stage_tx);
        __syncwarp();
        const int Kb = kb >> 1, j = kb & 1;
        if (mb <= Kb) {
          const int y = (int)((((p0 + pl) * nsq + sq_index(mb, Kb)) * 2 + j) * TC_M);
          if (lane == 0) tma2_load_2d(st, &maps.dhi, 0, y, fb);
          if (lane == 1) tma2_load_2d(st + BLOCK_BYTES, &maps.dlo, 0, y, fb);
        } else {
          const int z = (int)(((p0 + pl) * nsq + sq_index(Kb, mb)) * 16);
          if (lane == 0) tma2_load_3d(st, &maps.mhi, 0, 2 * j, z, fb);
          if (lane == 1) tma2_load_3d(st + BLOCK_BYTES, &maps.mlo, 0, 2 * j, z, fb);
        }
        // V in halves: stage kb holds half 0 then half 1, each (NH x 64) K-major
        const int yv = (kb * 2 + (int)rank) * NH;
        if (lane == 2) tma2_load_2d(st + 2 * BLOCK_BYTES, &maps.vhi, 0, yv, fb);
        if (lane == 3) tma2_load_2d(st + 2 * BLOCK_BYTES + C::VH_BYTES, &maps.vlo, 0, yv, fb);
      }
    }
  } else if (warp == 1) {
    if (lane == 0 && rank == 0) {
      const uint32_t idesc_k = idesc_bf16(2 * TC_M, nv, false);
      const uint32_t idesc_mn = idesc_bf16(2 * TC_M, nv, false, true);
      for (int64_t lt = 0; lt < my_tiles && ok; ++lt) {
        const int b = (int)(lt & 1);
        const int mb = (int)((pair + lt * NPR) % nmb);
        if (lt >= 2) ok = mbar_wait_cluster_bounded(&acc_empty[b], (uint32_t)(((lt / 2) - 1) & 1), err);
        if (!ok) break;
        tc_fence_after();
        const uint32_t d = tmem + (uint32_t)(b * NPAD);
        for (int kb = 0; kb < nkb && ok; ++kb) {
          const int64_t g = lt * nkb + kb;
          const int s = (int)(g % S);
          ok = mbar_wait_cluster_bounded(&full[s], (uint32_t)((g / S) & 1), err);
          if (!ok) break;
          tc_fence_after();
          const uint8_t* st = smem + s * C::STAGE_BYTES;
          const bool mirror = mb > (kb >> 1);
          const uint32_t idesc = mirror ? idesc_mn : idesc_k;
          const uint32_t a_lbo = mirror ? 128u : (TC_M / 8) * 128u, a_sbo = mirror ? 1024u : 128u;
#pragma unroll
          for (int ks = 0; ks < TC_KB / 16; ++ks) {
            const uint32_t ak = mirror ? 2 * ks * 128 : 2 * ks * (TC_M / 8) * 128, vk = 2 * ks * (NH / 8) * 128;
            const uint64_t dah = smem_desc(st + ak, a_lbo, a_sbo);
            const uint64_t dal = smem_desc(st + BLOCK_BYTES + ak, a_lbo, a_sbo);
            const uint64_t dvh = smem_desc(st + 2 * BLOCK_BYTES + vk, (NH / 8) * 128, 128);
            const uint64_t dvl = smem_desc(st + 2 * BLOCK_BYTES + C::VH_BYTES + vk, (NH / 8) * 128, 128);
            const uint32_t acc0 = (kb > 0 || ks > 0) ? 1u : 0u;
            tc2_mma(d, dah, dvh, idesc, acc0);
            tc2_mma(d, dah, dvl, idesc, 1u);
            tc2_mma(d, dal, dvh, idesc, 1u);
          }
          tc2_commit_pair(&empty[s]);
        }
        tc2_commit_pair(&acc_full[b]);
      }
    }
  } else {
    // epilogue warps 2..5: this CTA's 128 rows of accumulator b
    const int quad = warp & 3;
    const int m = quad * 32 + lane;
    const uint32_t acc_empty0 = cluster_addr(&acc_empty[0], 0);
    const uint32_t acc_empty1 = cluster_addr(&acc_empty[1], 0);
    for (int64_t lt = 0; lt < my_tiles; ++lt) {
      const int b = (int)(lt & 1);
      const bool got = mbar_wait_cluster_bounded(&acc_full[b], (uint32_t)((lt / 2) & 1), err);
      if (!__all_sync(0xffffffffu, got)) {
        ok = false;
        break;
      }
      tc_fence_after();
      const int64_t tile = pair + lt * NPR;
      const int64_t pl = 2 * (tile / nmb) + (int64_t)rank;
      const int mb = (int)(tile % nmb);
      const int row = mb * TC_M + m;
      double jacc = 0.0;
      if (pl < np) {
        const int64_t xbase = ((pl * nmb + mb) * (int64_t)nib) * BLOCK_ELEMS;
#pragma unroll 1
        for (int c0 = 0; c0 < NPAD; c0 += 32) {
          float v[32];
          if (c0 < nv)  // warp-uniform
            tc_ld32(tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)(b * NPAD + c0), v);
          // X's columns from nv on (beyond the MMA's N) are written as zeros
#pragma unroll
          for (int i = 0; i < 32; ++i)
            if (c0 + i >= nv) v[i] = 0.0f;
          // with wpart: this row's share of J's scalar <V, X_P> (V in FP64)
          if constexpr (WJ) {
            if (row < nrows) {
#pragma unroll 32
              for (int jj = 0; jj < 32 && c0 + jj < ncols; ++jj)
                jacc = fma((double)v[jj], Vd[(int64_t)(c0 + jj) * ldv + row], jacc);
            }
          }
          const int ib = c0 / TC_KB;
#pragma unroll
          for (int gq = 0; gq < 4; ++gq) {
            uint4 h, l;
            split_bf16x8(v + gq * 8, h, l);
            const int k = (c0 % TC_KB) + gq * 8;
            const int64_t off = xbase + (int64_t)ib * BLOCK_ELEMS + core_off(m, k, TC_M);
            *reinterpret_cast<uint4*>(Xhi + off) = h;
            *reinterpret_cast<uint4*>(Xlo + off) = l;
          }
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive_cluster(b ? acc_empty1 : acc_empty0);
      if (WJ && pl < np) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) jacc += __shfl_xor_sync(0xffffffffu, jacc, o);
        if (lane == 0) wpart[(pl * nmb + mb) * 4 + quad] = jacc;
      }
    }
  }
  tc_fence_before();
  cluster_sync_all();  // the pair's MMAs, copies and remote arrivals are over
  tc_fence_after();
  if (warp == 0) tc2_dealloc(tmem, 2 * NPAD);
}

// ---- rank update on tcgen05 --------------------------------------------------------
// CTA per (upper block pair q, P split): K[Ib][Jb] (128 x 128) = sum_p sum_ib
// X_p[Ib, ib] S X_p[Jb, ib]^T, FP32 in TMEM, written as an FP32 partial.
struct RankTc {
  static constexpr int STAGES = 3;
  static constexpr uint32_t STAGE_BYTES = 4 * BLOCK_BYTES;  // A hi, A lo, B hi, B lo
  // The whole per-CTA shared memory is reserved (one CTA per SM either way),
  // so descriptor strides never point outside the allocation.
  static constexpr size_t SMEM = 232448;
  static_assert((size_t)STAGES * STAGE_BYTES + 1024 + 256 <= SMEM, "rank stage budget");
};

__device__ __forceinline__ int64_t tri_root_tc(int64_t t) {
  int64_t j = (int64_t)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
  while (j * (j + 1) / 2 > t) --j;
  while ((j + 1) * (j + 2) / 2 <= t) ++j;
  return j;
}

__global__ void __launch_bounds__(128, 1)
    k_rank_tc(const __nv_bfloat16* __restrict__ Xhi, const __nv_bfloat16* __restrict__ Xlo, int nmb, int nib,
              int ncols, int npos_blocks, int64_t np, int splits, float* __restrict__ part, int* err) {
  using C = RankTc;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + C::STAGES * C::STAGE_BYTES);
  uint64_t* empty = full + C::STAGES;
  uint64_t* accf = empty + C::STAGES;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(accf + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t q = blockIdx.x;
  const int sp = blockIdx.y;
  const int64_t Jb = tri_root_tc(q), Ib = q - Jb * (Jb + 1) / 2;
  const int64_t pa = np * sp / splits, pb = np * (sp + 1) / splits;
  const int64_t nsteps = (pb - pa) * nib;

  if (threadIdx.x == 0) {
    for (int s = 0; s < C::STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(accf, 1);
    mbar_fence_init();
  }
  if (warp == 0) tc_alloc(tmem_slot, 128);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  bool ok = true;

  if (warp == 0 && lane == 0) {
    for (int64_t t = 0; t < nsteps && ok; ++t) {
      const int s = (int)(t % C::STAGES);
      if (t >= C::STAGES) ok = mbar_wait_bounded(&empty[s], (uint32_t)(((t / C::STAGES) - 1) & 1), err);
      if (!ok) break;
      const int64_t p = pa + t / nib;
      const int ib = (int)(t % nib);
      uint8_t* st = smem + s * C::STAGE_BYTES;
      mbar_arrive_expect_tx(&full[s], C::STAGE_BYTES);
      const int64_t ao = ((p * nmb + Ib) * (int64_t)nib + ib) * BLOCK_ELEMS;
      const int64_t bo = ((p * nmb + Jb) * (int64_t)nib + ib) * BLOCK_ELEMS;
      bulk_g2s(st, Xhi + ao, BLOCK_BYTES, &full[s]);
      bulk_g2s(st + BLOCK_BYTES, Xlo + ao, BLOCK_BYTES, &full[s]);
      bulk_g2s(st + 2 * BLOCK_BYTES, Xhi + bo, BLOCK_BYTES, &full[s]);
      bulk_g2s(st + 3 * BLOCK_BYTES, Xlo + bo, BLOCK_BYTES, &full[s]);
    }
  } else if (warp == 1 && lane == 0) {
    constexpr uint32_t id_pos = idesc_bf16(TC_M, TC_M, false);
    constexpr uint32_t id_neg = idesc_bf16(TC_M, TC_M, true);
    for (int64_t t = 0; t < nsteps && ok; ++t) {
      const int s = (int)(t % C::STAGES);
      ok = mbar_wait_bounded(&full[s], (uint32_t)((t / C::STAGES) & 1), err);
      if (!ok) break;
      tc_fence_after();
      const int ib = (int)(t % nib);
      const uint32_t idesc = ib < npos_blocks ? id_pos : id_neg;
      const uint8_t* st = smem + s * C::STAGE_BYTES;
#pragma unroll
      for (int ks = 0; ks < TC_KB / 16; ++ks) {
        if (ib * TC_KB + ks * 16 >= ncols) break;  // X's padding columns: no work
        const uint32_t kof = 2 * ks * (TC_M / 8) * 128;
        const uint64_t dah = smem_desc(st + kof, (TC_M / 8) * 128, 128);
        const uint64_t dal = smem_desc(st + BLOCK_BYTES + kof, (TC_M / 8) * 128, 128);
        const uint64_t dbh = smem_desc(st + 2 * BLOCK_BYTES + kof, (TC_M / 8) * 128, 128);
        const uint64_t dbl = smem_desc(st + 3 * BLOCK_BYTES + kof, (TC_M / 8) * 128, 128);
        const uint32_t acc0 = (t > 0 || ks > 0) ? 1u : 0u;
        tc_mma(tmem, dah, dbh, idesc, acc0);
        tc_mma(tmem, dah, dbl, idesc, 1u);
        tc_mma(tmem, dal, dbh, idesc, 1u);
      }
      tc_commit(&empty[s]);
    }
    tc_commit(accf);
  }
  __syncwarp();
  const bool acc_ok = __syncthreads_and(ok) && nsteps > 0 && mbar_wait_bounded(accf, 0, err);
  tc_fence_after();
  const int m = warp * 32 + lane;
  float* out = part + ((int64_t)sp * gridDim.x + q) * (TC_M * TC_M);
#pragma unroll 1
  for (int c0 = 0; c0 < TC_M; c0 += 32) {
    float v[32];
    if (acc_ok) {
      tc_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
    } else {
#pragma unroll
      for (int i = 0; i < 32; ++i) v[i] = 0.0f;
    }
#pragma unroll
    for (int i = 0; i < 32; ++i) out[m + TC_M * (c0 + i)] = v[i];
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tc_dealloc(tmem, 128);
}

// Paired rank update: a cluster of two CTAs computes the 2 x 2 group of K blocks
// {2a, 2a+1} x {2c, 2c+1} (a <= c) with M = 256, N = 256 MMAs over the pair:
// CTA r holds the A rows of block 2a + r and the B rows of block 2c + r, and
// its tensor memory receives rows 2a + r against both column blocks.  Per SM a
// stage is one A and one B block (64 KB) for twice the MMA work of the one-SM
// kernel, and each SM reads half the shared-memory operand bytes per flop.
// Blocks below the diagonal (the (2c+1, 2c) block of a diagonal group) and
// blocks beyond n are computed but not written.  Same partial layout as
// k_rank_tc: part[(sp pairs + q) 128 x 128], q = Jb (Jb + 1) / 2 + Ib.
// Synchronisation as in k_half_tc_pair (each CTA's X blocks by .cta_group::2
// tensor copies completing on CTA 0's full barrier, which CTA 0 arms with both
// CTAs' bytes; commit multicast over the pair, bounded waits, a cluster barrier
// before release).  mxh / mxl: the X planes as rows of 64 BF16, box 64 x 128
// (one 16 KB block).
__global__ void __launch_bounds__(128, 1)
    k_rank_tc_pair(const __grid_constant__ CUtensorMap mxh, const __grid_constant__ CUtensorMap mxl, int nmb, int nib,
                   int ncols, int npos_blocks, int64_t np, int splits, int64_t ngroups, float* __restrict__ part,
                   int* err) {
  using C = RankTc;
  constexpr int S = C::STAGES;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + S * C::STAGE_BYTES);  // used in CTA 0
  uint64_t* empty = full + S;
  uint64_t* accf = empty + S;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(accf + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = cluster_ctarank();
  const int64_t cl = blockIdx.x / 2;
  const int64_t gq = cl % ngroups;
  const int sp = (int)(cl / ngroups);
  const int64_t gc = tri_root_tc(gq), ga = gq - gc * (gc + 1) / 2;
  const int64_t Ib = 2 * ga + rank, Jb = 2 * gc + rank;  // this CTA's A rows and B rows
  const int64_t Ia = Ib < nmb ? Ib : 2 * ga, Ja = Jb < nmb ? Jb : 2 * gc;  // blocks actually read
  const int64_t pa = np * sp / splits, pb = np * (sp + 1) / splits;
  const int64_t nsteps = (pb - pa) * nib;
  const int64_t pairs = (int64_t)nmb * (nmb + 1) / 2;

  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(accf, 1);
    mbar_fence_init();
  }
  if (warp == 0) tc2_alloc(tmem_slot, 256);
  tc_fence_before();
  cluster_sync_all();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  bool ok = true;

  if (warp == 0 && lane == 0) {
    for (int64_t t = 0; t < nsteps && ok; ++t) {
      const int s = (int)(t % S);
      if (t >= S) ok = mbar_wait_cluster_bounded(&empty[s], (uint32_t)(((t / S) - 1) & 1), err);
      if (!ok) break;
      const int64_t p = pa + t / nib;
      const int ib = (int)(t % nib);
      uint8_t* st = smem + s * C::STAGE_BYTES;
      const uint32_t fb = cluster_addr(&full[s], 0);
      if (rank == 0) mbar_arrive_expect_tx(&full[s], 2 * C::STAGE_BYTES);
      const int ya = (int)(((p * nmb + Ia) * (int64_t)nib + ib) * TC_M);
      const int yb = (int)(((p * nmb + Ja) * (int64_t)nib + ib) * TC_M);
      tma2_load_2d(st, &mxh, 0, ya, fb);
      tma2_load_2d(st + BLOCK_BYTES, &mxl, 0, ya, fb);
      tma2_load_2d(st + 2 * BLOCK_BYTES, &mxh, 0, yb, fb);
      tma2_load_2d(st + 3 * BLOCK_BYTES, &mxl, 0, yb, fb);
    }
  } else if (warp == 1 && lane == 0 && rank == 0) {
    constexpr uint32_t id_pos = idesc_bf16(2 * TC_M, 2 * TC_M, false);
    constexpr uint32_t id_neg = idesc_bf16(2 * TC_M, 2 * TC_M, true);
    for (int64_t t = 0; t < nsteps && ok; ++t) {
      const int s = (int)(t % S);
      ok = mbar_wait_cluster_bounded(&full[s], (uint32_t)((t / S) & 1), err);
      if (!ok) break;
      tc_fence_after();
      const int ib = (int)(t % nib);
      const uint32_t idesc = ib < npos_blocks ? id_pos : id_neg;
      const uint8_t* st = smem + s * C::STAGE_BYTES;
#pragma unroll
      for (int ks = 0; ks < TC_KB / 16; ++ks) {
        if (ib * TC_KB + ks * 16 >= ncols) break;  // X's padding columns: no work
        const uint32_t kof = 2 * ks * (TC_M / 8) * 128;
        const uint64_t dah = smem_desc(st + kof, (TC_M / 8) * 128, 128);
        const uint64_t dal = smem_desc(st + BLOCK_BYTES + kof, (TC_M / 8) * 128, 128);
        const uint64_t dbh = smem_desc(st + 2 * BLOCK_BYTES + kof, (TC_M / 8) * 128, 128);
        const uint64_t dbl = smem_desc(st + 3 * BLOCK_BYTES + kof, (TC_M / 8) * 128, 128);
        const uint32_t acc0 = (t > 0 || ks > 0) ? 1u : 0u;
        tc2_mma(tmem, dah, dbh, idesc, acc0);
        tc2_mma(tmem, dah, dbl, idesc, 1u);
        tc2_mma(tmem, dal, dbh, idesc, 1u);
      }
      tc2_commit_pair(&empty[s]);
    }
    tc2_commit_pair(accf);
  }
  __syncwarp();
  const bool acc_ok = __syncthreads_and(ok) && nsteps > 0 && mbar_wait_cluster_bounded(accf, 0, err);
  tc_fence_after();
  const int m = warp * 32 + lane;
#pragma unroll 1
  for (int h = 0; h < 2; ++h) {
    const int64_t jb = 2 * gc + h;
    if (Ib >= nmb || jb >= nmb || Ib > jb) continue;  // uniform over the CTA
    const int64_t q = jb * (jb + 1) / 2 + Ib;
    float* out = part + ((int64_t)sp * pairs + q) * (TC_M * TC_M);
#pragma unroll 1
    for (int c0 = 0; c0 < TC_M; c0 += 32) {
      float v[32];
      if (acc_ok) {
        tc_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(h * TC_M + c0), v);
      } else {
#pragma unroll
        for (int i = 0; i < 32; ++i) v[i] = 0.0f;
      }
#pragma unroll
      for (int i = 0; i < 32; ++i) out[m + TC_M * (c0 + i)] = v[i];
    }
  }
  tc_fence_before();
  cluster_sync_all();
  tc_fence_after();
  if (warp == 0) tc2_dealloc(tmem, 256);
}

// FP32 partials -> packed upper K (FP64), out (+)= scale * sum_splits.
__global__ void __launch_bounds__(256) k_rank_tc_finalize(int64_t n, int64_t npair, const float* __restrict__ part,
                                                          int splits, int64_t pairs, double scale, int accumulate,
                                                          double* __restrict__ out) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < npair; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t j = tri_root_tc(e), i = e - j * (j + 1) / 2;
    const int64_t Ib = i / TC_M, Jb = j / TC_M;
    const int64_t q = Jb * (Jb + 1) / 2 + Ib;
    const int64_t off = (i % TC_M) + (int64_t)TC_M * (j % TC_M);
    double v = 0.0;
    for (int s = 0; s < splits; ++s) v += (double)part[((int64_t)s * pairs + q) * (TC_M * TC_M) + off];
    v *= scale;
    out[e] = accumulate ? out[e] + v : v;
  }
}

}  // namespace

// ============================================================================
// host launchers
// ============================================================================
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder();

TcGeom make_tc_geom(const Geom& g, int ncols) {
  TcGeom t;
  t.nmb = (int)cdiv_t(g.n, TC_M);
  t.nkb = (int)cdiv_t(g.n, TC_KB);
  t.npad = ncols <= 64 ? 64 : ncols <= 128 ? 128 : 256;
  t.nib = t.npad / TC_KB;
  t.block_elems = BLOCK_ELEMS;
  // SM-pair (cta_group::2) kernels, their copies completing on CTA 0's
  // barrier: measured on B200 (one SM per tile -> pair, ms), the half-transform
  // n = 600: 0.754 -> 0.698, 768: 1.442 -> 1.348, 1200: 9.86 -> 8.05; the rank
  // update n = 600: 0.387 -> 0.472 (few k steps per CTA), 768: 0.745 -> 0.593,
  // 1200: 6.28 -> 4.38.  So the half-transform pairs from five 128-row blocks,
  // the rank update from six.  RIJK_TC_PAIR=0 / 1 turns both off / on.
  const char* e = getenv("RIJK_TC_PAIR");
  if (e && e[0] == '0') {
    t.pair = t.pair_rank = 0;
  } else if (e && e[0] == '1') {
    t.pair = t.pair_rank = 1;
  } else {
    t.pair = t.nmb >= 5 ? 1 : 0;
    t.pair_rank = t.nmb >= 6 ? 1 : 0;
  }
  // the paired half-transform reads every operand by tensor copies: only
  // tensors whose planes the maps' 32-bit row index covers (V's halves are
  // split in the paired layout, so this is decided before anything runs)
  if (t.pair && (!tensor_map_encoder() || g.naux * ((int64_t)t.nmb * (t.nmb + 1) / 2) * 2 * TC_M > INT32_MAX))
    t.pair = 0;
  // the paired MMAs run N = ncols rounded up to 16 (16..256) rather than the
  // 64 / 128 / 256 of X's layout: 200 occupied columns take N = 208, not 256
  t.ncols = ncols;
  t.nv = t.pair ? std::min(t.npad, std::max(16, (ncols + 15) / 16 * 16)) : t.npad;
  return t;
}

// BF16 elements per aux row of one plane: the upper 128 x 128 squares
static int64_t tc_row_elems(const Geom& g) {
  const int64_t nmb = cdiv_t(g.n, TC_M);
  return nmb * (nmb + 1) / 2 * 2 * BLOCK_ELEMS;
}

int64_t tc_tensor_elems(const Geom& g) { return g.naux * tc_row_elems(g); }

void launch_split_tensor(const Geom& g, const double* B, int64_t p0, int64_t np, void* hi, void* lo,
                         cudaStream_t st) {
  const int nmb = (int)cdiv_t(g.n, TC_M);
  const int64_t per_p = tc_row_elems(g);
  auto* h = static_cast<__nv_bfloat16*>(hi) + p0 * per_p;
  auto* l = static_cast<__nv_bfloat16*>(lo) + p0 * per_p;
  const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>(cdiv_t(np * per_p, 256), 148 * 32));
  count_launch();
  k_split_tensor<<<blocks, 256, 0, st>>>(B, g.ldB, g.n, nmb, p0, np, h, l);
}

void launch_split_cols(const Geom& g, const TcGeom& t, const double* V, int64_t ldv, int ncols, void* hi, void* lo,
                       cudaStream_t st) {
  const int64_t total = (int64_t)(t.pair ? t.nv : t.npad) * TC_KB * t.nkb;
  const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>(cdiv_t(total, 256), 148 * 8));
  count_launch();
  k_split_cols<<<blocks, 256, 0, st>>>(V, ldv, g.n, ncols, t.pair ? t.nv : t.npad, t.nkb, t.pair ? 2 : 1,
                                       static_cast<__nv_bfloat16*>(hi), static_cast<__nv_bfloat16*>(lo));
}

static int sm_count() {
  int dev = 0, n = 148;
  cudaGetDevice(&dev);
  if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    cudaGetLastError();
    n = 148;
  }
  return n;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no libcuda link).
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
    else
      cudaGetLastError();
  });
  return fn;
}

// Map of one split plane for the mirrored reads (see k_half_tc_persistent).
// ks: K rows of the mirrored square per copy (64 or 32), i.e. ks / 32 of the
// four 256-element pieces of each of its K-group rows.
static bool mirror_map(CUtensorMap* m, const void* plane, int64_t rows, int ks = TC_KB) {
  auto enc = tensor_map_encoder();
  if (!enc || rows <= 0 || rows > (int64_t)INT32_MAX) return false;
  const cuuint64_t dims[3] = {256, 4, (cuuint64_t)rows};
  const cuuint64_t strides[2] = {512, 2048};  // bytes, dims 1 and 2
  const cuuint32_t box[3] = {256, (cuuint32_t)(ks / 32), 16};
  const cuuint32_t estr[3] = {1, 1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<void*>(plane), dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int NPAD, int KS>
static void half_tc_ks(const Geom& g, const TcGeom& t, const void* Bhi, const void* Blo, int64_t p0, int64_t np,
                       const void* Vhi, const void* Vlo, void* Xhi, void* Xlo, int* err, cudaStream_t st,
                       const CUtensorMap& mhi, const CUtensorMap& mlo, bool tm, const TcJ* jw) {
  using C = HalfTcP<NPAD, KS>;
  auto kern = jw ? k_half_tc_persistent<NPAD, KS, true> : k_half_tc_persistent<NPAD, KS, false>;
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM);
  const int64_t per_p = tc_row_elems(g);
  const int64_t ntiles = np * t.nmb;
  const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(ntiles, sm_count()));
  count_launch();
  kern<<<grid, 192, C::SMEM, st>>>(
      static_cast<const __nv_bfloat16*>(Bhi) + p0 * per_p, static_cast<const __nv_bfloat16*>(Blo) + p0 * per_p,
      t.nmb, t.nkb, static_cast<const __nv_bfloat16*>(Vhi), static_cast<const __nv_bfloat16*>(Vlo), t.nib, ntiles,
      static_cast<__nv_bfloat16*>(Xhi), static_cast<__nv_bfloat16*>(Xlo), err, mhi, mlo, tm ? 1 : 0, p0,
      jw ? jw->Vd : nullptr, jw ? jw->ldv : 0, jw ? jw->ncols : 0, (int)g.n, jw ? jw->wpart : nullptr);
  if (jw) {
    const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>(cdiv_t(np, 8), 148 * 8));
    count_launch();
    k_tc_wreduce<<<blocks, 256, 0, st>>>(jw->wpart, np, 4 * t.nmb, jw->sgn, p0, jw->w);
  }
}

// K 64 per stage; RIJK_TC_KS=32 halves the stage (twice the stages in the same
// shared memory, where the mirrored squares can be fetched by tensor copies).
// Measured on B200, K 32 is slower at every width (n = 1200: 9.8 against 9.7 ms
// at 256 columns, 9.3 against 5.5 ms at 128, 8.2 against 4.1 ms at 64), so the
// look-ahead of two 96 KB stages is not what bounds the kernel.
template <int NPAD>
static void half_tc(const Geom& g, const TcGeom& t, const void* Bhi, const void* Blo, int64_t p0, int64_t np,
                    const void* Vhi, const void* Vlo, void* Xhi, void* Xlo, int* err, cudaStream_t st,
                    const TcJ* jw) {
  const char* e = getenv("RIJK_TC_KS");
  int ks = (e && atoi(e) == 32) ? 32 : 64;
  // the maps cover the whole split tensor (g.naux rows of squares), from p = 0
  const int64_t rows = g.naux * (int64_t)t.nmb * (t.nmb + 1) / 2 * 16;
  CUtensorMap mhi, mlo;
  bool tm = mirror_map(&mhi, Bhi, rows, ks) && mirror_map(&mlo, Blo, rows, ks);
  if (!tm && ks != 64) {
    ks = 64;
    tm = mirror_map(&mhi, Bhi, rows, ks) && mirror_map(&mlo, Blo, rows, ks);
  }
  if (!tm) {
    memset(&mhi, 0, sizeof(mhi));
    memset(&mlo, 0, sizeof(mlo));
  }
  if (ks == 32)
    half_tc_ks<NPAD, 32>(g, t, Bhi, Blo, p0, np, Vhi, Vlo, Xhi, Xlo, err, st, mhi, mlo, tm, jw);
  else
    half_tc_ks<NPAD, 64>(g, t, Bhi, Blo, p0, np, Vhi, Vlo, Xhi, Xlo, err, st, mhi, mlo, tm, jw);
}

// Rows of 64 BF16 of a plane (box 64 x box_rows), for the paired kernel's
// direct blocks and V halves: one box is a contiguous run of the plane.
static bool row_map(CUtensorMap* m, const void* plane, int64_t rows, int box_rows) {
  auto enc = tensor_map_encoder();
  if (!enc || rows <= 0 || rows > (int64_t)INT32_MAX || box_rows <= 0 || box_rows > 256) return false;
  const cuuint64_t dims[2] = {64, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {128};  // bytes, dim 1
  const cuuint32_t box[2] = {64, (cuuint32_t)box_rows};
  const cuuint32_t estr[2] = {1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(plane), dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int NPAD>
static void half_tc_pair(const Geom& g, const TcGeom& t, const void* Bhi, const void* Blo, int64_t p0, int64_t np,
                         const void* Vhi, const void* Vlo, void* Xhi, void* Xlo, int* err, cudaStream_t st,
                         const TcJ* jw) {
  using C = HalfTcPair<NPAD>;
  // the maps cover the whole split tensor (g.naux rows of squares), from p = 0
  const int64_t nsq = (int64_t)t.nmb * (t.nmb + 1) / 2;
  PairMaps maps;
  const bool tm = mirror_map(&maps.mhi, Bhi, g.naux * nsq * 16) && mirror_map(&maps.mlo, Blo, g.naux * nsq * 16) &&
                  row_map(&maps.dhi, Bhi, g.naux * nsq * 2 * TC_M, TC_M) &&
                  row_map(&maps.dlo, Blo, g.naux * nsq * 2 * TC_M, TC_M) &&
                  row_map(&maps.vhi, Vhi, (int64_t)t.nkb * t.nv, t.nv / 2) &&
                  row_map(&maps.vlo, Vlo, (int64_t)t.nkb * t.nv, t.nv / 2);
  if (!tm) {  // make_tc_geom pairs only what the maps cover; should an encode fail, say so and launch nothing
    static const int map_err = DEV_TENSOR_MAP;
    (void)cudaMemcpyAsync(err, &map_err, sizeof(int), cudaMemcpyHostToDevice, st);
    return;
  }
  auto kern = jw ? k_half_tc_pair<NPAD, true> : k_half_tc_pair<NPAD, false>;
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM);
  const int64_t ntp = cdiv_t(np, 2) * t.nmb;  // (aux-row pair, row block) tiles
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = 2;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.blockDim = dim3(192, 1, 1);
  cfg.dynamicSmemBytes = C::SMEM;
  cfg.stream = st;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  // as many pairs as can be resident at once (an SM without a partner in its
  // cluster group takes none), at most one per tile; cached per device
  static std::mutex mu;
  static std::map<int, int> resident_of;
  int dev = 0;
  cudaGetDevice(&dev);
  int resident = 0;
  {
    std::lock_guard<std::mutex> lock(mu);
    auto it = resident_of.find(dev);
    if (it != resident_of.end()) resident = it->second;
  }
  if (resident == 0) {
    cfg.gridDim = dim3((unsigned)(2 * (sm_count() / 2)), 1, 1);
    int nc = 0;
    if (cudaOccupancyMaxActiveClusters(&nc, kern, &cfg) != cudaSuccess || nc <= 0) {
      cudaGetLastError();
      nc = sm_count() / 2;
    }
    resident = nc;
    std::lock_guard<std::mutex> lock(mu);
    resident_of[dev] = nc;
  }
  const int64_t pairs = std::max<int64_t>(1, std::min<int64_t>(ntp, resident));
  cfg.gridDim = dim3((unsigned)(2 * pairs), 1, 1);
  count_launch();
  // a failed launch stays the thread's last CUDA error, which the caller checks
  (void)cudaLaunchKernelEx(&cfg, kern, t.nmb, t.nkb, t.nib, t.nv, np, ntp, static_cast<__nv_bfloat16*>(Xhi),
                           static_cast<__nv_bfloat16*>(Xlo), err, maps, p0, jw ? jw->Vd : nullptr, jw ? jw->ldv : 0,
                           jw ? jw->ncols : 0, (int)g.n, jw ? jw->wpart : nullptr);
  if (jw) {
    const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>(cdiv_t(np, 8), 148 * 8));
    count_launch();
    k_tc_wreduce<<<blocks, 256, 0, st>>>(jw->wpart, np, 4 * t.nmb, jw->sgn, p0, jw->w);
  }
}

void launch_half_tc(const Geom& g, const TcGeom& t, const void* Bhi, const void* Blo, int64_t p0, int64_t np,
                    const void* Vhi, const void* Vlo, void* Xhi, void* Xlo, int* err, cudaStream_t st,
                    const TcJ* jw) {
  if (t.pair) {
    if (t.npad == 64)
      half_tc_pair<64>(g, t, Bhi, Blo, p0, np, Vhi, Vlo, Xhi, Xlo, err, st, jw);
    else if (t.npad == 128)
      half_tc_pair<128>(g, t, Bhi, Blo, p0, np, Vhi, Vlo, Xhi, Xlo, err, st, jw);
    else
      half_tc_pair<256>(g, t, Bhi, Blo, p0, np, Vhi, Vlo, Xhi, Xlo, err, st, jw);
    return;
  }
  if (t.npad == 64)
    half_tc<64>(g, t, Bhi, Blo, p0, np, Vhi, Vlo, Xhi, Xlo, err, st, jw);
  else if (t.npad == 128)
    half_tc<128>(g, t, Bhi, Blo, p0, np, Vhi, Vlo, Xhi, Xlo, err, st, jw);
  else
    half_tc<256>(g, t, Bhi, Blo, p0, np, Vhi, Vlo, Xhi, Xlo, err, st, jw);
}

// Each split accumulates at most ~64 aux rows in FP32 in tensor memory (the
// splits are then summed in FP64), and there are enough CTAs to fill the GPU.
int tc_rank_splits(const TcGeom& t, int64_t np) {
  const int64_t nmg = cdiv_t(t.nmb, 2);
  const int64_t ctas = t.pair_rank ? 2 * (nmg * (nmg + 1) / 2) : (int64_t)t.nmb * (t.nmb + 1) / 2;
  const int64_t s = std::max<int64_t>(cdiv_t(2 * 148, ctas), cdiv_t(np, 64));
  return (int)std::max<int64_t>(1, std::min<int64_t>(np, s));
}

void launch_rank_tc(const Geom& g, const TcGeom& t, const void* Xhi, const void* Xlo, int64_t np, int npos_blocks,
                    int splits, float* part, int* err, cudaStream_t st) {
  const int64_t pairs = (int64_t)t.nmb * (t.nmb + 1) / 2;
  CUtensorMap mxh, mxl;
  const int64_t xrows = np * t.nmb * (int64_t)t.nib * TC_M;  // the chunk's X planes as rows of 64 BF16
  if (t.pair_rank && row_map(&mxh, Xhi, xrows, TC_M) && row_map(&mxl, Xlo, xrows, TC_M)) {
    const int64_t nmg = cdiv_t(t.nmb, 2), ngroups = nmg * (nmg + 1) / 2;
    cudaFuncSetAttribute(k_rank_tc_pair, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)RankTc::SMEM);
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(2 * ngroups * splits), 1, 1);
    cfg.blockDim = dim3(128, 1, 1);
    cfg.dynamicSmemBytes = RankTc::SMEM;
    cfg.stream = st;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    count_launch();
    // a failed launch stays the thread's last CUDA error, which the caller checks
    (void)cudaLaunchKernelEx(&cfg, k_rank_tc_pair, mxh, mxl, t.nmb, t.nib, t.ncols, npos_blocks, np, splits, ngroups,
                             part, err);
    (void)g;
    return;
  }
  // one SM per K block (also where the X planes are beyond the maps' row index)
  cudaFuncSetAttribute(k_rank_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)RankTc::SMEM);
  dim3 grid((unsigned)pairs, (unsigned)splits);
  count_launch();
  k_rank_tc<<<grid, 128, RankTc::SMEM, st>>>(static_cast<const __nv_bfloat16*>(Xhi),
                                             static_cast<const __nv_bfloat16*>(Xlo), t.nmb, t.nib, t.ncols,
                                             npos_blocks, np, splits, part, err);
  (void)g;
}

void launch_rank_tc_finalize(const Geom& g, const TcGeom& t, const float* part, int splits, double scale,
                             int accumulate, double* out, cudaStream_t st) {
  const int64_t pairs = (int64_t)t.nmb * (t.nmb + 1) / 2;
  const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>(cdiv_t(g.npair, 256), 148 * 16));
  count_launch();
  k_rank_tc_finalize<<<blocks, 256, 0, st>>>(g.n, g.npair, part, splits, pairs, scale, accumulate, out);
}

}  // namespace rijk
