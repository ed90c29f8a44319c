// Shared definitions of the RI J/K kernels: tile-packed layout of the fitted
// three-centre tensor, error flag, bounded mbarrier waits, bulk copies.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

namespace rijk {

// ---------------------------------------------------------------------------
// Tile-packed layout of B[P, mu nu] in HBM.
//
// REST stores the fitted tensor either as RIFull[n,n,N] or as the packed upper
// triangle `rimatr` [npair, N] (src/molecule_io/mod.rs:1588).  On the device
// each B_P is kept as the upper triangle of 32x32 tiles: tile (I <= J) holds
// B_P[32I + r, 32J + c] at r + 32c, tiles are numbered J(J+1)/2 + I (the same
// column-by-column order REST uses for elements), diagonal tiles are stored
// full (both triangles), and entries with mu >= n or nu >= n are zero.  Row P
// of the device tensor is ntp*1024 doubles; every tile is one contiguous 8 KB
// block, so a 32x32 operand tile of either orientation is one bulk copy per
// column and no kernel needs bounds checks.
// ---------------------------------------------------------------------------
constexpr int TS = 32;                 // tile edge
constexpr int TILE_ELEMS = TS * TS;    // 1024 doubles per stored tile
constexpr int SLD = 36;                // smem leading dimension of a staged 32x32 slot
constexpr int SLOT_DOUBLES = TS * SLD; // 1152 doubles = 9216 bytes

__host__ __device__ inline int64_t tile_pair_index(int64_t I, int64_t J) {  // I <= J
  return J * (J + 1) / 2 + I;
}
__host__ __device__ inline int64_t packed_upper_index(int64_t i, int64_t j) {  // i <= j
  return j * (j + 1) / 2 + i;
}

// Status codes shared with the C ABI (include/rest_b200.h).
enum Status : int {
  OK = 0,
  ERR_ARG = 1,
  ERR_CUDA = 2,
  ERR_NOT_SPD = 3,
  ERR_NO_TENSOR = 4,
  ERR_TIMEOUT = 5,
  ERR_NOMEM = 6,
  ERR_NONFINITE = 7,
  ERR_TOO_LARGE = 8,
};

// Device-side error flag codes (written with atomicCAS so the first one wins).
enum DevErr : int {
  DEV_OK = 0,
  DEV_WAIT_TIMEOUT = 1,
  DEV_NONFINITE = 2,
  DEV_TENSOR_MAP = 3,  // set by the host: a kernel's tensor map could not be encoded, nothing was launched
};

// The error word a kernel receives is the first of four ints a context owns:
// [0] the device-side error flag, [1] the Cholesky failing pivot, [2..3] the
// context's wait budget in nanoseconds (uint64; 0 = WAIT_LIMIT_NS).
constexpr int ERR_WORDS = 4;

// A wait on an mbarrier gives up after this many nanoseconds of %globaltimer
// unless the context sets another budget.
constexpr uint64_t WAIT_LIMIT_NS = 2000000000ull;  // 2 s

__device__ __forceinline__ uint64_t wait_budget_ns(const int* err) {
  if (!err) return WAIT_LIMIT_NS;
  const uint64_t b = *reinterpret_cast<const volatile uint64_t*>(err + 2);
  return b ? b : WAIT_LIMIT_NS;
}

// Records a non-finite input value (first error wins).
__device__ __forceinline__ void flag_nonfinite(int* err, double v) {
  if (err && !isfinite(v)) atomicCAS(err, DEV_OK, DEV_NONFINITE);
}

__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait: returns false (and records DEV_WAIT_TIMEOUT) if the phase did
// not complete within the context's wait budget (WAIT_LIMIT_NS by default).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, int* err) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = globaltimer_ns();
  const uint64_t limit = wait_budget_ns(err);
  while (true) {
    if (mbar_try_wait(bar, parity)) return true;
    if (globaltimer_ns() - t0 > limit) {
      if (err) atomicCAS(err, DEV_OK, DEV_WAIT_TIMEOUT);
      return false;
    }
  }
}

// One bulk (TMA-engine, non-tensor) copy global -> this CTA's shared memory,
// completing on `bar`.  Both addresses 16-byte aligned, size a multiple of 16.
// No multicast form is used anywhere in this library.
__device__ __forceinline__ void bulk_g2s(void* smem_dst, const void* gmem_src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(smem_dst)),
      "l"(gmem_src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// FP64 tensor-core MMA (DMMA): D(8x8) = A(8x4) B(4x8) + C.
__device__ __forceinline__ void dmma_m8n8k4(double& d0, double& d1, double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// A 32x32 block of zeros that any out-of-range operand slot is copied from.
// Static device memory is zero-initialised when the module loads; each
// translation unit that includes this header has its own copy (8 KB).
static __device__ __align__(256) double g_zero_tile[TILE_ELEMS];

}  // namespace rijk
