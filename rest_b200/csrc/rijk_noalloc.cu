// Coulomb (J) build that allocates no device memory.
//
// Some callers cannot let a library call cudaMalloc: a host program whose
// device memory is all owned by another allocator (a framework's caching
// allocator, or one arena sized when the program starts so that a shared
// 180 GB device never runs out in the middle of an SCF), and latency-bound
// loops where cudaMalloc/cudaFree would synchronise the device between Fock
// builds.  For them, rijk_vj_upper_noalloc runs the same four J kernels as
// rijk_vj_upper_dev with every scratch buffer (the folded density, the per-aux
// scalars and the pass-2 partial sums) carved out of one fixed array of static
// device memory declared below.  The caller passes all inputs and outputs as
// device pointers and no context is involved.
//
// The array costs RIJK_NOALLOC_SCRATCH_BYTES of device memory on every GPU
// that loads this module, held until the process exits.  All calls share it:
// two calls whose work overlaps on the GPU (different streams, or different
// host threads) race on it and must be ordered by the caller.  Each call
// overwrites every scratch element it reads, so nothing needs clearing
// between calls.
//
// The array's device address is looked up once per device ordinal and cached
// for the life of the process.  The device that is current when the call is
// made must be the one the pointers belong to, and the library must not be
// used across a cudaDeviceReset of that device (the reset unloads the module,
// and the cached address would then point at released memory).
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <mutex>

#include "../../include/rest_b200.h"
#include "rijk_common.cuh"
#include "rijk_internal.h"

namespace {

constexpr size_t kScratchDoubles = RIJK_NOALLOC_SCRATCH_BYTES / sizeof(double);
static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device.  In host code
// the array's name is only a host-side stand-in, so the address is looked up
// once per device (with that device current) and cached.
int scratch_on_current_device(double** out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return RIJK_ERR_CUDA;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      return RIJK_ERR_CUDA;
    }
    g_scratch_ptr[dev] = static_cast<double*>(p);
  }
  *out = g_scratch_ptr[dev];
  return RIJK_OK;
}

}  // namespace

extern "C" int rijk_vj_upper_noalloc(const double* d_tensor, int64_t row_stride, int64_t num_basis,
                                     int64_t num_auxbas, const double* d_dm, int spin_channel,
                                     double scaling_factor, int dm_mode, double* d_vj, void* stream) {
  if (!d_tensor || !d_dm || !d_vj || num_basis <= 0 || num_auxbas <= 0) return RIJK_ERR_ARG;
  if (spin_channel != 1 && spin_channel != 2) return RIJK_ERR_ARG;
  if (dm_mode != 0 && dm_mode != 1) return RIJK_ERR_ARG;
  if (num_basis > 46000) return RIJK_ERR_TOO_LARGE;
  const rijk::Geom g = rijk::make_geom(num_basis, num_auxbas);
  // Scratch layout: W [spin][ldB] | w [spin][naux] (rounded to 32) | Jpart [spin][ldB]
  const int64_t w_off = spin_channel * g.ldB;
  const int64_t jp_off = w_off + ((spin_channel * g.naux + 31) / 32) * 32;
  const int64_t need = jp_off + spin_channel * g.ldB;
  if (need > (int64_t)kScratchDoubles) return RIJK_ERR_TOO_LARGE;
  if (row_stride != g.ldB) return RIJK_ERR_ARG;
  // An error left pending by the caller's own work is not this call's to
  // clear: report it and leave it for the caller's check.
  if (cudaPeekAtLastError() != cudaSuccess) return RIJK_ERR_CUDA;
  double* s = nullptr;
  const int st = scratch_on_current_device(&s);
  if (st != RIJK_OK) return st;
  // Pass 2 splits the aux rows over as many partial sums as the allocating
  // path uses, as far as the array has room for them (the same split count
  // gives the same summation order).
  const int64_t room = ((int64_t)kScratchDoubles - jp_off) / (spin_channel * g.ldB);
  const int splits = (int)std::max<int64_t>(1, std::min<int64_t>(rijk::j_pass2_splits(g), room));
  cudaStream_t cs = static_cast<cudaStream_t>(stream);
  double* W = s;
  double* w = s + w_off;
  double* Jp = s + jp_off;
  rijk::launch_j_weights(g, d_dm, spin_channel, dm_mode, W, nullptr, cs);
  if (cudaGetLastError() != cudaSuccess) return RIJK_ERR_CUDA;
  rijk::launch_j_pass1(g, d_tensor, W, spin_channel, w, cs);
  if (cudaGetLastError() != cudaSuccess) return RIJK_ERR_CUDA;
  rijk::launch_j_pass2(g, d_tensor, w, spin_channel, splits, Jp, cs);
  if (cudaGetLastError() != cudaSuccess) return RIJK_ERR_CUDA;
  rijk::launch_j_finalize(g, Jp, spin_channel, splits, scaling_factor, 0, d_vj, cs);
  if (cudaGetLastError() != cudaSuccess) return RIJK_ERR_CUDA;
  return RIJK_OK;
}
