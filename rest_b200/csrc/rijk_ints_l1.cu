// Three-centre integral kernels (rijk_ints_dev.cuh) for AO shell pairs whose
// first shell has l = 1, with this translation unit's table loader.
#include "rijk_ints_dev.cuh"

namespace rijk {
namespace intsdev {

Int3cKernel int3c_kernel_la1(int lb, int lc) { return class_kernel<1>(lb, lc); }
int int3c_tables_la1(const double* flat, const int* off, const double* boys) {
  return upload_tables(flat, off, boys);
}

}  // namespace intsdev
}  // namespace rijk
