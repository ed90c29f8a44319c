// One three-centre integral class (RIJK_LA RIJK_LB | RIJK_LC) of
// rijk_ints_dev.cuh, with this translation unit's table loader.  The library
// build compiles this file once per class (45 objects), so the long compiles of
// the unrolled classes run in parallel.
#include "rijk_ints_dev.cuh"

#ifndef RIJK_LA
#define RIJK_LA 0
#define RIJK_LB 0
#define RIJK_LC 0
#endif

namespace rijk {
namespace intsdev {

#define RIJK_CLS_NAME2(p, a, b, c) p##a##b##c
#define RIJK_CLS_NAME(p, a, b, c) RIJK_CLS_NAME2(p, a, b, c)

Int3cKernel RIJK_CLS_NAME(int3c_kernel_, RIJK_LA, RIJK_LB, RIJK_LC)() {
  return k_int3c2e_cls<RIJK_LA, RIJK_LB, RIJK_LC>;
}
int RIJK_CLS_NAME(int3c_tables_, RIJK_LA, RIJK_LB, RIJK_LC)(const double* flat, const int* off, const double* boys) {
  return upload_tables(flat, off, boys);
}

}  // namespace intsdev
}  // namespace rijk
