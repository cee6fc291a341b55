// Second-form stage kernels (stage2.cuh) of Euler 3-D, FP64 and the mixed
// form, p = 2..5 at q = p+2.  Registered after the plain tiles of the same
// (p, q), so the default tile is unchanged; dgmx_autotune picks among all.
#include "dispatch.cuh"

namespace dgmx {
namespace {
struct RegEuler3D2 {
  RegEuler3D2() {
#define R(P) reg2<DGMX_EULER3D, P, P + 2>(); reg2<DGMX_EULER3D, P, P + 2, true>();
    R(2) R(3) R(4) R(5)
#undef R
  }
} reg_euler3d2;
}  // namespace
}  // namespace dgmx
