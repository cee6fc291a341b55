// Mixed-precision tiles (FP32 working precision, FP64 solution register):
// Euler 3-D p = 1..7 (q = p+2), Euler 2-D and shallow water p = 1..8
// (q = p+1, p+2).  LSRK14 only.
#include "dispatch.cuh"

namespace dgmx {
namespace {
struct RegMixed {
  RegMixed() {
#define R3(P) reg<DGMX_EULER3D, P, P + 2, true>();
    R3(1) R3(2) R3(3) R3(4) R3(5) R3(6)
#undef R3
    // p = 7: 512 threads instead of one per point (736 threads at 80
    // registers spill 132 bytes); registered first, the default
    reg_variant<DGMX_EULER3D, 7, 9, 1, 0, true, 512>();
    reg<DGMX_EULER3D, 7, 9, true>();
#define R3B(P) reg2<DGMX_EULER3D, P, P + 2, true>();
    R3B(2) R3B(3) R3B(4) R3B(5)
#undef R3B
#define R2(P) reg<DGMX_EULER2D, P, P + 1, true>(); reg<DGMX_EULER2D, P, P + 2, true>(); \
              reg<DGMX_SHALLOW, P, P + 1, true>(); reg<DGMX_SHALLOW, P, P + 2, true>();
    R2(1) R2(2) R2(3) R2(4) R2(5) R2(6) R2(7) R2(8)
#undef R2
  }
} reg_mixed;
}  // namespace
}  // namespace dgmx
