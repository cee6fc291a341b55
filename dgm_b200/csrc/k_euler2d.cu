// Euler 2-D kernel instantiations (Quad, FP64), p = 1..8, q = p+1 and p+2.
#include "dispatch.cuh"

namespace dgmx {
namespace {
struct RegEuler2D {
  RegEuler2D() {
#define R(P) reg<DGMX_EULER2D, P, P + 1>(); reg<DGMX_EULER2D, P, P + 2>();
    R(1) R(2) R(3) R(4) R(5) R(6) R(7) R(8)
#undef R
  }
} reg_euler2d;
}  // namespace
}  // namespace dgmx
