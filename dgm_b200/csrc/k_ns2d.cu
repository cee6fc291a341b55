// Navier-Stokes 2-D kernel instantiations (Quad, FP64, BR1), p = 1..8.
#include "dispatch.cuh"

namespace dgmx {
namespace {
struct RegNS2D {
  RegNS2D() {
#define R(P) reg<DGMX_NS2D, P, P + 1>(); reg<DGMX_NS2D, P, P + 2>();
    R(1) R(2) R(3) R(4) R(5) R(6) R(7) R(8)
#undef R
  }
} reg_ns2d;
}  // namespace
}  // namespace dgmx
