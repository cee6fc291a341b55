// Navier-Stokes 3-D kernel instantiations (Hex, FP64, BR1), p = 1..7, q = p+2 (and p+1 from p = 2).
#include "dispatch.cuh"

namespace dgmx {
namespace {
struct RegNS3D {
  RegNS3D() {
    reg<DGMX_NS3D, 1, 3>();
#define R(P) reg<DGMX_NS3D, P, P + 1>(); reg<DGMX_NS3D, P, P + 2>();
    R(2) R(3) R(4) R(5) R(6) R(7)
#undef R
  }
} reg_ns3d;
}  // namespace
}  // namespace dgmx
