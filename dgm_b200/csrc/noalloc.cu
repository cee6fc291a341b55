// Domain::time_derivative without any device allocation on the call path.
//
// Some callers cannot call cudaMalloc when they need the RHS: a real-time
// solver loop may forbid allocation (an allocation can synchronise the
// device and takes unbounded time), and a caller whose device memory is
// owned by an arena (for example a framework's caching allocator, or a
// solver that sizes all its memory once at start-up) must not grow the
// footprint behind that arena's back.  For them,
// dgmx_time_derivative_static evaluates F = -dU/dt with the face traces --
// the only scratch the RHS needs beyond its input and output -- held in a
// file-scope device array of fixed size instead of a buffer allocated with
// the handle.  The call is made from an ordinary host thread: it does call
// the CUDA runtime (cudaSetDevice, two kernel launches, cudaGetLastError,
// and on its first use on a device cudaGetSymbolAddress), so it is not for
// contexts where CUDA API calls are forbidden, such as host functions
// enqueued with cudaLaunchHostFunc.
//
// Limits and sharing:
//  * the array holds kStaticTraceDoubles doubles (8 MiB) per device;
//  * the first call on a device resolves the array's address with
//    cudaGetSymbolAddress with that device current.  Under lazy module
//    loading (CUDA_MODULE_LOADING=LAZY, the default since CUDA 12.2) that
//    is when the module holding the array is loaded and its 8 MiB are
//    reserved on that device; they stay reserved until the process exits.
//    A caller that needs every later call to be allocation-free makes one
//    call at set-up time, and makes it before any stream capture;
//  * a mesh needing more trace storage (ne * faces * fields * side points)
//    is rejected with DGMX_ERR_ARGUMENT and nothing is enqueued;
//  * all calls on one device share the array and it keeps the last call's
//    contents; nothing in it needs to start at zero (the trace kernel writes
//    every entry before the RHS kernel reads it), but calls that overlap on
//    the GPU (two streams, two handles) race on it;
//  * partitioned handles (dgmx_create_partition) and Navier-Stokes return
//    DGMX_ERR_UNSUPPORTED.
#include <cstdio>
#include <mutex>
#include <string>

#include "dgmx_internal.hpp"

namespace {

constexpr size_t kStaticTraceDoubles = size_t(1) << 20;
constexpr int kMaxDevices = 64;

// In host code this name is only a stand-in for the symbol; the device
// address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) double g_trace_scratch[kStaticTraceDoubles];

std::mutex g_mu;
double *g_addr[kMaxDevices] = {};

// Device address of g_trace_scratch on `dev` (which must be current).
cudaError_t scratch_address(int dev, double **out) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_addr[dev]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_trace_scratch);
    if (e != cudaSuccess) return e;
    g_addr[dev] = static_cast<double *>(p);
  }
  *out = g_addr[dev];
  return cudaSuccess;
}

}  // namespace

extern "C" dgmx_status dgmx_time_derivative_static(dgmx_domain *d, const double *U_dev, double *F_dev) {
  dgmx::DomainView v;
  bool partitioned = false;
  std::string *err = nullptr;
  if (!dgmx::domain_view(d, &v, &partitioned, &err)) {
    if (partitioned && err) {
      *err = "the static-scratch RHS covers whole domains; a partitioned handle exchanges halo traces "
             "through the handle's buffers (use dgmx_time_derivative_device)";
      return DGMX_ERR_UNSUPPORTED;
    }
    return DGMX_ERR_ARGUMENT;
  }
  if (!U_dev || !F_dev) {
    *v.errmsg = "null device buffer";
    return DGMX_ERR_ARGUMENT;
  }
  if (v.base.V) {
    *v.errmsg = "the static-scratch RHS covers Euler and shallow water; Navier-Stokes needs the handle's "
                "viscous work buffers (use dgmx_time_derivative_device)";
    return DGMX_ERR_UNSUPPORTED;
  }
  if (v.device < 0 || v.device >= kMaxDevices) {
    *v.errmsg = "device ordinal out of range for the static trace scratch";
    return DGMX_ERR_ARGUMENT;
  }
  if (v.ntrace > kStaticTraceDoubles) {
    char buf[200];
    std::snprintf(buf, sizeof(buf),
                  "face traces need %zu doubles, above the static scratch maximum of %zu doubles (8 MiB)",
                  v.ntrace, kStaticTraceDoubles);
    *v.errmsg = buf;
    return DGMX_ERR_ARGUMENT;
  }
  cudaError_t e = cudaSetDevice(v.device);
  double *scratch = nullptr;
  if (e == cudaSuccess) e = scratch_address(v.device, &scratch);
  if (e != cudaSuccess) {
    *v.errmsg = std::string("static trace scratch: ") + cudaGetErrorString(e);
    return DGMX_ERR_CUDA;
  }
  dgmx::StageArgs a = v.base;
  a.Xn = U_dev;
  a.Fn = F_dev;
  a.Tout = scratch;
  e = v.ops->traces_nodal(a, v.stream);
  ++*v.launches;
  if (e != cudaSuccess) {
    *v.errmsg = std::string("nodal trace kernel: ") + cudaGetErrorString(e);
    return DGMX_ERR_CUDA;
  }
  a.Tin = scratch;
  if (v.sw_balance) {
    if (!*v.sw_captured) { a.Rcap = v.Rsw; *v.sw_captured = true; }
    a.Rsub = v.Rsw;
  }
  e = v.ops->rhs_nodal(a, v.stream);
  ++*v.launches;
  if (e != cudaSuccess) {
    *v.errmsg = std::string("nodal rhs kernel: ") + cudaGetErrorString(e);
    return DGMX_ERR_CUDA;
  }
  return DGMX_OK;
}
