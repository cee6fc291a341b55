// Kernel registry and small utility kernels.
#include <map>
#include <mutex>
#include <tuple>

#include "dgmx_internal.hpp"

namespace dgmx {
namespace {
std::map<std::tuple<int, int, int>, std::vector<KernelOps>> &table() {
  static std::map<std::tuple<int, int, int>, std::vector<KernelOps>> t;
  return t;
}
std::mutex &table_mutex() {
  static std::mutex m;
  return m;
}
}  // namespace

void register_ops(int physics, int L, int Q, const KernelOps &ops) {
  std::lock_guard<std::mutex> lk(table_mutex());
  table()[std::make_tuple(physics, L, Q)].push_back(ops);
}

const KernelOps *find_ops(int physics, int L, int Q) {
  std::lock_guard<std::mutex> lk(table_mutex());
  auto it = table().find(std::make_tuple(physics, L, Q));
  if (it == table().end() || it->second.empty()) return nullptr;
  // the default is the first plain CTA tile (it handles every stage kind and
  // boundary sides), whatever order the compilation units registered in
  for (const KernelOps &o : it->second)
    if (o.warp == 0) return &o;
  return &it->second.front();
}

const std::vector<KernelOps> *find_variants(int physics, int L, int Q) {
  std::lock_guard<std::mutex> lk(table_mutex());
  auto it = table().find(std::make_tuple(physics, L, Q));
  return it == table().end() ? nullptr : &it->second;
}

void list_ops(std::vector<std::vector<int>> &out) {
  std::lock_guard<std::mutex> lk(table_mutex());
  for (auto &kv : table())
    for (auto &o : kv.second)
      out.push_back({std::get<0>(kv.first), std::get<1>(kv.first), std::get<2>(kv.first), o.epb, o.nt,
                     (int)o.smem, o.minb});
}

// out[n] = c_d * sum_e J_e Um[e][n][0]: the integral of field n (the
// orthonormal mode 0 carries the element mean).  One block per field,
// FP64 tree reduction.
__global__ void integrals_kernel(int nf, int ne, int ld, double c_d, const double *Um, const double *J,
                                 double *out) {
  __shared__ double red[256];
  const int n = blockIdx.x;
  double acc = 0.0;
  for (int e = threadIdx.x; e < ne; e += blockDim.x) acc += J[e] * Um[((size_t)e * nf + n) * ld];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[n] = c_d * red[0];
}

cudaError_t launch_integrals(int nf, int ne, int ld, double c_d, const double *Um, const double *J, double *out,
                             cudaStream_t s) {
  integrals_kernel<<<nf, 256, 0, s>>>(nf, ne, ld, c_d, Um, J, out);
  return cudaGetLastError();
}

// The mixed form's reference integrals (order in dgmx_internal.hpp): one
// block of kRefLanes threads per field; products and sums rounded on
// their own so that no contraction changes the order's result.
__global__ void reference_integrals_kernel(int nf, int ne, int ld, double c_d, const double *Um, const double *J,
                                           double *out) {
  __shared__ double red[kRefLanes];
  const int n = blockIdx.x, l = threadIdx.x;
  double acc = 0.0;
  for (int e = l; e < ne; e += kRefLanes) acc = __dadd_rn(acc, __dmul_rn(J[e], Um[((size_t)e * nf + n) * ld]));
  red[l] = acc;
  __syncthreads();
  for (int s = kRefLanes / 2; s > 0; s >>= 1) {
    if (l < s) red[l] = __dadd_rn(red[l], red[l + s]);
    __syncthreads();
  }
  if (l == 0) out[n] = __dmul_rn(c_d, red[0]);
}

cudaError_t launch_reference_integrals(int nf, int ne, int ld, double c_d, const double *Um, const double *J,
                                       double *out, cudaStream_t s) {
  reference_integrals_kernel<<<nf, kRefLanes, 0, s>>>(nf, ne, ld, c_d, Um, J, out);
  return cudaGetLastError();
}

// out[e][n] = J_e * Um[e][n][0], rounded as reference_integrals_kernel does.
__global__ void element_integrands_kernel(int nf, int ne, int ld, const double *Um, const double *J, double *out) {
  const long long total = (long long)ne * nf;
  for (long long w = (long long)blockIdx.x * blockDim.x + threadIdx.x; w < total;
       w += (long long)gridDim.x * blockDim.x) {
    const int e = (int)(w / nf);
    out[w] = __dmul_rn(J[e], Um[(size_t)w * ld]);
  }
}

cudaError_t launch_element_integrands(int nf, int ne, int ld, const double *Um, const double *J, double *out,
                                      cudaStream_t s) {
  if (ne <= 0) return cudaSuccess;
  const long long b = ((long long)ne * nf + 255) / 256;
  element_integrands_kernel<<<(int)(b < 4 * 148 ? b : 4 * 148), 256, 0, s>>>(nf, ne, ld, Um, J, out);
  return cudaGetLastError();
}

// One thread: the domain means integ / vol and the derived reference row.
__global__ void reference_row_kernel(int physics, int nf, double gamma, double phi0, double vol,
                                     const double *integ, double *uref) {
  double h[kUrefStride];
  for (int k = 0; k < kUrefStride; ++k) h[k] = 0.0;
  for (int n = 0; n < nf; ++n) h[n] = integ[n] / vol;
  fill_reference_row(physics, gamma, phi0, h);
  for (int k = 0; k < kUrefStride; ++k) uref[k] = h[k];
}

cudaError_t launch_reference_row(int physics, int nf, double gamma, double phi0, double vol, const double *integ,
                                 double *uref, cudaStream_t s) {
  reference_row_kernel<<<1, 1, 0, s>>>(physics, nf, gamma, phi0, vol, integ, uref);
  return cudaGetLastError();
}

}  // namespace dgmx
