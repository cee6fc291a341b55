// Halo exchange of face traces between element partitions: gather the face
// blocks a peer needs into a contiguous send buffer, scatter a received
// buffer into the ghost slots.  A block is the blk values of one
// (element, face) pair in the [element][face][field][point] trace layout
// (the contiguous run the reference's Side::u holds per side and field,
// exchanged in src/vField.cpp:146-200): FP64 traces, or the mixed form's
// FP32 ones, whose blocks sit in the buffer at an even stride bs >= blk so
// that every block is a whole number of doubles on the wire.
#include "dgmx_internal.hpp"

namespace dgmx {
namespace {

template <class V>
__global__ void pack_kernel(const V *__restrict__ T, const int *__restrict__ idx, int n, int blk, int bs,
                            V *__restrict__ buf) {
  const long long total = (long long)n * blk;
  for (long long w = (long long)blockIdx.x * blockDim.x + threadIdx.x; w < total;
       w += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(w / blk), k = (int)(w - (long long)i * blk);
    buf[(size_t)i * bs + k] = T[(size_t)idx[i] * blk + k];
  }
}

template <class V>
__global__ void unpack_kernel(const V *__restrict__ buf, const int *__restrict__ idx, int n, int blk, int bs,
                              V *__restrict__ T) {
  const long long total = (long long)n * blk;
  for (long long w = (long long)blockIdx.x * blockDim.x + threadIdx.x; w < total;
       w += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(w / blk), k = (int)(w - (long long)i * blk);
    T[(size_t)idx[i] * blk + k] = buf[(size_t)i * bs + k];
  }
}

int grid_for(long long total) {
  const long long b = (total + 255) / 256;
  return (int)(b < 4 * 148 ? (b > 0 ? b : 1) : 4 * 148);
}

}  // namespace

cudaError_t launch_pack(const double *T, const int *idx, int n, int blk, double *buf, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  pack_kernel<<<grid_for((long long)n * blk), 256, 0, s>>>(T, idx, n, blk, blk, buf);
  return cudaGetLastError();
}

cudaError_t launch_unpack(const double *buf, const int *idx, int n, int blk, double *T, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  unpack_kernel<<<grid_for((long long)n * blk), 256, 0, s>>>(buf, idx, n, blk, blk, T);
  return cudaGetLastError();
}

cudaError_t launch_pack(const float *T, const int *idx, int n, int blk, int bs, float *buf, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  pack_kernel<<<grid_for((long long)n * blk), 256, 0, s>>>(T, idx, n, blk, bs, buf);
  return cudaGetLastError();
}

cudaError_t launch_unpack(const float *buf, const int *idx, int n, int blk, int bs, float *T, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  unpack_kernel<<<grid_for((long long)n * blk), 256, 0, s>>>(buf, idx, n, blk, bs, T);
  return cudaGetLastError();
}

}  // namespace dgmx
