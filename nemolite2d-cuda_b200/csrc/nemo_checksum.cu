// Field checksums SUM(ABS(f(1:jpi,1:jpj))) (field_mod.f90:935-956), as the
// reference prints them after the time loop (original/nemolite2d.f90:82-85).
//
// The reduction order is fixed and independent of the step kernel's tiling:
// pass 1 reduces each row with one 256-thread block (lane-strided partials in
// ascending index, then an xor butterfly inside each warp and across the 8
// warp sums); pass 2 reduces the column of row sums the same way.  The
// oracle reproduces this order exactly.
#include "nemo_internal.h"

namespace nemo {
namespace {

constexpr int CT = 256;

__device__ __forceinline__ double block_sum(double acc, double* smem) {
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1) acc = acc + __shfl_xor_sync(0xffffffffu, acc, off);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) smem[warp] = acc;
  __syncthreads();
  double r = 0.0;
  if (warp == 0) {
    double x = (lane < CT / 32) ? smem[lane] : 0.0;
#pragma unroll
    for (int off = CT / 64; off >= 1; off >>= 1) x = x + __shfl_xor_sync(0xffffffffu, x, off);
    r = x;
  }
  return r;  // valid in thread 0
}

struct FieldList {
  const double* f[4];
};

__global__ void __launch_bounds__(CT) k_row_sums(Layout L, FieldList F, double* partials) {
  __shared__ double smem[CT / 32];
  const int jj = 1 + blockIdx.x;
  const double* a = F.f[blockIdx.y] + L.idx(1, jj);
  double acc = 0.0;
  for (int k = threadIdx.x; k < L.jpi; k += CT) acc = acc + fabs(a[k]);
  double r = block_sum(acc, smem);
  if (threadIdx.x == 0) partials[(long)blockIdx.y * L.jpj + (jj - 1)] = r;
}

__global__ void __launch_bounds__(CT) k_col_sum(int n, const double* partials, double* out) {
  __shared__ double smem[CT / 32];
  const double* a = partials + (long)blockIdx.x * n;
  double acc = 0.0;
  for (int k = threadIdx.x; k < n; k += CT) acc = acc + a[k];
  double r = block_sum(acc, smem);
  if (threadIdx.x == 0) out[blockIdx.x] = r;
}

}  // namespace

cudaError_t launch_checksums(const Layout& L, const double* const* fields, int nf,
                             double* row_partials, double* out, cudaStream_t s) {
  if (nf < 1 || nf > 4) return cudaErrorInvalidValue;
  FieldList F{};
  for (int k = 0; k < nf; ++k) F.f[k] = fields[k];
  k_row_sums<<<dim3((unsigned)L.jpj, (unsigned)nf), CT, 0, s>>>(L, F, row_partials);
  k_col_sum<<<nf, CT, 0, s>>>(L.jpj, row_partials, out);
  return cudaGetLastError();
}

}  // namespace nemo
