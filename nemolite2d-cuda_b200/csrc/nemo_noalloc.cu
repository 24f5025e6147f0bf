// Allocation-free field checksums.
//
// Some callers cannot call cudaMalloc: a host program whose device memory is
// all owned by a pool it manages itself (a framework's caching allocator, a
// Fortran driver with a preallocated arena), or a time loop that must not
// pay cudaMalloc's implicit device synchronisation.  For them this file
// offers one entry point that computes the same checksums as nemo_checksums
// -- SUM(ABS(f(1:nx,1:ny))) with the identical fixed reduction order -- from
// plain device pointers, allocating nothing.  Its scratch (the per-row
// partial sums) is a fixed array inside the library, resident on every GPU
// that loads the library until the process exits.
#include <mutex>
#include <stdio.h>

#include "nemo_internal.h"

namespace {

constexpr int kMaxFields = 4;
constexpr int kMaxRows = NEMO_NOALLOC_MAX_ROWS;
constexpr int CT = 256;

// Row partial sums of up to kMaxFields fields: 4 x 16384 doubles = 512 KiB.
// Every call shares it; each call writes every partial it later reads, so no
// element has to start at zero.
static __device__ __align__(256) double g_noalloc_rows[kMaxFields * kMaxRows];

// Host-side address of g_noalloc_rows on each device.  The name itself is a
// host stand-in, not a device address, so the address is looked up once per
// device with cudaGetSymbolAddress while that device is current.
constexpr int kMaxDevices = 64;
double* g_rows_ptr[kMaxDevices];
std::once_flag g_rows_once[kMaxDevices];
cudaError_t g_rows_err[kMaxDevices];

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
  return r;
}

struct FieldPtrs {
  const double* f[kMaxFields];
};

// pass 1: one block per (row, field); lane-strided partials, xor butterflies
__global__ void __launch_bounds__(CT) k_rows_noalloc(FieldPtrs F, int nx, int ny, long ld,
                                                     double* rows) {
  __shared__ double smem[CT / 32];
  const int jj = blockIdx.x;
  const double* a = F.f[blockIdx.y] + (long)jj * ld;
  double acc = 0.0;
  for (int k = threadIdx.x; k < nx; k += CT) acc = acc + fabs(a[k]);
  double r = block_sum(acc, smem);
  if (threadIdx.x == 0) rows[(long)blockIdx.y * kMaxRows + jj] = r;
}

// pass 2: one block per field over its ny row sums
__global__ void __launch_bounds__(CT) k_cols_noalloc(int ny, const double* rows, double* out) {
  __shared__ double smem[CT / 32];
  const double* a = rows + (long)blockIdx.x * kMaxRows;
  double acc = 0.0;
  for (int k = threadIdx.x; k < ny; k += CT) acc = acc + a[k];
  double r = block_sum(acc, smem);
  if (threadIdx.x == 0) out[blockIdx.x] = r;
}

}  // namespace

extern "C" int nemo_checksums_noalloc(const double* const* fields, int nfields, int nx, int ny,
                                      long ld, double* out, void* stream) {
  if (!fields || !out || nfields < 1 || nfields > kMaxFields || nx < 1 || ny < 1 || ld < nx)
    return NEMO_ERR_INVALID;
  if (ny > kMaxRows) {
    fprintf(stderr,
            "nemo_checksums_noalloc: %d rows exceed the fixed scratch of %d rows; "
            "use nemo_checksum instead\n", ny, kMaxRows);
    return NEMO_ERR_INVALID;
  }
  for (int k = 0; k < nfields; ++k)
    if (!fields[k]) return NEMO_ERR_INVALID;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return NEMO_ERR_CUDA;
  if (dev < 0 || dev >= kMaxDevices) return NEMO_ERR_UNSUPPORTED;
  // set-up on this device's first call, with this device current
  std::call_once(g_rows_once[dev], [dev]() {
    g_rows_err[dev] = cudaGetSymbolAddress(reinterpret_cast<void**>(&g_rows_ptr[dev]),
                                           g_noalloc_rows);
  });
  if (g_rows_err[dev] != cudaSuccess || !g_rows_ptr[dev]) return NEMO_ERR_CUDA;
  FieldPtrs F{};
  for (int k = 0; k < nfields; ++k) F.f[k] = fields[k];
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  k_rows_noalloc<<<dim3((unsigned)ny, (unsigned)nfields), CT, 0, s>>>(F, nx, ny, ld, g_rows_ptr[dev]);
  k_cols_noalloc<<<nfields, CT, 0, s>>>(ny, g_rows_ptr[dev], out);
  e = cudaGetLastError();
  return e == cudaSuccess ? NEMO_OK : NEMO_ERR_CUDA;
}
