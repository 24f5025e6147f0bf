// 3x3 convolutions of the BF16 surrogate on the 5th-generation tensor cores
// (tcgen05 MMA, accumulators in tensor memory, operands staged by TMA).
//
// Activations are NHWC BF16 with 64 channels.  Weights are [tap][cout][cin]
// BF16 (tap = 3*(dy+1) + (dx+1)); FP32 accumulation throughout.
//
// k_conv_fwd -- implicit GEMM out[p, co] = sum_{tap,ci} x[p+off(tap), ci] *
//   w[tap, co, ci], M = 128 pixels of one image row, N = 64, K = 9 x 64.  For
//   every tap a TMA load brings the shifted 128 x 64 window into shared memory
//   (coordinates outside the image are zero-filled, which is the convolution's
//   zero padding); both operands are K-major with the 128-byte swizzle.  Warp 0
//   issues TMA, one thread of warp 1 issues the MMAs, warps 2-5 drain the
//   double-buffered accumulator and apply the fused epilogue: + bias, ReLU,
//   + residual, x (mask > 0).  The same kernel computes the data gradient of a
//   convolution when given the tap-flipped, transposed weights.
//
// k_conv_wgrad -- dw[tap, co, ci] += sum_p dz[p, co] * x[p+off(tap), ci] as
//   D[(tap pair, ci), co] with K = pixels: M = 128 rows (two taps x 64 input
//   channels), N = 64.  Both operands come straight from the NHWC tensors by
//   TMA and are read by the MMA as MN-major (channels contiguous); CTAs split
//   the pixel range and add their partial D into an FP32 dw with atomics.
//
// These two are the first forms; the defaults are k_conv_fwd_tri (three output
// rows per N = 192 MMA, outputs written by TMA stores) and k_conv_wgrad_strip
// (all nine taps per CTA over column strips, partial sums added in a fixed
// order by k_wgrad_reduce), described where they are defined.
//
// Every wait on an mbarrier is bounded; on timeout the kernel records an
// error code, lets in-flight copies and MMAs finish (also bounded), frees its
// tensor memory and returns.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>
#include <stdint.h>
#include <stdio.h>

#include <atomic>
#include <mutex>

#include "nemo_mbar.cuh"
#include "sur_internal.h"

namespace sur {
namespace {

constexpr int CH = 64;
constexpr int TM = 128;                    // pixels per forward tile
constexpr int NST = 4;                     // forward A stages (one tap each)
constexpr int A_BYTES = TM * CH * 2;       // 16 KiB
constexpr int WT_BYTES = CH * CH * 2;      // 8 KiB per tap
constexpr int W_BYTES = 9 * WT_BYTES;      // 72 KiB
constexpr int THREADS = 192;               // 6 warps
constexpr uint64_t WAIT_NS = 2000000000ull;  // 2 s per wait before giving up

constexpr int WG_NST = 4;                  // wgrad stages
constexpr int WG_PIX = 64;                 // pixels per wgrad K chunk
constexpr int WG_TILE = WG_PIX * CH * 2;   // 8 KiB

// ---- PTX wrappers ------------------------------------------------------------
using devsync::fence_barrier_init;
using devsync::mbar_arrive;
using devsync::mbar_expect_tx;
using devsync::mbar_init;
using devsync::mbar_try;
using devsync::smem_u32;
// Bounded wait for the phase with the given parity; false after `limit` ns
// (WAIT_NS by default) of wall time without completion.
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity, uint64_t limit = WAIT_NS) {
  return devsync::mbar_wait(b, parity, limit);
}
// The same, agreed across the warp (for .sync.aligned tcgen05 instructions).
__device__ __forceinline__ bool mbar_wait_warp(uint64_t* b, uint32_t parity, uint64_t limit = WAIT_NS) {
  return __all_sync(0xffffffffu, mbar_wait(b, parity, limit)) != 0;
}
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* tm, uint64_t* bar, int c0,
                                            int c1) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_u32(dst)),
      "l"(tm), "r"(c0), "r"(c1), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* tm, uint64_t* bar, int c0,
                                            int c1, int c2, int c3) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(
          smem_u32(dst)),
      "l"(tm), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void mma_bf16(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc,
                                         uint32_t accum) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(idesc), "r"(accum)
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}
// 32 consecutive fp32 columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
        "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
        "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
        "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// Shared-memory matrix descriptor (tcgen05): start, leading and stride byte
// offsets in 16-byte units, descriptor version 1, 128-byte swizzle.
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46) | (2ull << 61);
}

// Instruction descriptor, kind::f16: D f32, A and B bf16, M x N, operand
// majorness (0 K-major, 1 MN-major).
__host__ __device__ constexpr uint32_t idesc(int M, int N, int a_mn, int b_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
         ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

struct FwdSmem {
  uint8_t a[NST][A_BYTES];
  uint8_t w[W_BYTES];
  uint64_t full[NST], empty[NST];
  uint64_t wbar, done;
  uint64_t tfull[2], tempty[2];
  uint32_t tmem_base;
  float bias[CH];
};

__device__ __forceinline__ void fail(int* err, int code) { atomicCAS(err, 0, code); }

// Epilogue of one 128-pixel output tile for this thread's pixel `row`:
// v = acc (64 fp32 values) + bias, + residual, *(mask > 0), relu; the FP32
// output; the BF16 output is left to the caller.
__device__ __forceinline__ void epilogue_math(const ConvEpi& E, const float* bias, float* v, long p) {
#pragma unroll
  for (int c = 0; c < 64; ++c) v[c] += bias[c];
  if (E.residual) {
    const uint4* rp = reinterpret_cast<const uint4*>(E.residual + p * CH);
#pragma unroll
    for (int g = 0; g < 8; ++g) {
      uint4 u = rp[g];
      const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        float2 f = __bfloat1622float2(h[e]);
        v[8 * g + 2 * e] += f.x;
        v[8 * g + 2 * e + 1] += f.y;
      }
    }
  }
  if (E.mask) {
    const uint4* mp = reinterpret_cast<const uint4*>(E.mask + p * CH);
#pragma unroll
    for (int g = 0; g < 8; ++g) {
      uint4 u = mp[g];
      const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        float2 f = __bfloat1622float2(h[e]);
        if (!(f.x > 0.0f)) v[8 * g + 2 * e] = 0.0f;
        if (!(f.y > 0.0f)) v[8 * g + 2 * e + 1] = 0.0f;
      }
    }
  }
  if (E.relu) {
#pragma unroll
    for (int c = 0; c < 64; ++c) v[c] = fmaxf(v[c], 0.0f);
  }
  if (E.out32) {
    const int nq = E.out32_ch > 0 ? E.out32_ch >> 2 : 1;
    float4* o32 = reinterpret_cast<float4*>(E.out32 + p * (4 * nq));
#pragma unroll
    for (int g = 0; g < 16; ++g)
      if (g < nq) o32[g] = make_float4(v[4 * g], v[4 * g + 1], v[4 * g + 2], v[4 * g + 3]);
  }
}

// Eight 16-byte groups of BF16 channels (8 channels each) of one pixel.
__device__ __forceinline__ uint4 bf16x8(const float* v, int g) {
  uint4 u;
  __nv_bfloat162* h = reinterpret_cast<__nv_bfloat162*>(&u);
#pragma unroll
  for (int e = 0; e < 4; ++e) h[e] = __floats2bfloat162_rn(v[8 * g + 2 * e], v[8 * g + 2 * e + 1]);
  return u;
}

// The whole epilogue with the BF16 output stored by this thread.
__device__ __forceinline__ void epilogue_store(const ConvEpi& E, const float* bias, float* v, long p) {
  epilogue_math(E, bias, v, p);
  if (E.out) {
    uint4* op = reinterpret_cast<uint4*>(E.out + p * CH);
#pragma unroll
    for (int g = 0; g < 8; ++g) op[g] = bf16x8(v, g);
  }
}

// TMA store of a 64-channel x 32-pixel BF16 tile staged in shared memory
// (128-byte swizzle, as the tensor map's), and the bulk-group bookkeeping.
__device__ __forceinline__ void tma_store_4d(const CUtensorMap* tm, const void* src, int c0, int c1, int c2,
                                             int c3) {
  asm volatile("cp.async.bulk.tensor.4d.global.shared::cta.bulk_group [%0, {%2, %3, %4, %5}], [%1];" ::"l"(tm),
               "r"(smem_u32(src)), "r"(c0), "r"(c1), "r"(c2), "r"(c3)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// at most one group still reading its shared-memory source
__device__ __forceinline__ void bulk_wait_read1() { asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }


__global__ void __launch_bounds__(THREADS, 1)
k_conv_fwd(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmW,
           ConvEpi E) {
  extern __shared__ uint8_t smem_raw[];
  FwdSmem& S = *reinterpret_cast<FwdSmem*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int xtiles = E.W / TM;
  const int ntile = E.N * E.H * xtiles;

  if (threadIdx.x == 0) {
    for (int s = 0; s < NST; ++s) {
      mbar_init(&S.full[s], 1);
      mbar_init(&S.empty[s], 1);
    }
    mbar_init(&S.wbar, 1);
    mbar_init(&S.done, 1);
    for (int b = 0; b < 2; ++b) {
      mbar_init(&S.tfull[b], 1);
      mbar_init(&S.tempty[b], 128);
    }
    fence_barrier_init();
  }
  if (threadIdx.x < CH) S.bias[threadIdx.x] = E.bias ? E.bias[threadIdx.x] : 0.0f;
  if (warp == 1) tmem_alloc(&S.tmem_base, 128);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = S.tmem_base;

  if (warp == 0 && lane == 0) {
    // ---- TMA producer ----
    mbar_expect_tx(&S.wbar, W_BYTES);
    for (int tap = 0; tap < 9; ++tap) tma_load_2d(S.w + tap * WT_BYTES, &tmW, &S.wbar, 0, tap * CH);
    int stage = 0;
    uint32_t phase = 0;
    bool ok = true;
    for (int t = blockIdx.x; t < ntile && ok; t += gridDim.x) {
      const int xt = t % xtiles, r = t / xtiles, y = r % E.H, n = r / E.H;
      for (int tap = 0; tap < 9; ++tap) {
        if (!mbar_wait(&S.empty[stage], phase ^ 1)) { fail(E.err, 1); ok = false; break; }
        mbar_expect_tx(&S.full[stage], A_BYTES);
        tma_load_4d(S.a[stage], &tmA, &S.full[stage], 0, xt * TM + (tap % 3) - 1, y + tap / 3 - 1, n);
        if (++stage == NST) { stage = 0; phase ^= 1; }
      }
    }
    // let every armed copy land before the CTA may exit
    for (int s = 0; s < NST; ++s) {
      // stages armed in the current phase round are s < stage; earlier ones completed
      if (s < stage) mbar_wait(&S.full[s], phase);
      else mbar_wait(&S.full[s], phase ^ 1);
    }
    mbar_wait(&S.wbar, 0);
  } else if (warp == 1 && lane == 0) {
    // ---- MMA issuer ----
    const uint32_t ID = idesc(128, 64, 0, 0);
    bool ok = mbar_wait(&S.wbar, 0);
    if (!ok) fail(E.err, 2);
    int stage = 0;
    uint32_t phase = 0;
    int it = 0;
    const uint32_t wbase = smem_u32(S.w);
    for (int t = blockIdx.x; t < ntile && ok; t += gridDim.x, ++it) {
      const int b = it & 1;
      const uint32_t tph = (it >> 1) & 1;
      if (!mbar_wait(&S.tempty[b], tph ^ 1)) { fail(E.err, 3); ok = false; break; }
      tc_fence_after();
      const uint32_t d = tmem + (uint32_t)(b * 64);
      for (int tap = 0; tap < 9; ++tap) {
        if (!mbar_wait(&S.full[stage], phase)) { fail(E.err, 4); ok = false; break; }
        tc_fence_after();
        const uint32_t abase = smem_u32(S.a[stage]);
#pragma unroll
        for (int k = 0; k < 4; ++k)
          mma_bf16(d, sdesc(abase + 32 * k, 16, 1024), sdesc(wbase + tap * WT_BYTES + 32 * k, 16, 1024), ID,
                   (tap | k) != 0);
        mma_commit(&S.empty[stage]);
        if (++stage == NST) { stage = 0; phase ^= 1; }
      }
      if (ok) mma_commit(&S.tfull[b]);
    }
    mma_commit(&S.done);  // completes once every MMA issued above has finished
    mbar_wait(&S.done, 0);
  } else if (warp >= 2) {
    // ---- epilogue: TMEM -> registers -> bias/ReLU/residual/mask -> BF16 ----
    const int q = warp & 3;
    const int row = 32 * q + lane;
    int it = 0;
    for (int t = blockIdx.x; t < ntile; t += gridDim.x, ++it) {
      const int b = it & 1;
      const uint32_t tph = (it >> 1) & 1;
      if (!mbar_wait_warp(&S.tfull[b], tph)) { fail(E.err, 5); break; }
      tc_fence_after();
      float v[64];
      const uint32_t ta = tmem + (uint32_t)(b * 64) + ((uint32_t)(32 * q) << 16);
      tmem_ld32(ta, v);
      tmem_ld32(ta + 32, v + 32);
      tc_fence_before();
      mbar_arrive(&S.tempty[b]);
      const int xt = t % xtiles, r = t / xtiles, y = r % E.H, n = r / E.H;
      const long p = ((long)(n * E.H + y) * E.W + xt * TM + row);
      epilogue_store(E, S.bias, v, p);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    __syncwarp();
    tc_fence_after();
    tmem_dealloc(tmem, 128);
  }
}

// ---- forward over column strips with a ring of input rows ------------------
// A CTA takes strips (image n, 128-column tile xt, rows y0 .. y0+R-1) and
// marches down them.  Each input row r is loaded once (TMA, 144 pixels
// x0-8 .. x0+135, zero-filled outside the image) into a ring slot and serves
// the three output rows r-1, r, r+1; the three horizontal taps of a row read
// the slot through descriptors starting at pixels 7, 8, 9.  The 128-byte
// swizzle is a function of the absolute shared-memory address (the phase of
// a row is address bits 7-9, as TMA wrote it), so a view may start on any
// 128-byte row with the base-offset field left at zero; the exact-shift
// tests check this on the device.  One 18 KiB load feeds 36 MMAs instead
// of 4.
constexpr int RW_PIX = 144;
constexpr int RW_BYTES = RW_PIX * CH * 2;  // 18 KiB, a multiple of 1024
constexpr int NSLOT = 8;

struct RowSmem {
  uint8_t slot[NSLOT][RW_BYTES];
  uint8_t w[W_BYTES];
  uint64_t full[NSLOT], empty[NSLOT];
  uint64_t wbar, done;
  uint64_t tfull[2], tempty[2];
  uint32_t tmem_base;
  float bias[CH];
};

__global__ void __launch_bounds__(THREADS, 1)
k_conv_fwd_rows(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmW,
                ConvEpi E, int R) {
  extern __shared__ uint8_t smem_raw[];
  RowSmem& S = *reinterpret_cast<RowSmem*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int xtiles = E.W / TM;
  const int ystrips = (E.H + R - 1) / R;
  const int nstrip = E.N * xtiles * ystrips;

  if (threadIdx.x == 0) {
    for (int s = 0; s < NSLOT; ++s) {
      mbar_init(&S.full[s], 1);
      mbar_init(&S.empty[s], 1);
    }
    mbar_init(&S.wbar, 1);
    mbar_init(&S.done, 1);
    for (int b = 0; b < 2; ++b) {
      mbar_init(&S.tfull[b], 1);
      mbar_init(&S.tempty[b], 128);
    }
    fence_barrier_init();
  }
  if (threadIdx.x < CH) S.bias[threadIdx.x] = E.bias ? E.bias[threadIdx.x] : 0.0f;
  if (warp == 1) tmem_alloc(&S.tmem_base, 128);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = S.tmem_base;

  if (warp == 0 && lane == 0) {
    // ---- TMA producer: rows y0-1 .. y1+1 of every strip, in order ----
    mbar_expect_tx(&S.wbar, W_BYTES);
    for (int tap = 0; tap < 9; ++tap) tma_load_2d(S.w + tap * WT_BYTES, &tmW, &S.wbar, 0, tap * CH);
    uint32_t L = 0;  // loads issued
    bool ok = true;
    for (int st = blockIdx.x; st < nstrip && ok; st += gridDim.x) {
      const int ys = st % ystrips, r0 = st / ystrips, xt = r0 % xtiles, n = r0 / xtiles;
      const int y0 = ys * R, y1 = min(y0 + R, E.H) - 1;
      for (int r = y0 - 1; r <= y1 + 1; ++r, ++L) {
        const int slot = (int)(L % NSLOT);
        const uint32_t ph = (L / NSLOT) & 1;
        if (!mbar_wait(&S.empty[slot], ph ^ 1)) { fail(E.err, 21); ok = false; break; }
        mbar_expect_tx(&S.full[slot], RW_BYTES);
        tma_load_4d(S.slot[slot], &tmA, &S.full[slot], 0, xt * TM - 8, r, n);
      }
    }
    // every armed load lands before the CTA may exit
    for (int s = 0; s < NSLOT; ++s) {
      const uint32_t armed = L / NSLOT + ((uint32_t)s < L % NSLOT ? 1u : 0u);
      if (armed) mbar_wait(&S.full[s], (armed - 1) & 1);
    }
    mbar_wait(&S.wbar, 0);
  } else if (warp == 1 && lane == 0) {
    // ---- MMA issuer ----
    const uint32_t ID = idesc(128, 64, 0, 0);
    bool ok = mbar_wait(&S.wbar, 0);
    if (!ok) fail(E.err, 22);
    const uint32_t wbase = smem_u32(S.w);
    uint32_t L = 0;       // loads consumed (index of the strip's first row)
    uint32_t waited = 0;  // loads whose full barrier has been waited for
    int it = 0;
    for (int st = blockIdx.x; st < nstrip && ok; st += gridDim.x) {
      const int ys = st % ystrips;
      const int y0 = ys * R, y1 = min(y0 + R, E.H) - 1;
      const int rows = y1 - y0 + 1;
      for (int i = 0; i < rows && ok; ++i, ++it) {
        // rows y0+i-1, y0+i, y0+i+1 are loads L+i, L+i+1, L+i+2
        while (waited <= L + i + 2) {
          if (!mbar_wait(&S.full[waited % NSLOT], (waited / NSLOT) & 1)) { fail(E.err, 23); ok = false; break; }
          ++waited;
        }
        if (!ok) break;
        const int b = it & 1;
        const uint32_t tph = (it >> 1) & 1;
        if (!mbar_wait(&S.tempty[b], tph ^ 1)) { fail(E.err, 24); ok = false; break; }
        tc_fence_after();
        const uint32_t d = tmem + (uint32_t)(b * 64);
#pragma unroll
        for (int dy = 0; dy < 3; ++dy) {
          const uint32_t sbase = smem_u32(S.slot[(L + i + dy) % NSLOT]);
#pragma unroll
          for (int dx = 0; dx < 3; ++dx) {
            const uint32_t a0 = sbase + (uint32_t)(7 + dx) * 128u;
            const uint32_t b0 = wbase + (uint32_t)(3 * dy + dx) * WT_BYTES;
#pragma unroll
            for (int k = 0; k < 4; ++k)
              mma_bf16(d, sdesc(a0 + 32 * k, 16, 1024), sdesc(b0 + 32 * k, 16, 1024), ID,
                       (dy | dx | k) != 0);
          }
        }
        mma_commit(&S.tfull[b]);
        mma_commit(&S.empty[(L + i) % NSLOT]);  // row y0+i-1 has had its last use
      }
      if (ok) {
        mma_commit(&S.empty[(L + rows) % NSLOT]);
        mma_commit(&S.empty[(L + rows + 1) % NSLOT]);
      }
      L += rows + 2;
    }
    mma_commit(&S.done);
    mbar_wait(&S.done, 0);
  } else if (warp >= 2) {
    // ---- epilogue ----
    const int q = warp & 3;
    const int row = 32 * q + lane;
    int it = 0;
    bool ok = true;
    for (int st = blockIdx.x; st < nstrip && ok; st += gridDim.x) {
      const int ys = st % ystrips, r0 = st / ystrips, xt = r0 % xtiles, n = r0 / xtiles;
      const int y0 = ys * R, y1 = min(y0 + R, E.H) - 1;
      for (int y = y0; y <= y1; ++y, ++it) {
        const int b = it & 1;
        const uint32_t tph = (it >> 1) & 1;
        if (!mbar_wait_warp(&S.tfull[b], tph)) { fail(E.err, 25); ok = false; break; }
        tc_fence_after();
        float v[64];
        const uint32_t ta = tmem + (uint32_t)(b * 64) + ((uint32_t)(32 * q) << 16);
        tmem_ld32(ta, v);
        tmem_ld32(ta + 32, v + 32);
        tc_fence_before();
        mbar_arrive(&S.tempty[b]);
        const long p = ((long)(n * E.H + y) * E.W + xt * TM + row);
        epilogue_store(E, S.bias, v, p);
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    __syncwarp();
    tc_fence_after();
    tmem_dealloc(tmem, 128);
  }
}

// ---- forward with three output rows per MMA -----------------------------------
// The row-ring kernel issues 36 MMAs of N = 64 (one output channel block) per
// output row, and those narrow MMAs keep the tensor pipe about half busy.
// Here the weights of the three vertical taps of one horizontal tap are laid
// side by side as one 192-row B operand (dy = -1, 0, +1), so each input row
// r, multiplied once per horizontal tap and K chunk, accumulates into the
// three output rows it feeds (r+1, r, r-1) with one N = 192 MMA: 12 MMAs per
// input row instead of 36.  The three accumulators must be adjacent in tensor
// memory: output row g of the CTA (counted across its strips) owns TMEM block
// (-g) mod 8 of 64 columns, so consecutive output rows sit in descending
// blocks and the three blocks of one input row are ascending; where they
// wrap past block 7 the MMA is split in two.  Every MMA accumulates: the
// epilogue zeroes a block after draining it (and all blocks start zeroed), so
// no MMA needs to know whether it is an accumulator's first.  Strip edges use
// N = 64 or 128 (an edge input row feeds one or two output rows of the
// strip).  An input row's ring slot is released as soon as its 12 MMAs are
// issued.
// NS input-row slots, NB accumulator blocks of 64 TMEM columns; the default
// (6, 8) runs one CTA per SM with all 512 columns, (2, 4) two CTAs per SM.
// OST: bytes of output staging (two 4 KiB tiles per epilogue warp when the
// BF16 output leaves by TMA stores).
template <int NS, int NB, int OST = 1024>
struct TriSmem {
  uint8_t slot[NS][RW_BYTES];
  uint8_t ost[OST];
  uint8_t w[W_BYTES];  // [dx][dy][64 co][64 ci]: per dx a 192 x 64 K-major B operand
  uint64_t full[NS], empty[NS];
  uint64_t wbar, done;
  uint64_t tfull[NB], tempty[NB];
  uint32_t tmem_base;
  float bias[CH];
};

template <int NB>
__device__ __forceinline__ uint32_t tblk(uint32_t g) { return (NB - (g & (NB - 1))) & (NB - 1); }

__device__ __forceinline__ void tmem_zero32(uint32_t taddr) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,"
      "%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1};" ::"r"(taddr),
      "r"(0u)
      : "memory");
}
__device__ __forceinline__ void tmem_st_wait() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// TS: each epilogue warp stages its 32 pixels' BF16 outputs in shared memory
// (two tiles alternating) and writes them with one TMA store per output row
// (tensor map tmO, box 64 channels x 32 pixels) instead of per-thread stores.
template <int NS, int NB, int MINB, bool TS>
__global__ void __launch_bounds__(THREADS, MINB)
k_conv_fwd_tri(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmW,
               const __grid_constant__ CUtensorMap tmO, ConvEpi E, int R) {
  extern __shared__ uint8_t smem_raw[];
  using Smem = TriSmem<NS, NB, TS ? 8 * 4096 : 1024>;
  Smem& S = *reinterpret_cast<Smem*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int xtiles = E.W / TM;
  const int ystrips = (E.H + R - 1) / R;
  const int nstrip = E.N * xtiles * ystrips;

  if (threadIdx.x == 0) {
    for (int s = 0; s < NS; ++s) {
      mbar_init(&S.full[s], 1);
      mbar_init(&S.empty[s], 1);
    }
    mbar_init(&S.wbar, 1);
    mbar_init(&S.done, 1);
    for (int b = 0; b < NB; ++b) {
      mbar_init(&S.tfull[b], 1);
      mbar_init(&S.tempty[b], 128);
    }
    fence_barrier_init();
  }
  if (threadIdx.x < CH) S.bias[threadIdx.x] = E.bias ? E.bias[threadIdx.x] : 0.0f;
  if (warp == 1) tmem_alloc(&S.tmem_base, 64 * NB);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = S.tmem_base;
  // main waits (operands, accumulator hand-over); the drains keep WAIT_NS
  const uint64_t LIM = E.wait_ns ? (uint64_t)E.wait_ns : WAIT_NS;
  if (warp >= 2) {  // every accumulator block starts at zero
    const uint32_t tl = tmem + ((uint32_t)(32 * (warp & 3)) << 16);
    for (int c = 0; c < 64 * NB; c += 32) tmem_zero32(tl + (uint32_t)c);
    tmem_st_wait();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();

  if (warp == 0 && lane == 0) {
    // ---- TMA producer: rows y0-1 .. y1+1 of every strip, in order ----
    mbar_expect_tx(&S.wbar, W_BYTES);
    for (int tap = 0; tap < 9; ++tap)  // tap = 3*(dy+1) + (dx+1) -> [dx][dy]
      tma_load_2d(S.w + ((tap % 3) * 3 + tap / 3) * WT_BYTES, &tmW, &S.wbar, 0, tap * CH);
    uint32_t L = 0;  // loads issued
    bool ok = true;
    // test of the failure path: the first load is never issued, so the waits
    // for its row run out (the load is left out, not broken)
    const bool skip_first = E.skip_load && blockIdx.x == 0;
    for (int st = blockIdx.x; st < nstrip && ok; st += gridDim.x) {
      const int ys = st % ystrips, r0 = st / ystrips, xt = r0 % xtiles, n = r0 / xtiles;
      const int y0 = ys * R, y1 = min(y0 + R, E.H) - 1;
      for (int r = y0 - 1; r <= y1 + 1; ++r, ++L) {
        const int slot = (int)(L % NS);
        const uint32_t ph = (L / NS) & 1;
        if (!mbar_wait(&S.empty[slot], ph ^ 1, LIM)) { fail(E.err, 31); ok = false; break; }
        if (skip_first && L == 0) continue;
        mbar_expect_tx(&S.full[slot], RW_BYTES);
        tma_load_4d(S.slot[slot], &tmA, &S.full[slot], 0, xt * TM - 8, r, n);
      }
    }
    // every armed load lands before the CTA may exit (the omitted one is not armed)
    for (int s = 0; s < NS; ++s) {
      const uint32_t armed = L / NS + ((uint32_t)s < L % NS ? 1u : 0u);
      if (skip_first && s == 0 && armed == 1) continue;
      if (armed) mbar_wait(&S.full[s], (armed - 1) & 1);
    }
    mbar_wait(&S.wbar, 0);
  } else if (warp == 1 && lane == 0) {
    // ---- MMA issuer ----
    bool ok = mbar_wait(&S.wbar, 0);
    if (!ok) fail(E.err, 32);
    const uint32_t wbase = smem_u32(S.w);
    const uint64_t DK = sdesc(0, 16, 1024);  // K-major, 128-byte swizzle; address field zero
    const uint32_t ID192 = idesc(128, 192, 0, 0);
    uint32_t L = 0;  // loads consumed
    uint32_t g0 = 0;  // CTA-wide index of the strip's first output row
    for (int st = blockIdx.x; st < nstrip && ok; st += gridDim.x) {
      const int ys = st % ystrips;
      const int y0 = ys * R, y1 = min(y0 + R, E.H) - 1;
      const int rows = y1 - y0 + 1;
      for (int t = 0; t <= rows + 1 && ok; ++t) {
        // input row y0-1+t feeds the strip's output rows o_lo .. o_hi
        const int o_hi = min(t, rows - 1), o_lo = max(t - 2, 0);
        const uint32_t ld = L + (uint32_t)t;
        const int slot = (int)(ld % NS);
        if (t <= rows - 1) {  // output row t starts here: its block must be drained and zeroed
          const uint32_t g = g0 + (uint32_t)t;
          if (!mbar_wait(&S.tempty[tblk<NB>(g)], ((g / NB) & 1) ^ 1, LIM)) { fail(E.err, 33); ok = false; break; }
        }
        if (!mbar_wait(&S.full[slot], (ld / NS) & 1, LIM)) { fail(E.err, 34); ok = false; break; }
        tc_fence_after();
        const int nout = o_hi - o_lo + 1;
        const uint32_t dfirst = tblk<NB>(g0 + (uint32_t)o_hi);
        const int n1 = min(nout, NB - (int)dfirst), n2 = nout - n1;
        const int bfirst = t - o_hi;  // B block: 0 for dy = -1, 1 for 0, 2 for +1
        // descriptors as constant offsets (in 16-byte units) from two bases:
        // the input row's window starting at pixel 7 and the weight block of
        // dx = -1, dy = bfirst; dx steps 128 bytes / 3 weight blocks, k 32 bytes
        const uint64_t A0 = DK + ((smem_u32(S.slot[slot]) + 7u * 128u) >> 4);
        const uint64_t B0 = DK + ((wbase + (uint32_t)bfirst * WT_BYTES) >> 4);
        if (n2 == 0 && nout == 3) {  // an interior row, no wrap: 12 MMAs of N = 192
          const uint32_t d = tmem + dfirst * 64;
#pragma unroll
          for (int dx = 0; dx < 3; ++dx)
#pragma unroll
            for (int k = 0; k < 4; ++k)
              mma_bf16(d, A0 + (uint64_t)(8 * dx + 2 * k), B0 + (uint64_t)(dx * 3 * (WT_BYTES >> 4) + 2 * k), ID192, 1u);
        } else {
          const uint32_t id1 = idesc(128, 64 * n1, 0, 0);
          const uint32_t id2 = idesc(128, 64 * (n2 > 0 ? n2 : 1), 0, 0);
          const uint64_t B1 = B0 + (uint64_t)(n1 * (WT_BYTES >> 4));
#pragma unroll
          for (int dx = 0; dx < 3; ++dx)
#pragma unroll
            for (int k = 0; k < 4; ++k)
              mma_bf16(tmem + dfirst * 64, A0 + (uint64_t)(8 * dx + 2 * k),
                       B0 + (uint64_t)(dx * 3 * (WT_BYTES >> 4) + 2 * k), id1, 1u);
          if (n2 > 0) {
#pragma unroll
            for (int dx = 0; dx < 3; ++dx)
#pragma unroll
              for (int k = 0; k < 4; ++k)
                mma_bf16(tmem, A0 + (uint64_t)(8 * dx + 2 * k), B1 + (uint64_t)(dx * 3 * (WT_BYTES >> 4) + 2 * k),
                         id2, 1u);
          }
        }
        mma_commit(&S.empty[slot]);                         // the input row has had its last use
        if (t >= 2) mma_commit(&S.tfull[tblk<NB>(g0 + (uint32_t)(t - 2))]);  // output row t-2 is complete
      }
      L += (uint32_t)rows + 2;
      g0 += (uint32_t)rows;
    }
    mma_commit(&S.done);  // completes once every MMA issued above has finished
    mbar_wait(&S.done, 0);
  } else if (warp >= 2) {
    // ---- epilogue: drain, zero for the next use, then bias/ReLU/residual/mask -> BF16 ----
    const int q = warp & 3;
    const int row = 32 * q + lane;
    uint32_t g = 0;
    bool ok = true;
    for (int st = blockIdx.x; st < nstrip && ok; st += gridDim.x) {
      const int ys = st % ystrips, r0 = st / ystrips, xt = r0 % xtiles, n = r0 / xtiles;
      const int y0 = ys * R, y1 = min(y0 + R, E.H) - 1;
      for (int y = y0; y <= y1; ++y, ++g) {
        const uint32_t b = tblk<NB>(g);
        if (!mbar_wait_warp(&S.tfull[b], (g / NB) & 1, LIM)) { fail(E.err, 35); ok = false; break; }
        tc_fence_after();
        float v[64];
        const uint32_t ta = tmem + b * 64 + ((uint32_t)(32 * q) << 16);
        tmem_ld32(ta, v);
        tmem_ld32(ta + 32, v + 32);
        tmem_zero32(ta);
        tmem_zero32(ta + 32);
        tmem_st_wait();
        tc_fence_before();
        mbar_arrive(&S.tempty[b]);
        const long p = ((long)(n * E.H + y) * E.W + xt * TM + row);
        if constexpr (TS) {
          epilogue_math(E, S.bias, v, p);
          if (E.out) {
            uint8_t* buf = S.ost + (q * 2 + (int)(g & 1)) * 4096;
            if (lane == 0) bulk_wait_read1();  // the store two rows ago has read this tile
            __syncwarp();
#pragma unroll
            for (int c = 0; c < 8; ++c)  // 16-byte chunk c of row `lane`, 128-byte swizzle
              *reinterpret_cast<uint4*>(buf + lane * 128 + ((c ^ (lane & 7)) << 4)) = bf16x8(v, c);
            fence_proxy_async();
            __syncwarp();
            if (lane == 0) {
              tma_store_4d(&tmO, buf, 0, xt * TM + 32 * q, y, n);
              bulk_commit();
            }
          }
        } else {
          epilogue_store(E, S.bias, v, p);
        }
      }
    }
    if (TS && lane == 0) bulk_wait_all();  // every store has landed before the CTA exits
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    __syncwarp();
    tc_fence_after();
    tmem_dealloc(tmem, 64 * NB);
  }
}

struct WgSmem {
  // per stage: x window of tap a, x window of tap b (all ones for the last
  // tap pair, which then yields the bias gradient), dz window
  uint8_t st[WG_NST][3][WG_TILE];
  uint64_t full[WG_NST], empty[WG_NST];
  uint64_t done;
  uint32_t tmem_base;
  // Slack so that descriptor strides read no further than the allocation
  // even if a stride were misinterpreted; never written.
  uint8_t pad[8192];
};

// gridDim.y = 5 tap pairs: (0,1) (2,3) (4,5) (6,7) (8,bias).  gridDim.x CTAs
// split the pixel chunks of each pair.
__global__ void __launch_bounds__(THREADS, 1)
k_conv_wgrad(const __grid_constant__ CUtensorMap tmX, const __grid_constant__ CUtensorMap tmZ,
             WgradArgs G) {
  extern __shared__ uint8_t smem_raw[];
  WgSmem& S = *reinterpret_cast<WgSmem*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int mt = blockIdx.y;
  const bool bias_pair = (mt == 4);
  const int ta = 2 * mt, tb = 2 * mt + 1;  // tb unused for the bias pair
  const int xch = G.W / WG_PIX;
  const long nchunk = (long)G.N * G.H * xch;
  const long c_begin = nchunk * blockIdx.x / gridDim.x;
  const long c_end = nchunk * (blockIdx.x + 1) / gridDim.x;

  if (threadIdx.x == 0) {
    for (int s = 0; s < WG_NST; ++s) {
      mbar_init(&S.full[s], 1);
      mbar_init(&S.empty[s], 1);
    }
    mbar_init(&S.done, 1);
    fence_barrier_init();
  }
  if (bias_pair && warp >= 2) {
    // BF16 1.0 everywhere in the second A half of every stage
    const uint4 ones = make_uint4(0x3F803F80u, 0x3F803F80u, 0x3F803F80u, 0x3F803F80u);
    for (int s = 0; s < WG_NST; ++s) {
      uint4* d = reinterpret_cast<uint4*>(S.st[s][1]);
      for (int i = threadIdx.x - 64; i < WG_TILE / 16; i += THREADS - 64) d[i] = ones;
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 1) tmem_alloc(&S.tmem_base, 64);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = S.tmem_base;
  const bool have = c_end > c_begin;

  if (warp == 0 && lane == 0) {
    int stage = 0;
    uint32_t phase = 0;
    const uint32_t bytes = (bias_pair ? 2 : 3) * WG_TILE;
    for (long c = c_begin; c < c_end; ++c) {
      const int xc = (int)(c % xch);
      const long r = c / xch;
      const int y = (int)(r % G.H), n = (int)(r / G.H);
      const int x0 = xc * WG_PIX;
      if (!mbar_wait(&S.empty[stage], phase ^ 1)) { fail(G.err, 11); break; }
      mbar_expect_tx(&S.full[stage], bytes);
      tma_load_4d(S.st[stage][0], &tmX, &S.full[stage], 0, x0 + (ta % 3) - 1, y + ta / 3 - 1, n);
      if (!bias_pair)
        tma_load_4d(S.st[stage][1], &tmX, &S.full[stage], 0, x0 + (tb % 3) - 1, y + tb / 3 - 1, n);
      tma_load_4d(S.st[stage][2], &tmZ, &S.full[stage], 0, x0, y, n);
      if (++stage == WG_NST) { stage = 0; phase ^= 1; }
    }
    for (int s = 0; s < WG_NST; ++s) mbar_wait(&S.full[s], s < stage ? phase : phase ^ 1);
  } else if (warp == 1 && lane == 0) {
    // A: 128 rows (tap a ci 0-63, tap b ci 0-63) x K pixels with channels
    // contiguous -> MN-major; the two 64-row halves are 8 KiB apart (leading
    // byte offset), 8-pixel groups 1 KiB apart (stride byte offset).
    // B: 64 co x K pixels, MN-major likewise.
    const uint32_t ID = idesc(128, 64, 1, 1);
    int stage = 0;
    uint32_t phase = 0;
    bool first = true;
    for (long c = c_begin; c < c_end; ++c) {
      if (!mbar_wait(&S.full[stage], phase)) { fail(G.err, 12); break; }
      tc_fence_after();
      const uint32_t a = smem_u32(S.st[stage][0]);
      const uint32_t bz = smem_u32(S.st[stage][2]);
#pragma unroll
      for (int k = 0; k < WG_PIX / 16; ++k) {
        mma_bf16(tmem, sdesc(a + 2048 * k, WG_TILE, 1024), sdesc(bz + 2048 * k, WG_TILE, 1024), ID,
                 first ? 0u : 1u);
        first = false;
      }
      mma_commit(&S.empty[stage]);
      if (++stage == WG_NST) { stage = 0; phase ^= 1; }
    }
    mma_commit(&S.done);
    if (!mbar_wait(&S.done, 0)) fail(G.err, 13);
  }
  if (warp >= 2 && have) {
    const int q = warp & 3;
    const int row = 32 * q + lane;  // (tap half, ci)
    if (mbar_wait_warp(&S.done, 0)) {
      tc_fence_after();
      float v[64];
      const uint32_t taddr = tmem + ((uint32_t)(32 * q) << 16);
      tmem_ld32(taddr, v);
      tmem_ld32(taddr + 32, v + 32);
      if (row < 64 || !bias_pair) {
        const int tap = row < 64 ? ta : tb;
        float* dw = G.dw + (long)tap * CH * CH + (row & 63);
#pragma unroll
        for (int co = 0; co < 64; ++co) atomicAdd(dw + co * CH, v[co]);
      } else if (row == 64 && G.db) {
#pragma unroll
        for (int co = 0; co < 64; ++co) atomicAdd(G.db + co, v[co]);
      }
    } else {
      fail(G.err, 14);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    __syncwarp();
    tc_fence_after();
    tmem_dealloc(tmem, 64);
  }
}

// ---- weight gradient with three vertical taps per MMA ----------------------------
// dw[dy,dx][co][ci] = sum_q x[q + (0,dx)][ci] dz[q - (dy,0)][co]: for one pixel
// chunk q (64 pixels of an image row) the x windows of two horizontal taps
// form A (M = 128: dx_a ci 0-63, dx_b ci 0-63) and the dz windows of rows
// y+1, y, y-1 form B (N = 192: dy = -1, 0, +1), so one chunk's 4 MMAs of
// 128 x 192 x 16 cover six taps.  gridDim.y = 2 tap groups: dx = (-1, 0) and
// (+1, ones); the all-ones window of the second group gives the bias
// gradient in its dy = 0 block (the other two blocks of those rows are not
// used).  Operands are MN-major straight from the NHWC tensors: the A halves
// and the B blocks sit WG_TILE bytes apart (leading byte offset).
constexpr int WT_NST = 4;  // stages of 5 windows (40 KiB)

struct WtSmem {
  uint8_t st[WT_NST][5][WG_TILE];  // x_a, x_b, dz(y+1), dz(y), dz(y-1)
  uint64_t full[WT_NST], empty[WT_NST];
  uint64_t done;
  uint32_t tmem_base;
  uint8_t pad[8192];  // descriptor strides never reach past the allocation
};

__global__ void __launch_bounds__(THREADS, 1)
k_conv_wgrad_tri(const __grid_constant__ CUtensorMap tmX, const __grid_constant__ CUtensorMap tmZ,
                 WgradArgs G) {
  extern __shared__ uint8_t smem_raw[];
  WtSmem& S = *reinterpret_cast<WtSmem*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const bool bias_group = (blockIdx.y == 1);
  const int dxa = bias_group ? 1 : -1;  // second half: dx = 0, or the ones window
  const int xch = G.W / WG_PIX;
  const long nchunk = (long)G.N * G.H * xch;
  const long c_begin = nchunk * blockIdx.x / gridDim.x;
  const long c_end = nchunk * (blockIdx.x + 1) / gridDim.x;

  if (threadIdx.x == 0) {
    for (int s = 0; s < WT_NST; ++s) {
      mbar_init(&S.full[s], 1);
      mbar_init(&S.empty[s], 1);
    }
    mbar_init(&S.done, 1);
    fence_barrier_init();
  }
  if (bias_group && warp >= 2) {
    const uint4 ones = make_uint4(0x3F803F80u, 0x3F803F80u, 0x3F803F80u, 0x3F803F80u);
    for (int s = 0; s < WT_NST; ++s) {
      uint4* d = reinterpret_cast<uint4*>(S.st[s][1]);
      for (int i = threadIdx.x - 64; i < WG_TILE / 16; i += THREADS - 64) d[i] = ones;
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 1) tmem_alloc(&S.tmem_base, 256);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = S.tmem_base;
  const bool have = c_end > c_begin;

  if (warp == 0 && lane == 0) {
    int stage = 0;
    uint32_t phase = 0;
    const uint32_t bytes = (bias_group ? 4 : 5) * WG_TILE;
    for (long c = c_begin; c < c_end; ++c) {
      const int xc = (int)(c % xch);
      const long r = c / xch;
      const int y = (int)(r % G.H), n = (int)(r / G.H);
      const int x0 = xc * WG_PIX;
      if (!mbar_wait(&S.empty[stage], phase ^ 1)) { fail(G.err, 41); break; }
      mbar_expect_tx(&S.full[stage], bytes);
      tma_load_4d(S.st[stage][0], &tmX, &S.full[stage], 0, x0 + dxa, y, n);
      if (!bias_group) tma_load_4d(S.st[stage][1], &tmX, &S.full[stage], 0, x0, y, n);
      for (int j = 0; j < 3; ++j)  // dz rows y+1, y, y-1 (dy = -1, 0, +1)
        tma_load_4d(S.st[stage][2 + j], &tmZ, &S.full[stage], 0, x0, y + 1 - j, n);
      if (++stage == WT_NST) { stage = 0; phase ^= 1; }
    }
    for (int s = 0; s < WT_NST; ++s) mbar_wait(&S.full[s], s < stage ? phase : phase ^ 1);
  } else if (warp == 1 && lane == 0) {
    const uint32_t ID = idesc(128, 192, 1, 1);
    int stage = 0;
    uint32_t phase = 0;
    bool first = true;
    for (long c = c_begin; c < c_end; ++c) {
      if (!mbar_wait(&S.full[stage], phase)) { fail(G.err, 42); break; }
      tc_fence_after();
      const uint32_t a = smem_u32(S.st[stage][0]);
      const uint32_t bz = smem_u32(S.st[stage][2]);
#pragma unroll
      for (int k = 0; k < WG_PIX / 16; ++k) {
        mma_bf16(tmem, sdesc(a + 2048 * k, WG_TILE, 1024), sdesc(bz + 2048 * k, WG_TILE, 1024), ID,
                 first ? 0u : 1u);
        first = false;
      }
      mma_commit(&S.empty[stage]);
      if (++stage == WT_NST) { stage = 0; phase ^= 1; }
    }
    mma_commit(&S.done);
    if (!mbar_wait(&S.done, 0)) fail(G.err, 43);
  }
  if (warp >= 2 && have) {
    const int q = warp & 3;
    const int row = 32 * q + lane;  // (half, ci)
    if (mbar_wait_warp(&S.done, 0)) {
      tc_fence_after();
      const uint32_t taddr = tmem + ((uint32_t)(32 * q) << 16);
      const int half = row >> 6, ci = row & 63;
      for (int j = 0; j < 3; ++j) {  // dy = j - 1
        float v[64];
        tmem_ld32(taddr + 64 * j, v);
        tmem_ld32(taddr + 64 * j + 32, v + 32);
        if (half == 0 || !bias_group) {
          const int dx = half == 0 ? dxa : 0;
          const int tap = 3 * j + (dx + 1);
          float* dw = G.dw + (long)tap * CH * CH + ci;
#pragma unroll
          for (int co = 0; co < 64; ++co) atomicAdd(dw + co * CH, v[co]);
        } else if (j == 1 && ci == 0 && G.db) {
#pragma unroll
          for (int co = 0; co < 64; ++co) atomicAdd(G.db + co, v[co]);
        }
      }
    } else {
      fail(G.err, 44);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    __syncwarp();
    tc_fence_after();
    tmem_dealloc(tmem, 256);
  }
}

// ---- weight gradient over column strips, all taps per CTA (default) ---------------
// dw[dy,dx][co][ci] = sum_q x[q + (0,dx)][ci] dz[q - (dy,0)][co] as above, but one
// CTA computes all nine taps and the bias gradient: its accumulator holds
// group A = [x(dx=-1) | x(dx=0)]^T [dz(y+1) | dz(y) | dz(y-1)] in TMEM columns
// 0..191 and group B = [x(dx=+1) | ones]^T [...] in columns 256..447 (the ones
// half yields the bias gradient in its dy = 0 block).  The CTA owns a
// contiguous range of (image, 64-pixel column chunk, row) units ordered so
// that consecutive units march down the rows of one column strip:
//  * x row y: ONE load of the 80-pixel window x0-8 .. x0+71 (zero outside the
//    image); the operand is MN-major, one pixel per 128-byte K row, so the
//    horizontal taps are descriptors shifted by one pixel (128 bytes), and the
//    two M halves of group A, one pixel apart, are one descriptor with a
//    leading byte offset of 128;
//  * dz rows: each is loaded once into a ring of KZ rows.  Row loads take slots
//    in descending order, so rows y+1, y, y-1 sit at three consecutive slots
//    (one descriptor, leading byte offset = one slot) and each N block of the
//    accumulator always receives the same dy.  The descriptor of the top slot
//    reads two slots past the ring, so rows landing in slots 0 and 1 are
//    loaded a second time into slots KZ and KZ+1 (2 of every KZ rows).
// Per unit (PIX = 64): one 10 KiB x window, 8 KiB of dz (plus the occasional
// second copy) and 8 MMAs of 128 x 192 x 16 (the earlier kernels move 40 KiB
// per 4 MMAs); PIX = 128 doubles the unit, halving the per-unit waits and
// commits of the single producer and MMA threads.  At the end the CTA writes
// its 9 x 64 x 64 + 64 sums to its own row of a scratch array and
// k_wgrad_reduce adds the rows in a fixed order into dw and db, so the result
// does not depend on timing (no atomics).
static_assert(WS_NPART == 9 * CH * CH + CH, "one CTA's partial dw and db");

template <int PIX, int KX, int KZ>
struct WsSmem {
  static constexpr int XPIX = PIX + 16;            // x window pixels: x0-8 .. x0+PIX+7
  static constexpr int XBYTES = XPIX * CH * 2;     // 10 KiB at PIX = 64
  static constexpr int ZBYTES = PIX * CH * 2;      // 8 KiB at PIX = 64
  uint8_t x[KX][XBYTES];
  uint8_t z[KZ + 2][ZBYTES];
  uint8_t ones[16 * 128];  // 16 pixel rows of ones: the second M half of group B's A operand
  uint64_t xfull[KX], xempty[KX], zfull[KZ], zempty[KZ];
  uint64_t done;
  uint32_t tmem_base;
};

// Ring slot of the l-th dz row load: consecutive loads take descending slots.
template <int KZ>
__device__ __forceinline__ uint32_t ws_zslot(uint32_t l) { return (KZ - l % KZ) % KZ; }
// Loads among the first n whose slot is s (the ring visits each slot once per KZ loads).
template <int KZ>
__device__ __forceinline__ uint32_t ws_zcount(uint32_t n, uint32_t s) {
  const uint32_t j = (KZ - s) % KZ;
  return n / KZ + (j < n % KZ ? 1u : 0u);
}

template <int PIX, int KX, int KZ>
__global__ void __launch_bounds__(THREADS, 1)
k_conv_wgrad_strip(const __grid_constant__ CUtensorMap tmX, const __grid_constant__ CUtensorMap tmZ,
                   WgradArgs G) {
  using Smem = WsSmem<PIX, KX, KZ>;
  static_assert(Smem::XBYTES % 1024 == 0 && Smem::ZBYTES % 1024 == 0, "128-byte swizzle atoms");
  static_assert(KZ >= 4 && KX >= 2, "ring depths");
  extern __shared__ uint8_t smem_raw[];
  Smem& S = *reinterpret_cast<Smem*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int xch = G.W / PIX;
  const long nunit = (long)G.N * xch * G.H;
  const long u_begin = nunit * blockIdx.x / gridDim.x;
  const long u_end = nunit * (blockIdx.x + 1) / gridDim.x;
  const bool have = u_end > u_begin;

  if (threadIdx.x == 0) {
    for (int s = 0; s < KX; ++s) {
      mbar_init(&S.xfull[s], 1);
      mbar_init(&S.xempty[s], 1);
    }
    for (int s = 0; s < KZ; ++s) {
      mbar_init(&S.zfull[s], 1);
      mbar_init(&S.zempty[s], 1);
    }
    mbar_init(&S.done, 1);
    fence_barrier_init();
  }
  if (warp >= 2) {  // the all-ones half of group B's A operand
    const uint4 ones = make_uint4(0x3F803F80u, 0x3F803F80u, 0x3F803F80u, 0x3F803F80u);
    uint4* d = reinterpret_cast<uint4*>(S.ones);
    for (int i = threadIdx.x - 64; i < 16 * 128 / 16; i += THREADS - 64) d[i] = ones;
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 1) tmem_alloc(&S.tmem_base, 512);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = S.tmem_base;
  if (warp >= 2) {  // every accumulator starts at zero, so every MMA accumulates
    const uint32_t tl = tmem + ((uint32_t)(32 * (warp & 3)) << 16);
    for (int c = 0; c < 512; c += 32) tmem_zero32(tl + (uint32_t)c);
    tmem_st_wait();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();

  // unit u = (n * xch + column chunk) * H + y: the coordinates of the range's
  // first unit, then stepped per unit (a 64-bit division per unit would cost
  // the single producer and MMA threads more than the unit's MMAs take)
  const int y_begin = have ? (int)(u_begin % G.H) : 0;
  const long t_begin = have ? u_begin / G.H : 0;
  const int xc_begin = (int)(t_begin % xch), n_begin = (int)(t_begin / xch);
  if (warp == 0 && lane == 0) {
    // ---- TMA producer: per unit the next dz row and the x window ----
    uint32_t lx = 0, lz = 0;
    bool ok = true;
    int y = y_begin, xc = xc_begin, n = n_begin;
    for (long u = u_begin; u < u_end && ok; ++u) {
      const int x0 = xc * PIX;
      // a strip starts at the range's first unit or at row 0: rows y-1 and y first
      for (int dr = (u == u_begin || y == 0) ? -1 : 1; dr <= 1 && ok; ++dr) {
        const uint32_t s = ws_zslot<KZ>(lz);
        if (!mbar_wait(&S.zempty[s], ((lz / KZ) & 1) ^ 1)) { ok = false; break; }
        mbar_expect_tx(&S.zfull[s], (s < 2 ? 2 : 1) * Smem::ZBYTES);
        tma_load_4d(S.z[s], &tmZ, &S.zfull[s], 0, x0, y + dr, n);
        if (s < 2) tma_load_4d(S.z[s + KZ], &tmZ, &S.zfull[s], 0, x0, y + dr, n);
        ++lz;
      }
      if (!ok) break;
      const uint32_t s = lx % KX;
      if (!mbar_wait(&S.xempty[s], ((lx / KX) & 1) ^ 1)) { ok = false; break; }
      mbar_expect_tx(&S.xfull[s], Smem::XBYTES);
      tma_load_4d(S.x[s], &tmX, &S.xfull[s], 0, x0 - 8, y, n);
      ++lx;
      if (++y == G.H) {
        y = 0;
        if (++xc == xch) { xc = 0; ++n; }
      }
    }
    if (!ok) fail(G.err, 51);
    // every armed load lands before the CTA may exit
    for (uint32_t s = 0; s < (uint32_t)KX; ++s) {
      const uint32_t armed = lx / KX + (s < lx % KX ? 1u : 0u);
      if (armed) mbar_wait(&S.xfull[s], (armed - 1) & 1);
    }
    for (uint32_t s = 0; s < (uint32_t)KZ; ++s) {
      const uint32_t armed = ws_zcount<KZ>(lz, s);
      if (armed) mbar_wait(&S.zfull[s], (armed - 1) & 1);
    }
  } else if (warp == 1 && lane == 0) {
    // ---- MMA issuer ----
    // A single thread issues the MMAs, so its per-unit work is kept to a few
    // independent operations: ring slots and phases are stepped, not divided
    // out, and the descriptors of group A and of dz are constant offsets from
    // two bases (their address fields are addresses / 16).
    const uint32_t ID = idesc(128, 192, 1, 1);
    const uint32_t ones = smem_u32(S.ones);
    const uint32_t xbase = smem_u32(S.x[0]), zbase = smem_u32(S.z[0]);
    const uint64_t DA = sdesc(0, 128, 1024), DB = sdesc(0, Smem::ZBYTES, 1024);
    uint32_t xsl = 0, xph = 0;   // x window slot and phase of the next unit
    uint32_t zsl = 0, zph = 0;   // dz slot and phase of the next row load
    uint32_t s1 = 0, s2 = 0;     // slots of rows y and y-1
    bool ok = true;
    int y = y_begin;
    auto zstep = [&]() {
      zsl = zsl ? zsl - 1 : (uint32_t)KZ - 1;
      if (zsl == 0) zph ^= 1u;
    };
    for (long u = u_begin; u < u_end; ++u, y = (y + 1 == G.H) ? 0 : y + 1) {
      const bool start = (u == u_begin) || y == 0;
      const bool last = (u + 1 == u_end) || (y + 1 == G.H);
      if (start) {  // rows y-1 and y are this strip's first two loads
        s2 = zsl;
        ok = mbar_wait(&S.zfull[zsl], zph);
        zstep();
        s1 = zsl;
        if (ok) ok = mbar_wait(&S.zfull[zsl], zph);
        zstep();
      }
      const uint32_t s0 = zsl;  // row y+1
      if (ok) ok = mbar_wait(&S.zfull[zsl], zph);
      zstep();
      if (ok) ok = mbar_wait(&S.xfull[xsl], xph);
      if (!ok) break;
      tc_fence_after();
      const uint32_t xs = xbase + xsl * (uint32_t)Smem::XBYTES;
      const uint64_t a1 = DA + ((xs + 7u * 128u) >> 4);                            // [x(-1) | x(0)]
      const uint64_t bd = DB + ((zbase + s0 * (uint32_t)Smem::ZBYTES) >> 4);     // dz rows y+1, y, y-1
#pragma unroll
      for (int k = 0; k < PIX / 16; ++k) {
        const uint64_t dk = (uint64_t)(128 * k);  // 16 pixel rows of 128 bytes, in 16-byte units
        mma_bf16(tmem, a1 + dk, bd + dk, ID, 1u);
        const uint32_t xb = xs + (9u + 16u * k) * 128u;  // x(+1) rows of this K step
        mma_bf16(tmem + 256, sdesc(xb, ones - xb, 1024), bd + dk, ID, 1u);  // ones lie after the rings
      }
      mma_commit(&S.xempty[xsl]);
      mma_commit(&S.zempty[s2]);  // row y-1 has had its last use
      if (last) {                 // so have rows y and y+1 at a strip's end
        mma_commit(&S.zempty[s1]);
        mma_commit(&S.zempty[s0]);
      }
      s2 = s1;
      s1 = s0;
      if (++xsl == (uint32_t)KX) {
        xsl = 0;
        xph ^= 1u;
      }
    }
    if (!ok) fail(G.err, 52);
    mma_commit(&S.done);  // completes once every MMA issued above has finished
    if (!mbar_wait(&S.done, 0)) fail(G.err, 53);
  }
  if (warp >= 2) {
    // ---- this CTA's partial sums -> its row of the scratch array ----
    const int q = warp & 3;
    const int row = 32 * q + lane;  // TMEM lane: (M half, ci)
    const int half = row >> 6, ci = row & 63;
    float* part = G.partial + (long)blockIdx.x * WS_NPART;
    bool ok = true;
    if (have) {
      ok = mbar_wait_warp(&S.done, 0);
      if (!ok) fail(G.err, 54);
      tc_fence_after();
    }
    for (int grp = 0; grp < 2; ++grp) {
      for (int j = 0; j < 3; ++j) {  // dy = j - 1
        float v[64];
        if (have && ok) {
          const uint32_t ta = tmem + (uint32_t)(256 * grp + 64 * j) + ((uint32_t)(32 * q) << 16);
          tmem_ld32(ta, v);
          tmem_ld32(ta + 32, v + 32);
        } else {
#pragma unroll
          for (int c = 0; c < 64; ++c) v[c] = 0.0f;
        }
        if (grp == 0 || half == 0) {
          const int dx = grp == 1 ? 1 : (half == 0 ? -1 : 0);
          float* d = part + (long)(3 * j + dx + 1) * CH * CH + ci;
#pragma unroll
          for (int co = 0; co < 64; ++co) d[co * CH] = v[co];
        } else if (j == 1 && ci == 0) {
#pragma unroll
          for (int co = 0; co < 64; ++co) part[9 * CH * CH + co] = v[co];
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    __syncwarp();
    tc_fence_after();
    tmem_dealloc(tmem, 512);
  }
}

// The strip kernel's configurations: unit width and ring depths.
using WsA = WsSmem<64, 8, 12>;   // wgrad variant 2
#ifndef NEMO_WS_WIDE_KX
#define NEMO_WS_WIDE_KX 5
#endif
#ifndef NEMO_WS_WIDE_KZ
#define NEMO_WS_WIDE_KZ 6
#endif
using WsB = WsSmem<128, NEMO_WS_WIDE_KX, NEMO_WS_WIDE_KZ>;  // wgrad variant 3, the default (WsA unless W % 128 == 0)
static_assert(sizeof(WsA) + 1024 <= 232448 && sizeof(WsB) + 1024 <= 232448, "shared memory per CTA");

// dw[i] += sum_b part[b][i] (i < 9*64*64), db[i - 9*64*64] += ... (the rest),
// b = 0 .. nblk-1 in a fixed tree: 8 segments of consecutive rows summed in
// order, then the segment sums in order.  A block serves 32 consecutive i.
__global__ void __launch_bounds__(256)
k_wgrad_reduce(const float* __restrict__ part, int nblk, float* dw, float* db) {
  __shared__ float seg[8][32];
  const int i = blockIdx.x * 32 + (threadIdx.x & 31);
  const int g = threadIdx.x >> 5;
  const int b0 = nblk * g / 8, b1 = nblk * (g + 1) / 8;
  float s = 0.0f;
  if (i < WS_NPART) {
#pragma unroll 4
    for (int b = b0; b < b1; ++b) s += part[(long)b * WS_NPART + i];
  }
  seg[g][threadIdx.x & 31] = s;
  __syncthreads();
  if (g == 0 && i < WS_NPART) {
    float t = seg[0][threadIdx.x];
#pragma unroll
    for (int k = 1; k < 8; ++k) t += seg[k][threadIdx.x];
    if (i < 9 * CH * CH) dw[i] += t;
    else if (db) db[i - 9 * CH * CH] += t;
  }
}

// ---- tensor maps ---------------------------------------------------------------
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;

cudaError_t get_encoder() {
  if (g_encode) return cudaSuccess;
  cudaDriverEntryPointQueryResult q;
  void* fn = nullptr;
  cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
  if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn) return cudaErrorNotSupported;
  g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  return cudaSuccess;
}

// NHWC activations (64 channels) as a 4-D map (C, W, H, N); box = 64 x box_w.
cudaError_t act_map(CUtensorMap* m, const void* base, int N, int H, int W, int box_w) {
  cuuint64_t dims[4] = {(cuuint64_t)CH, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)N};
  cuuint64_t strides[3] = {(cuuint64_t)CH * 2, (cuuint64_t)W * CH * 2, (cuuint64_t)H * W * CH * 2};
  cuuint32_t box[4] = {(cuuint32_t)CH, (cuuint32_t)box_w, 1, 1};
  cuuint32_t es[4] = {1, 1, 1, 1};
  CUresult r = g_encode(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void*>(base), dims, strides, box,
                        es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

// Weights [9*64 rows][64 cols] BF16; box 64 x 64 (one tap).
cudaError_t w_map(CUtensorMap* m, const void* base) {
  cuuint64_t dims[2] = {(cuuint64_t)CH, (cuuint64_t)9 * CH};
  cuuint64_t strides[1] = {(cuuint64_t)CH * 2};
  cuuint32_t box[2] = {(cuuint32_t)CH, (cuuint32_t)CH};
  cuuint32_t es[2] = {1, 1};
  CUresult r = g_encode(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, es,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

int g_sms[64];
bool g_attr[64];
int g_fwd_variant = 4;  // 4: three output rows per MMA (k_conv_fwd_tri), outputs by TMA
                        // stores; 2: the same with per-thread stores; 3: as 2, two CTAs
                        // per SM; 1: row ring (k_conv_fwd_rows); 0: a TMA window per tap
int g_fwd_rows = 32;    // rows per strip of the ring kernels
int g_wgrad_variant = 3;  // 3: all taps per CTA over column strips (k_conv_wgrad_strip)
                          // in 128-pixel units where the width allows, else as 2;
                          // 2: the same in 64-pixel units; 1: three vertical taps per MMA
                          // (k_conv_wgrad_tri), 0: tap pairs
// Scratch of k_conv_wgrad_strip for callers that pass none: one array per
// device, grown on demand and kept until the process exits.
// Test settings of the forward kernel's failure path (set_test_wait).
std::atomic<unsigned long long> g_test_wait_ns{0};
std::atomic<int> g_test_skip{0};
std::mutex g_part_mu;
float* g_part[64];
int g_part_blocks[64];

// SM count of the current device; opts the kernels into their shared memory.
cudaError_t prepare_device(int* sms) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  if (!g_attr[dev]) {
    e = cudaDeviceGetAttribute(&g_sms[dev], cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_conv_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(sizeof(FwdSmem) + 1024));
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_conv_wgrad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(sizeof(WgSmem) + 1024));
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_conv_wgrad_tri, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(sizeof(WtSmem) + 1024));
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_conv_wgrad_strip<64, 8, 12>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(sizeof(WsA) + 1024));
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_conv_wgrad_strip<128, NEMO_WS_WIDE_KX, NEMO_WS_WIDE_KZ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(sizeof(WsB) + 1024));
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_conv_fwd_rows, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(sizeof(RowSmem) + 1024));
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_conv_fwd_tri<6, 8, 1, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(sizeof(TriSmem<6, 8>) + 1024));
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_conv_fwd_tri<6, 8, 1, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(sizeof(TriSmem<6, 8, 8 * 4096>) + 1024));
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_conv_fwd_tri<2, 4, 2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(sizeof(TriSmem<2, 4>) + 1024));
    if (e != cudaSuccess) return e;
    g_attr[dev] = true;
  }
  *sms = g_sms[dev];
  return cudaSuccess;
}

}  // namespace

cudaError_t conv_fwd(const __nv_bfloat16* x, const __nv_bfloat16* w, const ConvEpi& epi, cudaStream_t s) {
  if (epi.W % TM != 0 || epi.W < TM || epi.N < 1 || epi.H < 1 || !x || !w || !epi.err ||
      epi.out32_ch < 0 || epi.out32_ch > 64 || epi.out32_ch % 4 != 0)
    return cudaErrorInvalidValue;
  if ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(w) | reinterpret_cast<uintptr_t>(epi.out) |
       reinterpret_cast<uintptr_t>(epi.out32) | reinterpret_cast<uintptr_t>(epi.residual) |
       reinterpret_cast<uintptr_t>(epi.mask)) & 15)
    return cudaErrorInvalidValue;
  cudaError_t e = get_encoder();
  if (e != cudaSuccess) return e;
  int sms = 0;
  if ((e = prepare_device(&sms)) != cudaSuccess) return e;
  CUtensorMap ta, tw;
  if ((e = w_map(&tw, w)) != cudaSuccess) return e;
  if (g_fwd_variant >= 2) {
    if ((e = act_map(&ta, x, epi.N, epi.H, epi.W, RW_PIX)) != cudaSuccess) return e;
    const int R = g_fwd_rows;
    const long nstrip = (long)epi.N * (epi.W / TM) * ((epi.H + R - 1) / R);
    const long slots = g_fwd_variant == 3 ? 2L * sms : (long)sms;  // resident CTAs
    const int grid = (int)(nstrip < slots ? nstrip : slots);
    ConvEpi E = epi;
    E.wait_ns = g_test_wait_ns.load();
    int k = g_test_skip.load();
    E.skip_load = 0;
    while (k > 0 && !g_test_skip.compare_exchange_weak(k, k - 1)) {
    }
    if (k > 0) E.skip_load = 1;
    if (g_fwd_variant == 3) {
      k_conv_fwd_tri<2, 4, 2, false><<<grid, THREADS, sizeof(TriSmem<2, 4>) + 1024, s>>>(ta, tw, ta, E, R);
    } else if (g_fwd_variant == 4 && epi.out) {
      CUtensorMap to;
      if ((e = act_map(&to, epi.out, epi.N, epi.H, epi.W, 32)) != cudaSuccess) return e;
      k_conv_fwd_tri<6, 8, 1, true><<<grid, THREADS, sizeof(TriSmem<6, 8, 8 * 4096>) + 1024, s>>>(ta, tw, to, E, R);
    } else {
      k_conv_fwd_tri<6, 8, 1, false><<<grid, THREADS, sizeof(TriSmem<6, 8>) + 1024, s>>>(ta, tw, ta, E, R);
    }
    return cudaGetLastError();
  }
  if (g_fwd_variant == 1) {
    if ((e = act_map(&ta, x, epi.N, epi.H, epi.W, RW_PIX)) != cudaSuccess) return e;
    const int R = g_fwd_rows;
    const long nstrip = (long)epi.N * (epi.W / TM) * ((epi.H + R - 1) / R);
    const int grid = (int)(nstrip < sms ? nstrip : sms);
    k_conv_fwd_rows<<<grid, THREADS, sizeof(RowSmem) + 1024, s>>>(ta, tw, epi, R);
    return cudaGetLastError();
  }
  if ((e = act_map(&ta, x, epi.N, epi.H, epi.W, TM)) != cudaSuccess) return e;
  const long ntile = (long)epi.N * epi.H * (epi.W / TM);
  const int grid = (int)(ntile < sms ? ntile : sms);
  k_conv_fwd<<<grid, THREADS, sizeof(FwdSmem) + 1024, s>>>(ta, tw, epi);
  return cudaGetLastError();
}

int set_wgrad_variant(int variant) {
  const int prev = g_wgrad_variant;
  if (variant >= 0 && variant <= 3) g_wgrad_variant = variant;
  return prev;
}

int wgrad_kernels() { return g_wgrad_variant >= 2 ? 2 : 1; }

unsigned long long set_test_wait(unsigned long long wait_ns, int skip_launches) {
  g_test_skip.store(skip_launches > 0 ? skip_launches : 0);
  return g_test_wait_ns.exchange(wait_ns);
}

int set_fwd_variant(int variant, int rows) {
  const int prev = g_fwd_variant;
  if (variant >= 0 && variant <= 4) g_fwd_variant = variant;
  if (rows >= 1 && rows <= 4096) g_fwd_rows = rows;
  return prev;
}

cudaError_t conv_wgrad(const __nv_bfloat16* x, const __nv_bfloat16* dz, const WgradArgs& g, int ctas,
                       cudaStream_t s) {
  if (g.W % WG_PIX != 0 || g.W < WG_PIX || g.N < 1 || g.H < 1 || !x || !dz || !g.dw || !g.err)
    return cudaErrorInvalidValue;
  if ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(dz)) & 15) return cudaErrorInvalidValue;
  cudaError_t e = get_encoder();
  if (e != cudaSuccess) return e;
  int sms = 0;
  if ((e = prepare_device(&sms)) != cudaSuccess) return e;
  CUtensorMap tx, tz;
  if (g_wgrad_variant >= 2) {
    const bool wide = g_wgrad_variant == 3 && g.W % 128 == 0;
    const int pix = wide ? 128 : 64;
    if ((e = act_map(&tz, dz, g.N, g.H, g.W, pix)) != cudaSuccess) return e;
    if ((e = act_map(&tx, x, g.N, g.H, g.W, pix + 16)) != cudaSuccess) return e;
    const long nunit = (long)g.N * g.H * (g.W / pix);
    long gx = ctas > 0 ? ctas : sms;  // one CTA per SM (shared and tensor memory)
    if (gx > nunit) gx = nunit;
    WgradArgs a = g;
    if (!a.partial) {
      int dev = 0;
      if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
      std::lock_guard<std::mutex> lock(g_part_mu);
      const int want = (int)(gx > sms ? gx : sms);
      if (g_part_blocks[dev] < want) {
        float* p = nullptr;
        if ((e = nemo::dev_alloc(&p, (size_t)want * WS_NPART * sizeof(float))) != cudaSuccess) return e;
        if (g_part[dev]) {
          // the old array may still be read by work queued on another stream
          cudaDeviceSynchronize();
          cudaFree(g_part[dev]);
        }
        g_part[dev] = p;
        g_part_blocks[dev] = want;
      }
      a.partial = g_part[dev];
      a.partial_blocks = g_part_blocks[dev];
    }
    if (gx > a.partial_blocks) gx = a.partial_blocks;
    if (gx < 1) return cudaErrorInvalidValue;
    if (wide)
      k_conv_wgrad_strip<128, NEMO_WS_WIDE_KX, NEMO_WS_WIDE_KZ><<<(unsigned)gx, THREADS, sizeof(WsB) + 1024, s>>>(tx, tz, a);
    else
      k_conv_wgrad_strip<64, 8, 12><<<(unsigned)gx, THREADS, sizeof(WsA) + 1024, s>>>(tx, tz, a);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    k_wgrad_reduce<<<(WS_NPART + 31) / 32, 256, 0, s>>>(a.partial, (int)gx, g.dw, g.db);
    return cudaGetLastError();
  }
  if ((e = act_map(&tz, dz, g.N, g.H, g.W, WG_PIX)) != cudaSuccess) return e;
  if ((e = act_map(&tx, x, g.N, g.H, g.W, WG_PIX)) != cudaSuccess) return e;
  if (g_wgrad_variant == 1) {
    // one CTA per SM: one wave of the 2 tap groups
    int gx = ctas > 0 ? ctas : sms / 2;
    const long nchunk = (long)g.N * g.H * (g.W / WG_PIX);
    if (gx > nchunk) gx = (int)nchunk;
    if (gx < 1) gx = 1;
    k_conv_wgrad_tri<<<dim3((unsigned)gx, 2), THREADS, sizeof(WtSmem) + 1024, s>>>(tx, tz, g);
    return cudaGetLastError();
  }
  // two CTAs fit on an SM (shared memory and tensor memory): one wave of 5 pairs
  int gx = ctas > 0 ? ctas : (2 * sms) / 5;
  const long nchunk = (long)g.N * g.H * (g.W / WG_PIX);
  if (gx > nchunk) gx = (int)nchunk;
  if (gx < 1) gx = 1;
  k_conv_wgrad<<<dim3((unsigned)gx, 5), THREADS, sizeof(WgSmem) + 1024, s>>>(tx, tz, g);
  return cudaGetLastError();
}

}  // namespace sur
