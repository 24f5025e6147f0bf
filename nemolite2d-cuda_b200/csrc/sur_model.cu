// BF16 residual CNN surrogate of the NEMOLite2D step (no reference
// counterpart): training and inference on the tcgen05 convolution kernels,
// data packing from ensemble members, and the hybrid controller that lets
// the surrogate advance the ensemble k steps per call under FP64 re-anchoring.
//
// Network (all convolutions 3x3, 64 -> 64 channels, zero padding):
//   h0 = relu(conv_0(x0) + b_0)
//   t_i = relu(conv_{2i+1}(h_i) + b), h_{i+1} = h_i + conv_{2i+2}(t_i) + b   (i < nblocks)
//   y = conv_{L-1}(h_nb) + b           (channels 0-2: normalised 10-step deltas)
// The network runs on a grid of P x P patches of T-cells (P = 1, 2 or 4, the
// `patch` of the configuration): network pixel (X, Y) holds T-cells
// (ji, jj) = (P*X + sx + 1, P*Y + sy + 1), sub-cell k = P*sy + sx.  Input
// channels: ssh at k, u on the cell's west face u(ji-1, jj) at P^2 + k, v on
// its south face v(ji, jj-1) at 2 P^2 + k; depth (P = 1: channel 3; else the
// means over the four (P/2 x P/2) quadrants, channels 3 P^2 .. 3 P^2 + 3);
// then the open-boundary row flag and the boundary row's tidal SSH at the
// target time on network row 0; the rest zero.  Output channel f P^2 + k is
// the normalised 10-step delta of field f (ssh, u, v) at sub-cell k; the FP32
// output holds 4 channels per pixel for P = 1, 3 P^2 otherwise.  A patch of
// 4 runs the same network on 1/16 of the pixels.  Parameters are FP32
// masters with BF16 copies (and the tap-flipped transposes the data gradient
// needs) refreshed by AdamW.
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <chrono>
#include <new>
#include <vector>

#include "sur_internal.h"

using nemo::MemberState;

namespace {

constexpr int CH = 64;
constexpr int WL = 9 * CH * CH;  // weights per layer

struct Norm {
  float in_scale[4], in_shift[4], out_scale[3];
};

int status_of(cudaError_t e) {
  if (e == cudaSuccess) return NEMO_OK;
  if (e == cudaErrorMemoryAllocation) return NEMO_ERR_ALLOC;
  if (e == cudaErrorInvalidValue) return NEMO_ERR_INVALID;
  return NEMO_ERR_CUDA;
}
#define ECK(call)                                \
  do {                                           \
    cudaError_t e_ = (call);                     \
    if (e_ != cudaSuccess) return status_of(e_); \
  } while (0)
#define SCK(call)              \
  do {                         \
    int s_ = (call);           \
    if (s_ != NEMO_OK) return s_; \
  } while (0)

__device__ __forceinline__ uint4 pack8(const float* f) {
  uint4 u;
  __nv_bfloat162* h = reinterpret_cast<__nv_bfloat162*>(&u);
#pragma unroll
  for (int e = 0; e < 4; ++e) h[e] = __floats2bfloat162_rn(f[2 * e], f[2 * e + 1]);
  return u;
}

// FP32 output channels per network pixel
__host__ __device__ constexpr int out_channels(int P) { return P == 1 ? 4 : 3 * P * P; }
// first channel after the depth channels: the boundary flag, then the tide
__host__ __device__ constexpr int flag_channel(int P) { return P == 1 ? 4 : 3 * P * P + 4; }

// x0 from FP32 snapshots (ssh, u_west, v_south, depth per T-cell, layout
// [n][H][W]) and per-image tides, over nnet = n * (H/P) * (W/P) network pixels.
template <int P>
__global__ void k_make_input(const float4* __restrict__ snap, const float* __restrict__ tide, Norm nm,
                             uint4* __restrict__ x0, long nnet, int H, int W) {
  const int Hn = H / P, Wn = W / P;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < nnet; q += (long)gridDim.x * blockDim.x) {
    const long img = q / ((long)Hn * Wn);
    const int Y = (int)((q / Wn) % Hn), X = (int)(q % Wn);
    float f[CH];
#pragma unroll
    for (int c = 0; c < CH; ++c) f[c] = 0.0f;
    float dq[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int sy = 0; sy < P; ++sy)
#pragma unroll
      for (int sx = 0; sx < P; ++sx) {
        const float4 v = snap[(img * H + (long)(P * Y + sy)) * W + P * X + sx];
        const int k = P * sy + sx;
        f[k] = (v.x - nm.in_shift[0]) * nm.in_scale[0];
        f[P * P + k] = (v.y - nm.in_shift[1]) * nm.in_scale[1];
        f[2 * P * P + k] = (v.z - nm.in_shift[2]) * nm.in_scale[2];
        dq[P == 1 ? 0 : 2 * (2 * sy / P) + (2 * sx / P)] += (v.w - nm.in_shift[3]) * nm.in_scale[3];
      }
    if (P == 1) {
      f[3] = dq[0];
    } else {
#pragma unroll
      for (int i = 0; i < 4; ++i) f[3 * P * P + i] = dq[i] * (4.0f / (float)(P * P));
    }
    f[flag_channel(P)] = Y == 0 ? 1.0f : 0.0f;
    f[flag_channel(P) + 1] = Y == 0 ? (tide[img] - nm.in_shift[0]) * nm.in_scale[0] : 0.0f;
    uint4* o = x0 + q * 8;
#pragma unroll
    for (int g = 0; g < 8; ++g) o[g] = pack8(f + 8 * g);
  }
}

// Index of output channel (field f, T-cell (x, y) of image img) in the FP32
// network output.
template <int P>
__device__ __forceinline__ long out_index(long img, int y, int x, int Hn, int Wn, int f) {
  const long q = (img * Hn + y / P) * Wn + x / P;
  return q * out_channels(P) + f * P * P + (y % P) * P + (x % P);
}

// Normalised 10-step deltas (channels 0-2; channel 3 zero).
__global__ void k_make_target(const float4* __restrict__ s0, const float4* __restrict__ s1, Norm nm,
                              float4* __restrict__ tgt, long npix) {
  for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < npix; p += (long)gridDim.x * blockDim.x) {
    const float4 a = s0[p], b = s1[p];
    tgt[p] = make_float4((b.x - a.x) * nm.out_scale[0], (b.y - a.y) * nm.out_scale[1],
                         (b.z - a.z) * nm.out_scale[2], 0.0f);
  }
}

template <int BT>
__device__ __forceinline__ double block_sum_d(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) sh[w] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < BT / 32; ++i) t += sh[i];
  __syncthreads();
  return t;
}

// Mean squared error of the deltas against targets tgt ([n][H][W] float4,
// channels 0-2) and its gradient (BF16, 64 channels per network pixel).
template <int P>
__global__ void __launch_bounds__(256) k_loss(const float* __restrict__ out, const float4* __restrict__ tgt,
                                              uint4* __restrict__ dout, double* __restrict__ loss, long nnet,
                                              int H, int W, float gscale) {
  __shared__ double sh[8];
  constexpr int NO = out_channels(P);
  const int Hn = H / P, Wn = W / P;
  double acc = 0.0;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < nnet; q += (long)gridDim.x * blockDim.x) {
    const long img = q / ((long)Hn * Wn);
    const int Y = (int)((q / Wn) % Hn), X = (int)(q % Wn);
    float f[CH];
#pragma unroll
    for (int c = 0; c < CH; ++c) f[c] = 0.0f;
#pragma unroll
    for (int sy = 0; sy < P; ++sy)
#pragma unroll
      for (int sx = 0; sx < P; ++sx) {
        const int k = P * sy + sx;
        const float4 t = tgt[(img * H + (long)(P * Y + sy)) * W + P * X + sx];
        const float d0 = out[q * NO + k] - t.x, d1 = out[q * NO + P * P + k] - t.y,
                    d2 = out[q * NO + 2 * P * P + k] - t.z;
        acc += (double)d0 * d0 + (double)d1 * d1 + (double)d2 * d2;
        f[k] = 2.0f * gscale * d0;
        f[P * P + k] = 2.0f * gscale * d1;
        f[2 * P * P + k] = 2.0f * gscale * d2;
      }
    uint4* g = dout + q * 8;
#pragma unroll
    for (int e = 0; e < 8; ++e) g[e] = pack8(f + 8 * e);
  }
  const double s = block_sum_d<256>(acc, sh);
  if (threadIdx.x == 0) atomicAdd(loss, s);
}

// BF16 copies of layer weights: w[l][tap][co][ci] and the data-gradient
// weights wt[l][8 - tap][ci][co].
__device__ __forceinline__ void put_weight(long i, float p, __nv_bfloat16* wbf, __nv_bfloat16* wt) {
  const __nv_bfloat16 b = __float2bfloat16_rn(p);
  wbf[i] = b;
  const long l = i / WL;
  const int r = (int)(i % WL);
  const int tap = r / (CH * CH), co = (r / CH) % CH, ci = r % CH;
  wt[l * WL + (long)(8 - tap) * CH * CH + ci * CH + co] = b;
}

__global__ void k_prep_weights(const float* __restrict__ p, long nw, __nv_bfloat16* wbf, __nv_bfloat16* wt) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < nw; i += (long)gridDim.x * blockDim.x)
    put_weight(i, p[i], wbf, wt);
}

struct AdamArgs {
  float lr, b1, b2, eps, wd, bc1, bc2;
};

// AdamW (decoupled weight decay on weights, not biases); refreshes the BF16
// copies and clears the gradient for the next accumulation.
__global__ void k_adamw(float* __restrict__ p, float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                        long np, long nw, AdamArgs a, __nv_bfloat16* wbf, __nv_bfloat16* wt) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < np; i += (long)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = a.b1 * m[i] + (1.0f - a.b1) * gi;
    const float vi = a.b2 * v[i] + (1.0f - a.b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float mh = mi / a.bc1, vh = vi / a.bc2;
    float pi = p[i];
    const float upd = mh / (sqrtf(vh) + a.eps) + (i < nw ? a.wd * pi : 0.0f);
    pi -= a.lr * upd;
    p[i] = pi;
    g[i] = 0.0f;
    if (i < nw) put_weight(i, pi, wbf, wt);
  }
}

// ---- ensemble <-> network tensors -------------------------------------------
__device__ __forceinline__ long gidx(int pitch, int ji, int jj) { return (long)(jj + 1) * pitch + ji + 2; }

__global__ void k_pack(const MemberState* __restrict__ ms, int m0, int nm, int H, int W, float4* __restrict__ snap) {
  const long npix = (long)nm * H * W;
  for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < npix; p += (long)gridDim.x * blockDim.x) {
    const int m = (int)(p / ((long)H * W));
    const int y = (int)((p / W) % H), x = (int)(p % W);
    const MemberState& M = ms[m0 + m];
    const int ji = x + 1, jj = y + 1;
    snap[p] = make_float4((float)M.sshn[gidx(M.pitch, ji, jj)], (float)M.un[gidx(M.pitch, ji - 1, jj)],
                          (float)M.vn[gidx(M.pitch, ji, jj - 1)], (float)M.ht[gidx(M.pitch, ji, jj)]);
  }
}

// state += delta / out_scale; the boundary row takes the exact tidal SSH;
// u(0, :), u(jpi, :) and v(:, jpj) (walls) are left at zero.
template <int P>
__global__ void k_apply(const MemberState* __restrict__ ms, int m0, int nm, int H, int W,
                        const float* __restrict__ out, Norm nm_, const double* __restrict__ tide) {
  const long npix = (long)nm * H * W;
  const int Hn = H / P, Wn = W / P;
  for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < npix; p += (long)gridDim.x * blockDim.x) {
    const int m = (int)(p / ((long)H * W));
    const int y = (int)((p / W) % H), x = (int)(p % W);
    const MemberState& M = ms[m0 + m];
    const int ji = x + 1, jj = y + 1;
    const float4 d = make_float4(out[out_index<P>(m, y, x, Hn, Wn, 0)], out[out_index<P>(m, y, x, Hn, Wn, 1)],
                                 out[out_index<P>(m, y, x, Hn, Wn, 2)], 0.0f);
    float4 c = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (M.corr) c = reinterpret_cast<const float4*>(M.corr)[(long)y * W + x];
    double* s = M.sshn + gidx(M.pitch, ji, jj);
    *s = (jj == 1) ? tide[m0 + m] : *s + (double)(d.x / nm_.out_scale[0]) + (double)c.x;
    if (ji >= 2) {
      double* u = M.un + gidx(M.pitch, ji - 1, jj);
      *u = *u + (double)(d.y / nm_.out_scale[1]) + (double)c.y;
    }
    double* v = M.vn + gidx(M.pitch, ji, jj - 1);
    *v = *v + (double)(d.z / nm_.out_scale[2]) + (double)c.z;
  }
}

// The open boundary after a surrogate call, as the solver closes every step
// (original/nemolite2d.f90:684-695): v(ji,0) = v(ji,1) + sqrt(g/hv(ji,0)) *
// (sshn_v(ji,0) - sshn_v(ji,1)), with sshn_v(ji,1) the mean of sshn on rows 1
// and 2 (uniform metrics) and sshn_v(ji,0) the stored boundary value.  The
// network's own v(ji,0) is replaced: the boundary velocity is diagnostic.
__global__ void k_flather(const MemberState* __restrict__ ms, int m0) {
  const MemberState& M = ms[m0 + blockIdx.y];
  for (int ji = 1 + blockIdx.x * blockDim.x + threadIdx.x; ji <= M.jpi; ji += gridDim.x * blockDim.x) {
    const double s1 = M.sshn[gidx(M.pitch, ji, 1)];
    const double sv1 = M.jpj >= 2 ? 0.5 * (s1 + M.sshn[gidx(M.pitch, ji, 2)]) : s1;
    const double v1 = M.vn[gidx(M.pitch, ji, 1)];
    M.vn[gidx(M.pitch, ji, 0)] = v1 + sqrt(9.80665 / M.hv[gidx(M.pitch, ji, 0)]) * (M.sshv0[gidx(M.pitch, ji, 0)] - sv1);
  }
}

// Per member: sum (pred - ref)^2 and sum ref^2 for ssh, u, v (acc[m][6]).
// pred = snap + delta / out_scale when out != null, else the state of `pm`.
// With corr (and out), ref - pred per T-cell goes to corr[m][y][x].
template <int P>
__global__ void __launch_bounds__(256) k_err(const MemberState* __restrict__ ref, const float4* __restrict__ snap,
                                             const float* __restrict__ out, Norm nm_,
                                             const MemberState* __restrict__ pm, int m0, int H, int W,
                                             double* __restrict__ acc, float4* __restrict__ corr = nullptr) {
  __shared__ double sh[8];
  const int m = blockIdx.y;
  const MemberState& R = ref[m0 + m];
  double a[6] = {0, 0, 0, 0, 0, 0};
  const long np = (long)H * W;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < np; q += (long)gridDim.x * blockDim.x) {
    const int y = (int)(q / W), x = (int)(q % W);
    const int ji = x + 1, jj = y + 1;
    const double rs = R.sshn[gidx(R.pitch, ji, jj)];
    const double ru = R.un[gidx(R.pitch, ji - 1, jj)];
    const double rv = R.vn[gidx(R.pitch, ji, jj - 1)];
    double ps, pu, pv;
    if (out) {
      const long p = (long)m * np + q;
      const int Hn = H / P, Wn = W / P;
      const float4 s = snap[p];
      const float4 d = make_float4(out[out_index<P>(m, y, x, Hn, Wn, 0)], out[out_index<P>(m, y, x, Hn, Wn, 1)],
                                   out[out_index<P>(m, y, x, Hn, Wn, 2)], 0.0f);
      ps = (jj == 1) ? rs : (double)s.x + (double)(d.x / nm_.out_scale[0]);
      pu = (ji >= 2) ? (double)s.y + (double)(d.y / nm_.out_scale[1]) : 0.0;
      pv = (double)s.z + (double)(d.z / nm_.out_scale[2]);
      if (corr) corr[p] = make_float4((float)(rs - ps), (float)(ru - pu), (float)(rv - pv), 0.0f);
    } else {
      const MemberState& Q = pm[m0 + m];
      ps = Q.sshn[gidx(Q.pitch, ji, jj)];
      pu = Q.un[gidx(Q.pitch, ji - 1, jj)];
      pv = Q.vn[gidx(Q.pitch, ji, jj - 1)];
    }
    a[0] += (ps - rs) * (ps - rs);
    a[1] += rs * rs;
    a[2] += (pu - ru) * (pu - ru);
    a[3] += ru * ru;
    a[4] += (pv - rv) * (pv - rv);
    a[5] += rv * rv;
  }
  for (int k = 0; k < 6; ++k) {
    const double s = block_sum_d<256>(a[k], sh);
    if (threadIdx.x == 0) atomicAdd(acc + (m0 + m) * 6 + k, s);
  }
}

int grid_for(long n, int block) {
  long g = (n + block - 1) / block;
  if (g > 148 * 16) g = 148 * 16;
  return (int)(g < 1 ? 1 : g);
}

uint64_t smix(uint64_t* s) {
  uint64_t z = (*s += 0x9E3779B97F4A7C15ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
double unif(uint64_t* s) { return ((double)(smix(s) >> 11) + 0.5) * 0x1.0p-53; }
double gauss(uint64_t* s) {
  const double u = unif(s), v = unif(s);
  return sqrt(-2.0 * log(u)) * cos(6.283185307179586 * v);
}

}  // namespace

struct nemo_sur {
  nemo_sur_config cfg{};
  int L = 0;
  long np = 0, nw = 0;          // parameters, of which weights
  long npix = 0;                 // batch * H * W (T-cells)
  int P = 1, Hn = 0, Wn = 0;     // patch and network grid (H/P x W/P)
  int NO = 4;                    // FP32 output channels per network pixel
  long nnet = 0;                 // batch * Hn * Wn (network pixels)
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  Norm norm{};
  float* p = nullptr;            // params (weights of all layers, then biases)
  float* g = nullptr;
  float* m = nullptr;
  float* v = nullptr;
  __nv_bfloat16* wbf = nullptr;
  __nv_bfloat16* wt = nullptr;
  std::vector<__nv_bfloat16*> act;  // activation tensors
  __nv_bfloat16 *x0 = nullptr, *dout = nullptr, *g0 = nullptr, *g1 = nullptr, *dt = nullptr;
  std::vector<__nv_bfloat16*> h, t;
  float* out32 = nullptr;        // [batch][Hn][Wn][NO]
  float* tgt = nullptr;
  float* snap = nullptr;         // [batch][H][W][4] (ensemble calls)
  float* tide_f = nullptr;       // [batch]
  double* tide_d = nullptr;      // [members]
  double* loss = nullptr;
  double* h_loss = nullptr;
  int* err = nullptr;
  MemberState* d_ms = nullptr;
  MemberState* d_ms2 = nullptr;
  int ms_cap = 0;
  double* d_acc = nullptr;
  int acc_cap = 0;
  float* wpart = nullptr;        // weight-gradient partial sums, one row per CTA
  int wpart_blocks = 0;
  long adam_t = 0;
  long long nlaunch = 0;  // kernels this surrogate has launched
};

namespace {

__nv_bfloat16* W_of(nemo_sur* s, int l) { return s->wbf + (long)l * WL; }
__nv_bfloat16* WT_of(nemo_sur* s, int l) { return s->wt + (long)l * WL; }
float* B_of(nemo_sur* s, int l) { return s->p + s->nw + (long)l * CH; }
float* dW_of(nemo_sur* s, int l) { return s->g + (long)l * WL; }
float* dB_of(nemo_sur* s, int l) { return s->g + s->nw + (long)l * CH; }

int set_dev(nemo_sur* s) {
  if (s->cfg.device >= 0) ECK(cudaSetDevice(s->cfg.device));
  return NEMO_OK;
}

int conv(nemo_sur* s, const __nv_bfloat16* x, const __nv_bfloat16* w, const float* bias,
         const __nv_bfloat16* res, const __nv_bfloat16* mask, int relu, __nv_bfloat16* out, float* out32, int n) {
  sur::ConvEpi e{bias, res, mask, out, out32, relu, n, s->Hn, s->Wn, s->err, out32 ? s->NO : 0};
  ECK(sur::conv_fwd(x, w, e, s->stream));
  s->nlaunch += 1;
  return NEMO_OK;
}

int wgrad(nemo_sur* s, const __nv_bfloat16* x, const __nv_bfloat16* dz, int l, int n) {
  sur::WgradArgs a{dW_of(s, l), dB_of(s, l), n, s->Hn, s->Wn, s->err, s->wpart, s->wpart_blocks};
  ECK(sur::conv_wgrad(x, dz, a, 0, s->stream));
  s->nlaunch += sur::wgrad_kernels();
  return NEMO_OK;
}

// Launches of the patch-templated kernels for the surrogate's patch.
cudaError_t make_input(nemo_sur* s, const float* snap, const float* tide, int n) {
  s->nlaunch += 1;
  const long nn = (long)n * s->Hn * s->Wn;
  const int H = s->cfg.height, W = s->cfg.width, g = grid_for(nn, 256);
  const float4* sp = reinterpret_cast<const float4*>(snap);
  uint4* x0 = reinterpret_cast<uint4*>(s->x0);
  switch (s->P) {
    case 1: k_make_input<1><<<g, 256, 0, s->stream>>>(sp, tide, s->norm, x0, nn, H, W); break;
    case 2: k_make_input<2><<<g, 256, 0, s->stream>>>(sp, tide, s->norm, x0, nn, H, W); break;
    default: k_make_input<4><<<g, 256, 0, s->stream>>>(sp, tide, s->norm, x0, nn, H, W); break;
  }
  return cudaGetLastError();
}

cudaError_t launch_loss(nemo_sur* s, int n, long npix) {
  s->nlaunch += 1;
  const long nn = (long)n * s->Hn * s->Wn;
  const int H = s->cfg.height, W = s->cfg.width, g = grid_for(nn, 256);
  const float gs = (float)(1.0 / (3.0 * (double)npix));
  const float4* t = reinterpret_cast<const float4*>(s->tgt);
  uint4* d = reinterpret_cast<uint4*>(s->dout);
  switch (s->P) {
    case 1: k_loss<1><<<g, 256, 0, s->stream>>>(s->out32, t, d, s->loss, nn, H, W, gs); break;
    case 2: k_loss<2><<<g, 256, 0, s->stream>>>(s->out32, t, d, s->loss, nn, H, W, gs); break;
    default: k_loss<4><<<g, 256, 0, s->stream>>>(s->out32, t, d, s->loss, nn, H, W, gs); break;
  }
  return cudaGetLastError();
}

cudaError_t launch_apply(nemo_sur* s, int m0, int n, const float* out) {
  s->nlaunch += 2;  // apply, open-boundary closure
  const int H = s->cfg.height, W = s->cfg.width, g = grid_for((long)n * H * W, 256);
  switch (s->P) {
    case 1: k_apply<1><<<g, 256, 0, s->stream>>>(s->d_ms, m0, n, H, W, out, s->norm, s->tide_d); break;
    case 2: k_apply<2><<<g, 256, 0, s->stream>>>(s->d_ms, m0, n, H, W, out, s->norm, s->tide_d); break;
    default: k_apply<4><<<g, 256, 0, s->stream>>>(s->d_ms, m0, n, H, W, out, s->norm, s->tide_d); break;
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_flather<<<dim3((unsigned)((W + 255) / 256), (unsigned)n), 256, 0, s->stream>>>(s->d_ms, m0);
  return cudaGetLastError();
}

// flag[m] = 1 when member m holds a non-finite sshn, un or vn value, or an
// |sshn| above ssh_limit[m], anywhere in its storage (grid x: chunks of the
// storage, grid y: members).
__global__ void k_diverged(const MemberState* __restrict__ ms, const double* __restrict__ ssh_limit, int* flag) {
  const int m = blockIdx.y;
  const MemberState M = ms[m];
  const double lim = ssh_limit[m];
  const long n = (long)(M.jpj + 3) * M.pitch;
  bool bad = false;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    bad |= !(fabs(M.sshn[i]) <= lim) | !isfinite(M.un[i]) | !isfinite(M.vn[i]);
  if (__syncthreads_or(bad) && threadIdx.x == 0) flag[m] = 1;
}

cudaError_t launch_err(nemo_sur* s, int nm, const float* snap, const float* out, float* corr = nullptr) {
  s->nlaunch += 1;
  const int H = s->cfg.height, W = s->cfg.width;
  const dim3 g((unsigned)(grid_for((long)H * W, 256) / 16 + 1), (unsigned)nm);
  const float4* sp = reinterpret_cast<const float4*>(snap);
  float4* c4 = reinterpret_cast<float4*>(corr);
  switch (s->P) {
    case 1: k_err<1><<<g, 256, 0, s->stream>>>(s->d_ms, sp, out, s->norm, nullptr, 0, H, W, s->d_acc, c4); break;
    case 2: k_err<2><<<g, 256, 0, s->stream>>>(s->d_ms, sp, out, s->norm, nullptr, 0, H, W, s->d_acc, c4); break;
    default: k_err<4><<<g, 256, 0, s->stream>>>(s->d_ms, sp, out, s->norm, nullptr, 0, H, W, s->d_acc, c4); break;
  }
  return cudaGetLastError();
}

// Forward from x0 over n images; training keeps every activation.
int forward(nemo_sur* s, int n, bool train, float* out32) {
  const int nb = s->cfg.nblocks;
  __nv_bfloat16* hcur = train ? s->h[0] : s->act[1];
  SCK(conv(s, s->x0, W_of(s, 0), B_of(s, 0), nullptr, nullptr, 1, hcur, nullptr, n));
  for (int i = 0; i < nb; ++i) {
    __nv_bfloat16* ti = train ? s->t[i] : s->act[3];
    __nv_bfloat16* hn = train ? s->h[i + 1] : (hcur == s->act[1] ? s->act[2] : s->act[1]);
    SCK(conv(s, hcur, W_of(s, 1 + 2 * i), B_of(s, 1 + 2 * i), nullptr, nullptr, 1, ti, nullptr, n));
    SCK(conv(s, ti, W_of(s, 2 + 2 * i), B_of(s, 2 + 2 * i), hcur, nullptr, 0, hn, nullptr, n));
    hcur = hn;
  }
  SCK(conv(s, hcur, W_of(s, s->L - 1), B_of(s, s->L - 1), nullptr, nullptr, 0, nullptr, out32, n));
  return NEMO_OK;
}

// Gradients of the loss held in dout (accumulated into g).
int backward(nemo_sur* s, int n) {
  const int nb = s->cfg.nblocks, L = s->L;
  SCK(wgrad(s, s->h[nb], s->dout, L - 1, n));
  __nv_bfloat16* gcur = s->g0;
  __nv_bfloat16* gnext = s->g1;
  SCK(conv(s, s->dout, WT_of(s, L - 1), nullptr, nullptr, nullptr, 0, gcur, nullptr, n));
  for (int i = nb - 1; i >= 0; --i) {
    const int la = 1 + 2 * i, lb = 2 + 2 * i;
    SCK(wgrad(s, s->t[i], gcur, lb, n));
    SCK(conv(s, gcur, WT_of(s, lb), nullptr, nullptr, s->t[i], 0, s->dt, nullptr, n));
    SCK(wgrad(s, s->h[i], s->dt, la, n));
    // d h_i = g + dgrad_a(dt), through the input ReLU for h_0
    SCK(conv(s, s->dt, WT_of(s, la), nullptr, gcur, i == 0 ? s->h[0] : nullptr, 0, gnext, nullptr, n));
    __nv_bfloat16* tmp = gcur;
    gcur = gnext;
    gnext = tmp;
  }
  if (nb == 0)  // no blocks: apply the input ReLU here
    SCK(conv(s, s->dout, WT_of(s, L - 1), nullptr, nullptr, s->h[0], 0, gcur, nullptr, n));
  SCK(wgrad(s, s->x0, gcur, 0, n));
  return NEMO_OK;
}

int check_err(nemo_sur* s) {
  int h = 0;
  ECK(cudaMemcpyAsync(&h, s->err, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
  ECK(cudaStreamSynchronize(s->stream));
  if (h != 0) {
    fprintf(stderr, "nemo_sur: device wait gave up (code %d)\n", h);
    cudaMemsetAsync(s->err, 0, sizeof(int), s->stream);
    return NEMO_ERR_TIMEOUT;
  }
  return NEMO_OK;
}

int loss_grad(nemo_sur* s, const float* snap0, const float* snap1, const float* tide, int n, double* loss) {
  if (n < 1 || n > s->cfg.batch || !snap0 || !snap1 || !tide || !s->cfg.train) return NEMO_ERR_INVALID;
  const long npix = (long)n * s->cfg.height * s->cfg.width;
  ECK(make_input(s, snap0, tide, n));
  k_make_target<<<grid_for(npix, 256), 256, 0, s->stream>>>(reinterpret_cast<const float4*>(snap0),
                                                          reinterpret_cast<const float4*>(snap1), s->norm,
                                                          reinterpret_cast<float4*>(s->tgt), npix);
  ECK(cudaGetLastError());
  SCK(forward(s, n, true, s->out32));
  ECK(cudaMemsetAsync(s->loss, 0, sizeof(double), s->stream));
  ECK(launch_loss(s, n, npix));
  SCK(backward(s, n));
  ECK(cudaMemcpyAsync(s->h_loss, s->loss, sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  SCK(check_err(s));
  if (loss) *loss = *s->h_loss / (3.0 * (double)npix);
  return NEMO_OK;
}

int ensure_members(nemo_sur* s, nemo_ens* e, std::vector<MemberState>& ms, MemberState** dst) {
  const int nm = nemo::ens_member_count(e);
  ms.resize(nm);
  for (int i = 0; i < nm; ++i) {
    SCK(nemo::ens_member_state(e, i, &ms[i]));
    if (ms[i].jpi != s->cfg.width || ms[i].jpj != s->cfg.height) return NEMO_ERR_INVALID;
  }
  if (nm > s->ms_cap) {
    cudaFree(s->d_ms);
    cudaFree(s->d_ms2);
    cudaFree(s->tide_d);
    s->d_ms = s->d_ms2 = nullptr;
    s->tide_d = nullptr;
    s->ms_cap = 0;
    ECK(nemo::dev_alloc(&s->d_ms, nm * sizeof(MemberState)));
    ECK(nemo::dev_alloc(&s->d_ms2, nm * sizeof(MemberState)));
    ECK(nemo::dev_alloc(&s->tide_d, nm * sizeof(double)));
    s->ms_cap = nm;
  }
  if (6 * nm > s->acc_cap) {
    cudaFree(s->d_acc);
    s->d_acc = nullptr;
    s->acc_cap = 0;
    ECK(nemo::dev_alloc(&s->d_acc, 6 * nm * sizeof(double)));
    s->acc_cap = 6 * nm;
  }
  MemberState* d = dst ? *dst : s->d_ms;
  ECK(cudaMemcpyAsync(d, ms.data(), nm * sizeof(MemberState), cudaMemcpyHostToDevice, s->stream));
  return NEMO_OK;
}

// Orders the surrogate's stream after the ensemble's work (and back).
int join(cudaStream_t wait_on, cudaStream_t waiter) {
  if (wait_on == waiter) return NEMO_OK;
  cudaEvent_t ev;
  ECK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  cudaError_t e = cudaEventRecord(ev, wait_on);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(waiter, ev, 0);
  cudaEventDestroy(ev);
  ECK(e);
  return NEMO_OK;
}

// Surrogate forward for members [m0, m0+n) of e from their current state
// (d_ms); tide_next[m] is the boundary SSH at the target time.  The chunk's
// snapshot goes to snap_dst and the normalised deltas to out_dst.
int predict_chunk(nemo_sur* s, int m0, int n, const std::vector<double>& tide_next, float* snap_dst,
                  float* out_dst) {
  const int H = s->cfg.height, W = s->cfg.width;
  const long npix = (long)n * H * W;
  std::vector<float> tf(n);
  for (int i = 0; i < n; ++i) tf[i] = (float)tide_next[m0 + i];
  // pageable source: the call returns once tf has been staged
  ECK(cudaMemcpyAsync(s->tide_f, tf.data(), n * sizeof(float), cudaMemcpyHostToDevice, s->stream));
  k_pack<<<grid_for(npix, 256), 256, 0, s->stream>>>(s->d_ms, m0, n, H, W, reinterpret_cast<float4*>(snap_dst));
  s->nlaunch += 1;
  ECK(cudaGetLastError());
  ECK(make_input(s, snap_dst, s->tide_f, n));
  return forward(s, n, false, out_dst);
}

// One surrogate call for the members of ms with sel[m] != 0 (all if sel is
// null): each advances from its current state to step istp_end.  Leaves the
// selected members' table in d_ms.
int advance_members(nemo_sur* s, nemo_ens* e, const std::vector<MemberState>& ms, const char* sel,
                    int istp_end) {
  std::vector<MemberState> sub;
  std::vector<double> tide;
  for (int m = 0; m < (int)ms.size(); ++m)
    if (!sel || sel[m]) {
      sub.push_back(ms[m]);
      tide.push_back(nemo::ens_tide(e, m, istp_end));
    }
  const int n_sel = (int)sub.size();
  if (n_sel == 0) return NEMO_OK;
  // pageable sources: staged before the calls return
  ECK(cudaMemcpyAsync(s->d_ms, sub.data(), n_sel * sizeof(MemberState), cudaMemcpyHostToDevice, s->stream));
  ECK(cudaMemcpyAsync(s->tide_d, tide.data(), n_sel * sizeof(double), cudaMemcpyHostToDevice, s->stream));
  for (int m0 = 0; m0 < n_sel; m0 += s->cfg.batch) {
    const int n = n_sel - m0 < s->cfg.batch ? n_sel - m0 : s->cfg.batch;
    SCK(predict_chunk(s, m0, n, tide, s->snap, s->out32));
    ECK(launch_apply(s, m0, n, s->out32));
  }
  return NEMO_OK;
}

}  // namespace

extern "C" {

int nemo_sur_default_config(nemo_sur_config* c) {
  if (!c) return NEMO_ERR_INVALID;
  memset(c, 0, sizeof(*c));
  c->nblocks = 8;
  c->batch = 64;
  c->height = 256;
  c->width = 256;
  c->train = 1;
  c->seed = 1234;
  c->stream = nullptr;
  c->device = -1;
  c->patch = 1;
  return NEMO_OK;
}

int nemo_sur_destroy(nemo_sur* s) {
  if (!s) return NEMO_ERR_INVALID;
  if (s->cfg.device >= 0) cudaSetDevice(s->cfg.device);
  if (s->stream) cudaStreamSynchronize(s->stream);
  for (auto* a : s->act) cudaFree(a);
  cudaFree(s->p);
  cudaFree(s->g);
  cudaFree(s->m);
  cudaFree(s->v);
  cudaFree(s->wbf);
  cudaFree(s->wt);
  cudaFree(s->out32);
  cudaFree(s->tgt);
  cudaFree(s->snap);
  cudaFree(s->tide_f);
  cudaFree(s->tide_d);
  cudaFree(s->loss);
  cudaFree(s->err);
  cudaFree(s->d_ms);
  cudaFree(s->d_ms2);
  cudaFree(s->d_acc);
  cudaFree(s->wpart);
  if (s->h_loss) cudaFreeHost(s->h_loss);
  if (s->own_stream && s->stream) cudaStreamDestroy(s->stream);
  delete s;
  return NEMO_OK;
}

int nemo_sur_create(const nemo_sur_config* c, nemo_sur** out) {
  if (!c || !out) return NEMO_ERR_INVALID;
  *out = nullptr;
  const int P = c->patch == 0 ? 1 : c->patch;
  if (c->nblocks < 0 || c->nblocks > 64 || c->batch < 1 || (P != 1 && P != 2 && P != 4) || c->height < P ||
      c->height % P != 0 || c->width % P != 0 || c->width / P < 128 || (c->width / P) % 128 != 0)
    return NEMO_ERR_INVALID;
  nemo_sur* s = new (std::nothrow) nemo_sur;
  if (!s) return NEMO_ERR_ALLOC;
  s->cfg = *c;
  s->L = 2 * c->nblocks + 2;
  s->nw = (long)s->L * WL;
  s->np = s->nw + (long)s->L * CH;
  s->cfg.patch = P;
  s->npix = (long)c->batch * c->height * c->width;
  s->P = P;
  s->Hn = c->height / P;
  s->Wn = c->width / P;
  s->NO = out_channels(P);
  s->nnet = (long)c->batch * s->Hn * s->Wn;
  for (int k = 0; k < 4; ++k) {
    s->norm.in_scale[k] = 1.0f;
    s->norm.in_shift[k] = 0.0f;
  }
  for (int k = 0; k < 3; ++k) s->norm.out_scale[k] = 1.0f;
  auto fail = [&](int st) {
    nemo_sur_destroy(s);
    return st;
  };
  if (set_dev(s)) return fail(NEMO_ERR_CUDA);
  if (c->stream) {
    s->stream = (cudaStream_t)c->stream;
  } else {
    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(NEMO_ERR_CUDA);
    s->own_stream = true;
  }
  const size_t pb = s->np * sizeof(float);
  if (nemo::dev_alloc(&s->p, pb) || nemo::dev_alloc(&s->g, pb) || nemo::dev_alloc(&s->wbf, s->nw * 2) ||
      nemo::dev_alloc(&s->wt, s->nw * 2) || nemo::dev_alloc(&s->loss, sizeof(double)) || nemo::dev_alloc(&s->err, sizeof(int)) ||
      nemo::host_alloc(&s->h_loss, sizeof(double)))
    return fail(NEMO_ERR_ALLOC);
  if (c->train && (nemo::dev_alloc(&s->m, pb) || nemo::dev_alloc(&s->v, pb))) return fail(NEMO_ERR_ALLOC);
  const size_t ab = (size_t)s->nnet * CH * 2;
  const int nact = c->train ? 1 + (c->nblocks + 1) + c->nblocks + 4 : 4;
  for (int i = 0; i < nact; ++i) {
    __nv_bfloat16* a = nullptr;
    if (nemo::dev_alloc(&a, ab)) return fail(NEMO_ERR_ALLOC);
    s->act.push_back(a);
  }
  s->x0 = s->act[0];
  if (c->train) {
    int k = 1;
    for (int i = 0; i <= c->nblocks; ++i) s->h.push_back(s->act[k++]);
    for (int i = 0; i < c->nblocks; ++i) s->t.push_back(s->act[k++]);
    s->dout = s->act[k++];
    s->g0 = s->act[k++];
    s->g1 = s->act[k++];
    s->dt = s->act[k++];
  }
  if (nemo::dev_alloc(&s->out32, s->nnet * s->NO * sizeof(float)) || nemo::dev_alloc(&s->snap, s->npix * 16) ||
      nemo::dev_alloc(&s->tide_f, c->batch * sizeof(float)))
    return fail(NEMO_ERR_ALLOC);
  if (c->train && nemo::dev_alloc(&s->tgt, s->npix * 16)) return fail(NEMO_ERR_ALLOC);
  if (c->train) {  // the weight gradient's per-CTA partial sums (one CTA per SM)
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev))
      return fail(NEMO_ERR_CUDA);
    if (nemo::dev_alloc(&s->wpart, (size_t)sms * sur::WS_NPART * sizeof(float))) return fail(NEMO_ERR_ALLOC);
    s->wpart_blocks = sms;
  }
  if (cudaMemsetAsync(s->err, 0, sizeof(int), s->stream) || cudaMemsetAsync(s->g, 0, pb, s->stream) ||
      (c->train && (cudaMemsetAsync(s->m, 0, pb, s->stream) || cudaMemsetAsync(s->v, 0, pb, s->stream))))
    return fail(NEMO_ERR_CUDA);
  // seeded initialisation: He-normal convolutions; the residual branches'
  // second convolutions and the output convolution start small
  std::vector<float> hp(s->np, 0.0f);
  uint64_t st = c->seed;
  for (int l = 0; l < s->L; ++l) {
    const bool first = l == 0, last = l == s->L - 1, branch_out = l > 0 && !last && (l % 2 == 0);
    const int cin = first ? 6 : CH;
    const int cout = last ? 3 : CH;
    double sd = sqrt(2.0 / (9.0 * cin));
    if (branch_out) sd *= 0.1;
    if (last) sd = 0.1 * sqrt(1.0 / (9.0 * cin));
    for (int tap = 0; tap < 9; ++tap)
      for (int co = 0; co < cout; ++co)
        for (int ci = 0; ci < cin; ++ci)
          hp[(long)l * WL + tap * CH * CH + co * CH + ci] = (float)(sd * gauss(&st));
  }
  if (cudaMemcpyAsync(s->p, hp.data(), pb, cudaMemcpyHostToDevice, s->stream)) return fail(NEMO_ERR_CUDA);
  k_prep_weights<<<grid_for(s->nw, 256), 256, 0, s->stream>>>(s->p, s->nw, s->wbf, s->wt);
  if (cudaGetLastError() || cudaStreamSynchronize(s->stream)) return fail(NEMO_ERR_CUDA);
  *out = s;
  return NEMO_OK;
}

int nemo_sur_info(nemo_sur* s, long long* nparams, long long* flops_per_pixel) {
  if (!s) return NEMO_ERR_STATE;
  if (nparams) *nparams = s->np;
  if (flops_per_pixel) *flops_per_pixel = (long long)s->L * 2 * WL / ((long long)s->P * s->P);
  return NEMO_OK;
}

int nemo_sur_get_params(nemo_sur* s, float* host) {
  if (!s || !host) return NEMO_ERR_INVALID;
  SCK(set_dev(s));
  ECK(cudaMemcpyAsync(host, s->p, s->np * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
  ECK(cudaStreamSynchronize(s->stream));
  return NEMO_OK;
}

int nemo_sur_set_params(nemo_sur* s, const float* host) {
  if (!s || !host) return NEMO_ERR_INVALID;
  SCK(set_dev(s));
  ECK(cudaMemcpyAsync(s->p, host, s->np * sizeof(float), cudaMemcpyHostToDevice, s->stream));
  k_prep_weights<<<grid_for(s->nw, 256), 256, 0, s->stream>>>(s->p, s->nw, s->wbf, s->wt);
  ECK(cudaGetLastError());
  ECK(cudaStreamSynchronize(s->stream));
  return NEMO_OK;
}

int nemo_sur_get_grads(nemo_sur* s, float* host) {
  if (!s || !host) return NEMO_ERR_INVALID;
  SCK(set_dev(s));
  ECK(cudaMemcpyAsync(host, s->g, s->np * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
  ECK(cudaStreamSynchronize(s->stream));
  return NEMO_OK;
}

int nemo_sur_set_norm(nemo_sur* s, const float* norm11) {
  if (!s || !norm11) return NEMO_ERR_INVALID;
  Norm n;
  memcpy(n.in_scale, norm11, 4 * sizeof(float));
  memcpy(n.in_shift, norm11 + 4, 4 * sizeof(float));
  memcpy(n.out_scale, norm11 + 8, 3 * sizeof(float));
  for (int k = 0; k < 3; ++k)
    if (!(n.out_scale[k] > 0.0f) || !isfinite(n.out_scale[k])) return NEMO_ERR_INVALID;
  s->norm = n;
  return NEMO_OK;
}

int nemo_sur_get_norm(nemo_sur* s, float* norm11) {
  if (!s || !norm11) return NEMO_ERR_INVALID;
  memcpy(norm11, s->norm.in_scale, 4 * sizeof(float));
  memcpy(norm11 + 4, s->norm.in_shift, 4 * sizeof(float));
  memcpy(norm11 + 8, s->norm.out_scale, 3 * sizeof(float));
  return NEMO_OK;
}

int nemo_sur_predict(nemo_sur* s, const float* snap, const float* tide, int n, float* out) {
  if (!s || !snap || !tide || n < 1 || n > s->cfg.batch) return NEMO_ERR_INVALID;
  SCK(set_dev(s));
  ECK(make_input(s, snap, tide, n));
  SCK(forward(s, n, false, out ? out : s->out32));
  return check_err(s);
}

int nemo_sur_loss_grad(nemo_sur* s, const float* snap0, const float* snap1, const float* tide, int n,
                       double* loss) {
  if (!s) return NEMO_ERR_STATE;
  SCK(set_dev(s));
  ECK(cudaMemsetAsync(s->g, 0, s->np * sizeof(float), s->stream));
  return loss_grad(s, snap0, snap1, tide, n, loss);
}

int nemo_sur_adamw(nemo_sur* s, const nemo_adamw* hp) {
  if (!s || !hp || !s->cfg.train) return NEMO_ERR_INVALID;
  SCK(set_dev(s));
  s->adam_t += 1;
  AdamArgs a{hp->lr, hp->beta1, hp->beta2, hp->eps, hp->weight_decay,
             (float)(1.0 - pow((double)hp->beta1, (double)s->adam_t)),
             (float)(1.0 - pow((double)hp->beta2, (double)s->adam_t))};
  k_adamw<<<grid_for(s->np, 256), 256, 0, s->stream>>>(s->p, s->g, s->m, s->v, s->np, s->nw, a, s->wbf, s->wt);
  ECK(cudaGetLastError());
  return NEMO_OK;
}

int nemo_sur_train_step(nemo_sur* s, const float* snap0, const float* snap1, const float* tide, int n,
                        const nemo_adamw* hp, double* loss) {
  if (!s || !hp) return NEMO_ERR_INVALID;
  SCK(set_dev(s));
  SCK(loss_grad(s, snap0, snap1, tide, n, loss));  // g is clear after the last AdamW
  return nemo_sur_adamw(s, hp);
}

int nemo_sur_pack_ens(nemo_sur* s, nemo_ens* e, float* snap) {
  if (!s || !e || !snap) return NEMO_ERR_INVALID;
  SCK(set_dev(s));
  std::vector<MemberState> ms;
  SCK(join(nemo::ens_stream(e), s->stream));
  SCK(ensure_members(s, e, ms, nullptr));
  const int nm = (int)ms.size();
  const long npix = (long)nm * s->cfg.height * s->cfg.width;
  k_pack<<<grid_for(npix, 256), 256, 0, s->stream>>>(s->d_ms, 0, nm, s->cfg.height, s->cfg.width,
                                                   reinterpret_cast<float4*>(snap));
  ECK(cudaGetLastError());
  ECK(cudaStreamSynchronize(s->stream));  // ms (host) copied
  return NEMO_OK;
}

int nemo_sur_advance_ens(nemo_sur* s, nemo_ens* e, int istp_end) {
  if (!s || !e) return NEMO_ERR_INVALID;
  SCK(set_dev(s));
  std::vector<MemberState> ms;
  SCK(join(nemo::ens_stream(e), s->stream));
  SCK(ensure_members(s, e, ms, nullptr));
  SCK(advance_members(s, e, ms, nullptr, istp_end));
  SCK(check_err(s));
  return join(s->stream, nemo::ens_stream(e));
}

int nemo_ens_compare(nemo_ens* a, nemo_ens* ref, double* out) {
  if (!a || !ref || !out) return NEMO_ERR_INVALID;
  const int nm = nemo::ens_member_count(a);
  if (nm != nemo::ens_member_count(ref)) return NEMO_ERR_INVALID;
  if (nemo::ens_device(a) >= 0) ECK(cudaSetDevice(nemo::ens_device(a)));
  std::vector<MemberState> ma(nm), mr(nm);
  for (int i = 0; i < nm; ++i) {
    SCK(nemo::ens_member_state(a, i, &ma[i]));
    SCK(nemo::ens_member_state(ref, i, &mr[i]));
    if (ma[i].jpi != mr[i].jpi || ma[i].jpj != mr[i].jpj) return NEMO_ERR_INVALID;
  }
  cudaStream_t st = nemo::ens_stream(a);
  SCK(join(nemo::ens_stream(ref), st));
  MemberState *da = nullptr, *dr = nullptr;
  double* acc = nullptr;
  cudaError_t e = nemo::dev_alloc(&da, nm * sizeof(MemberState));
  if (e == cudaSuccess) e = nemo::dev_alloc(&dr, nm * sizeof(MemberState));
  if (e == cudaSuccess) e = nemo::dev_alloc(&acc, 6 * nm * sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpyAsync(da, ma.data(), nm * sizeof(MemberState), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dr, mr.data(), nm * sizeof(MemberState), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(acc, 0, 6 * nm * sizeof(double), st);
  std::vector<double> h(6 * nm);
  if (e == cudaSuccess) {
    // one launch per member (sizes differ)
    for (int m = 0; m < nm && e == cudaSuccess; ++m) {
      Norm dummy{};
      k_err<1><<<dim3((unsigned)grid_for((long)ma[m].jpi * ma[m].jpj, 256) / 16 + 1, 1), 256, 0, st>>>(
          dr, nullptr, nullptr, dummy, da, m, ma[m].jpj, ma[m].jpi, acc);
      e = cudaGetLastError();
    }
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), acc, 6 * nm * sizeof(double), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(da);
  cudaFree(dr);
  cudaFree(acc);
  ECK(e);
  for (int m = 0; m < nm; ++m)
    for (int f = 0; f < 3; ++f) {
      const double num = h[6 * m + 2 * f], den = h[6 * m + 2 * f + 1];
      out[3 * m + f] = den > 0 ? sqrt(num / den) : sqrt(num);
    }
  return NEMO_OK;
}

int nemo_hyb_default_config(nemo_hyb_config* c) {
  if (!c) return NEMO_ERR_INVALID;
  c->k = 10;
  c->anchor = 100;
  c->tol = 0.01;
  c->per_member = 1;
  c->quarantine = 0.05;
  c->rewind = 1;
  c->correct = 0;
  return NEMO_OK;
}

// Advances e from the state after step istp0 by nsteps (a multiple of
// anchor, anchor a multiple of k).  Each anchor window: the surrogate
// predicts the first k steps of every member, the FP64 solver runs them (the
// shadow step, which also re-anchors the state), and each member whose
// relative SSH L2 error of the prediction exceeds tol (or is not finite)
// falls back: the solver runs the rest of its window.  The other members
// advance by surrogate calls, k steps each.  A member whose shadow error
// exceeds `quarantine` stays on the solver for the rest of the run (errors
// that large precede the corner instability the surrogate's perturbations
// can excite).  With `rewind`, such a member is first restored to its FP64
// state at the start of the latest of the two previous windows the surrogate
// advanced it in (saved at every window start, three per member) and the
// solver re-runs from there, so those unchecked calls leave no trace.  With
// per_member = 0 one failing member sends the whole ensemble to the solver
// for the window.  Statistics count member-windows and member-steps.
int nemo_hyb_run(nemo_sur* s, nemo_ens* e, const nemo_hyb_config* c, int istp0, int nsteps,
                 nemo_hyb_stats* stats) {
  if (!s || !e || !c || c->k < 1 || c->anchor < c->k || c->anchor % c->k || nsteps % c->anchor ||
      !(c->tol > 0) || (c->per_member && (c->anchor - c->k) % 2 != 0))
    return NEMO_ERR_INVALID;
  SCK(set_dev(s));
  nemo_hyb_stats st{};
  std::vector<MemberState> ms;
  SCK(join(nemo::ens_stream(e), s->stream));
  SCK(ensure_members(s, e, ms, nullptr));
  const int nm = (int)ms.size();
  const int H = s->cfg.height, W = s->cfg.width;
  const long hw = (long)H * W;
  // predictions of all members are kept for the shadow comparison
  float *snap_all = s->snap, *out_all = s->out32;
  float* own = nullptr;
  const size_t out_per = (size_t)s->Hn * s->Wn * s->NO;  // FP32 outputs per member
  if (nm > s->cfg.batch) {
    ECK(nemo::dev_alloc(&own, (size_t)nm * (hw * 4 + out_per) * sizeof(float)));
    snap_all = own;
    out_all = own + (size_t)nm * hw * 4;
  }
  // per-cell corrections from the shadow step (correct = 1)
  float* corr = nullptr;
  if (c->correct && nm > 0) {
    cudaError_t ae = nemo::dev_alloc(&corr, (size_t)nm * hw * 4 * sizeof(float));
    if (ae != cudaSuccess) {
      if (own) cudaFree(own);
      return status_of(ae);
    }
  }
  std::vector<double> tide(nm), acc(6 * nm);
  std::vector<char> pass(nm), fail(nm), quar(nm, 0);
  // saved FP64 states (sshn, un, vn) of every member at the last NS window
  // starts, for rewinding
  constexpr int NS = 3;
  const size_t field_elems = (size_t)(ms.empty() ? 0 : (long)(ms[0].jpj + 3) * ms[0].pitch);
  double* saved = nullptr;
  const bool rewind = c->rewind && c->quarantine > 0 && c->per_member;
  if (rewind && nm > 0) {
    cudaError_t ae = nemo::dev_alloc(&saved, (size_t)NS * nm * 3 * field_elems * sizeof(double));
    if (ae != cudaSuccess) {
      if (own) cudaFree(own);
      if (corr) cudaFree(corr);
      return status_of(ae);
    }
  }
  // slot x % NS holds the start of window x
  auto saved_field = [&](int slot, int m, int f) {
    return saved + (((size_t)slot * nm + m) * 3 + f) * field_elems;
  };
  // per member and slot: the window whose start the slot holds, and the
  // window (if it is the same one) the surrogate advanced the member in
  std::vector<int> saved_at(NS * nm, -1), accepted_at(NS * nm, -1);
  // latest window x in [w - d_hi, w - d_lo] the surrogate advanced member m
  // in whose start is saved, as w - x; -1 when none
  auto back_to = [&](int m, int w, int d_lo, int d_hi) {
    for (int d = d_lo; d <= d_hi; ++d) {
      const int x = w - d;
      if (x < 0) break;
      if (saved_at[NS * m + x % NS] == x && accepted_at[NS * m + x % NS] == x) return d;
    }
    return -1;
  };
  const long long launches0 = s->nlaunch;
  long long solver_launches = 0;  // one persistent ensemble launch per solver step
  // Members with sel[m] go back to the state saved in `slot` (the start of
  // step istp_from + 1) and the solver runs them n steps (n even, so their
  // state buffers keep their parity).
  auto rewind_to = [&](int slot, const char* sel, int istp_from, int n, int count) -> int {
    for (int m = 0; m < nm; ++m) {
      if (!sel[m]) continue;
      double* dst[3] = {ms[m].sshn, ms[m].un, ms[m].vn};
      for (int f = 0; f < 3; ++f) {
        const int r = status_of(cudaMemcpyAsync(dst[f], saved_field(slot, m, f), field_elems * sizeof(double),
                                                cudaMemcpyDeviceToDevice, s->stream));
        if (r != NEMO_OK) return r;
      }
    }
    int r = join(s->stream, nemo::ens_stream(e));
    if (r == NEMO_OK) r = nemo::ens_step_subset(e, istp_from + 1, n, sel);
    if (r != NEMO_OK) return r;
    solver_launches += n;
    st.solver_steps += (long long)n * count;
    st.rewound += count;
    return NEMO_OK;
  };
  const auto t_start = std::chrono::steady_clock::now();
  int istp = istp0;
  int rc = NEMO_OK;
  const int rest = c->anchor - c->k;
  for (int w = 0; w < nsteps / c->anchor && rc == NEMO_OK; ++w) {
    // every member's state is final once the solver work queued so far is done
    rc = join(nemo::ens_stream(e), s->stream);
    if (rc != NEMO_OK) break;
    if (saved) {  // the window's starting states, while the members are still in them
      for (int m = 0; m < nm && rc == NEMO_OK; ++m) {
        if (quar[m]) continue;
        double* src[3] = {ms[m].sshn, ms[m].un, ms[m].vn};
        for (int f = 0; f < 3 && rc == NEMO_OK; ++f)
          rc = status_of(cudaMemcpyAsync(saved_field(w % NS, m, f), src[f], field_elems * sizeof(double),
                                         cudaMemcpyDeviceToDevice, s->stream));
        saved_at[NS * m + w % NS] = w;
      }
      if (rc != NEMO_OK) break;
    }
    for (int i = 0; i < nm; ++i) tide[i] = nemo::ens_tide(e, i, istp + c->k);
    for (int m0 = 0; m0 < nm && rc == NEMO_OK; m0 += s->cfg.batch) {
      const int n = nm - m0 < s->cfg.batch ? nm - m0 : s->cfg.batch;
      rc = predict_chunk(s, m0, n, tide, snap_all + (size_t)m0 * hw * 4, out_all + (size_t)m0 * out_per);
    }
    // shadow / re-anchor: the FP64 solver runs the same k steps
    if (rc == NEMO_OK) rc = join(s->stream, nemo::ens_stream(e));
    if (rc == NEMO_OK) rc = nemo_ens_step_n(e, istp + 1, c->k);
    solver_launches += c->k;
    if (rc == NEMO_OK) rc = join(nemo::ens_stream(e), s->stream);
    if (rc == NEMO_OK) rc = ensure_members(s, e, ms, nullptr);  // buffers swapped
    if (rc != NEMO_OK) break;
    cudaError_t ce = cudaMemsetAsync(s->d_acc, 0, 6 * nm * sizeof(double), s->stream);
    if (ce == cudaSuccess) ce = launch_err(s, nm, snap_all, out_all, corr);
    if (ce == cudaSuccess)
      ce = cudaMemcpyAsync(acc.data(), s->d_acc, 6 * nm * sizeof(double), cudaMemcpyDeviceToHost, s->stream);
    if (ce != cudaSuccess) { rc = status_of(ce); break; }
    if ((rc = check_err(s)) != NEMO_OK) break;
    // a non-finite error (a member whose state blew up) counts as a failure
    double worst = 0.0;
    int nfail = 0;
    std::vector<char> back[NS];
    int nback[NS] = {0};
    for (int d = 1; d < NS; ++d) back[d].assign(nm, 0);
    for (int m = 0; m < nm; ++m) {
      const double r = acc[6 * m + 1] > 0 ? sqrt(acc[6 * m] / acc[6 * m + 1]) : sqrt(acc[6 * m]);
      if (c->quarantine > 0 && !quar[m] && !(r <= c->quarantine)) {
        quar[m] = 1;  // far off: the solver keeps this member from now on
        st.quarantined += 1;
        // back to the start of the latest window the surrogate advanced it in
        const int d = saved ? back_to(m, w, 1, NS - 1) : -1;
        if (d > 0) back[d][m] = 1, nback[d] += 1;
      }
      fail[m] = quar[m] || !(r <= c->tol);
      nfail += fail[m];
      if (!(r <= worst)) worst = r;  // NaN propagates
    }
    // the solver re-runs the windows from there and this window's first k steps
    for (int d = 1; d < NS && rc == NEMO_OK; ++d)
      if (nback[d] > 0)
        rc = rewind_to((w - d) % NS, back[d].data(), istp - d * c->anchor, d * c->anchor + c->k, nback[d]);
    if (rc != NEMO_OK) break;
    if (!c->per_member && nfail > 0) {
      for (int m = 0; m < nm; ++m) fail[m] = 1;
      nfail = nm;
    }
    for (int m = 0; m < nm; ++m) {
      pass[m] = !fail[m];
      accepted_at[NS * m + w % NS] = pass[m] ? w : -1;
    }
    st.last_shadow_err = worst;
    if (!(worst <= st.max_shadow_err)) st.max_shadow_err = worst;
    st.windows += nm;
    st.fallbacks += nfail;
    st.solver_steps += (long long)c->k * nm;
    st.sur_calls += 1;
    istp += c->k;
    if (nfail == nm) {  // the whole ensemble: the graph-captured path
      rc = nemo_ens_step_n(e, istp + 1, rest);
    } else if (nfail > 0) {
      rc = nemo::ens_step_subset(e, istp + 1, rest, fail.data());
    }
    if (nfail > 0) solver_launches += rest;
    st.solver_steps += (long long)rest * nfail;
    if (rc != NEMO_OK) break;
    if (nfail < nm) {
      // the accepted members' surrogate calls overlap the fallen-back
      // members' solver steps (disjoint states; the next window starts after both)
      if (corr)
        for (int m = 0; m < nm; ++m) ms[m].corr = corr + (size_t)m * hw * 4;
      for (int j = c->k; j < c->anchor && rc == NEMO_OK; j += c->k) {
        rc = advance_members(s, e, ms, pass.data(), istp + j);
        st.sur_calls += 1;
        st.sur_steps += (long long)c->k * (nm - nfail);
      }
      if (rc == NEMO_OK) rc = check_err(s);
      if (rc == NEMO_OK) rc = join(s->stream, nemo::ens_stream(e));
      if (rc == NEMO_OK) rc = ensure_members(s, e, ms, nullptr);  // all members' table again
    }
    istp += rest;
  }
  // The last window meets no later shadow check.  A member it left diverged
  // (a non-finite value, or |ssh| above 10 times its tidal amplitude) goes
  // back: to the window's start when the surrogate advanced it there, else
  // (the solver ran it, from a state earlier surrogate calls may have led
  // astray) to the previous window's start; the solver runs the windows from
  // there.
  if (rc == NEMO_OK && saved && nsteps > 0) {
    const int wl = nsteps / c->anchor - 1;
    int* d_flag = nullptr;
    double* d_lim = nullptr;
    std::vector<int> flag(nm, 0);
    std::vector<double> lim(nm);
    for (int m = 0; m < nm; ++m) {  // no tide: only non-finite values count
      const double a = nemo::ens_amp(e, m);
      lim[m] = a > 0.0 ? 10.0 * a : INFINITY;
    }
    cudaError_t fe = nemo::dev_alloc(&d_lim, nm * (sizeof(double) + sizeof(int)));
    if (fe == cudaSuccess) {
      d_flag = reinterpret_cast<int*>(d_lim + nm);
      fe = join(nemo::ens_stream(e), s->stream) == NEMO_OK ? cudaSuccess : cudaErrorUnknown;
    }
    if (fe == cudaSuccess) fe = cudaMemsetAsync(d_flag, 0, nm * sizeof(int), s->stream);
    if (fe == cudaSuccess)
      fe = cudaMemcpyAsync(d_lim, lim.data(), nm * sizeof(double), cudaMemcpyHostToDevice, s->stream);
    if (fe == cudaSuccess) {
      k_diverged<<<dim3(64, (unsigned)nm), 256, 0, s->stream>>>(s->d_ms, d_lim, d_flag);
      s->nlaunch += 1;
      fe = cudaGetLastError();
    }
    if (fe == cudaSuccess) fe = cudaMemcpyAsync(flag.data(), d_flag, nm * sizeof(int), cudaMemcpyDeviceToHost, s->stream);
    if (fe == cudaSuccess) fe = cudaStreamSynchronize(s->stream);
    if (d_lim) cudaFree(d_lim);
    if (fe != cudaSuccess) rc = status_of(fe);
    // back to the start of the latest window the surrogate advanced the
    // member in (the last one included); with none saved it stays as it is
    std::vector<char> back[NS];
    int nback[NS] = {0};
    for (int d = 0; d < NS; ++d) back[d].assign(nm, 0);
    for (int m = 0; m < nm; ++m) {
      if (!flag[m]) continue;
      const int d = back_to(m, wl, 0, NS - 1);
      if (d >= 0) back[d][m] = 1, nback[d] += 1;
    }
    for (int d = 0; d < NS && rc == NEMO_OK; ++d)
      if (nback[d] > 0)
        rc = rewind_to((wl - d) % NS, back[d].data(), istp - (d + 1) * c->anchor, (d + 1) * c->anchor, nback[d]);
  }
  cudaError_t ce = cudaStreamSynchronize(nemo::ens_stream(e));
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(s->stream);
  if (own) cudaFree(own);
  if (saved) cudaFree(saved);
  if (corr) cudaFree(corr);
  if (rc != NEMO_OK) return rc;
  ECK(ce);
  st.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
  st.launches = solver_launches + (s->nlaunch - launches0);
  if (stats) *stats = st;
  return NEMO_OK;
}

// ---- single kernels on caller-owned device buffers (for parity tests) -------
int nemo_conv3x3_fwd(const void* x, const void* w, const float* bias, const void* residual, const void* mask,
                     int relu, void* out, float* out32, int n, int h, int wd, int* err, void* stream) {
  if (!x || !w || !err || (!out && !out32)) return NEMO_ERR_INVALID;
  sur::ConvEpi e{bias, (const __nv_bfloat16*)residual, (const __nv_bfloat16*)mask, (__nv_bfloat16*)out, out32,
                 relu, n, h, wd, err};
  ECK(sur::conv_fwd((const __nv_bfloat16*)x, (const __nv_bfloat16*)w, e, (cudaStream_t)stream));
  return NEMO_OK;
}

int nemo_conv3x3_fwd_variant(int variant, int rows) { return sur::set_fwd_variant(variant, rows); }

int nemo_conv3x3_wgrad_variant(int variant) { return sur::set_wgrad_variant(variant); }

int nemo_debug_conv_wait(unsigned long long wait_ns, int skip_launches) {
  if (skip_launches < 0) return NEMO_ERR_INVALID;
  sur::set_test_wait(wait_ns, skip_launches);
  return NEMO_OK;
}

int nemo_conv3x3_wgrad(const void* x, const void* dz, float* dw, float* db, int n, int h, int wd, int ctas,
                       int* err, void* stream) {
  if (!x || !dz || !dw || !err) return NEMO_ERR_INVALID;
  sur::WgradArgs a{dw, db, n, h, wd, err, nullptr, 0};
  ECK(sur::conv_wgrad((const __nv_bfloat16*)x, (const __nv_bfloat16*)dz, a, ctas, (cudaStream_t)stream));
  return NEMO_OK;
}

}  // extern "C"
