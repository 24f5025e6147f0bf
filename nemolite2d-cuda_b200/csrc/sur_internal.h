// Internals of the BF16 convolutional surrogate shared between its
// translation units.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "nemo_alloc.h"
#include "nemo_b200.h"

namespace sur {

// Fused epilogue of a 3x3 convolution (64 -> 64 channels, NHWC BF16):
//   v = acc + bias; v += residual; v *= (mask > 0); v = max(v, 0) if relu;
//   out <- bf16(v) (64 channels), out32 <- v[0:out32_ch] (FP32, out32_ch per
//   pixel; out32_ch a multiple of 4 up to 64, 0 meaning 4).
// Every pointer but err may be null.
struct ConvEpi {
  const float* bias;
  const __nv_bfloat16* residual;
  const __nv_bfloat16* mask;
  __nv_bfloat16* out;
  float* out32;
  int relu;
  int N, H, W;
  int* err;  // device flag, first failing wait's code
  int out32_ch;
  // set by conv_fwd from the process-wide test settings (set_test_wait):
  unsigned long long wait_ns;  // limit of the main waits; 0: the default 2 s
  int skip_load;               // 1: CTA 0 omits its first input-row load
};

// Test settings of the forward kernel's failure path: the next conv_fwd
// launches use `wait_ns` for their main waits (0: the default 2 s), and the
// next `skip_launches` of them have CTA 0 omit one input-row load, so that a
// wait for it runs out without any fault.  Returns the previous wait limit.
unsigned long long set_test_wait(unsigned long long wait_ns, int skip_launches);

// dw[tap][co][ci] += sum_p dz[p][co] x[p + off(tap)][ci]; db[co] += sum_p dz[p][co].
// One CTA's partial weight and bias gradient in the default (strip) kernel.
constexpr int WS_NPART = 9 * 64 * 64 + 64;

struct WgradArgs {
  float* dw;
  float* db;
  int N, H, W;
  int* err;
  // scratch of the default kernel: partial_blocks rows of WS_NPART floats, one
  // per CTA, summed in a fixed order afterwards; null: a scratch array the
  // library keeps per device (calls that overlap on the GPU then race on it)
  float* partial;
  int partial_blocks;
};

// W % 128 == 0, x and w 16-byte aligned; w = [9][64 out][64 in] BF16.
cudaError_t conv_fwd(const __nv_bfloat16* x, const __nv_bfloat16* w, const ConvEpi& epi, cudaStream_t s);
// Process-wide choice of the forward kernel: 2 = three output rows per MMA
// (default), 1 = row ring, 0 = a TMA window per tap; rows per strip of the
// ring kernels.  Returns the previous variant; out-of-range values leave the
// setting unchanged.
int set_fwd_variant(int variant, int rows);
// Process-wide choice of the weight-gradient kernel: 2 = all taps per CTA over
// column strips, summed in a fixed order (default, deterministic), 1 = three
// vertical taps per MMA, 0 = tap pairs (1 and 0 add with atomics).  Returns the
// previous variant.
int set_wgrad_variant(int variant);
// Kernels one conv_wgrad call launches with the current variant.
int wgrad_kernels();
// W % 64 == 0.  ctas <= 0 picks the count from the SM count.
cudaError_t conv_wgrad(const __nv_bfloat16* x, const __nv_bfloat16* dz, const WgradArgs& g, int ctas,
                       cudaStream_t s);

}  // namespace sur

namespace nemo {
// Current-state view of one ensemble member (device pointers, pitched
// single-grid layout: element (ji, jj) at (jj + 1) * pitch + ji + 2).
struct MemberState {
  double *sshn, *un, *vn;
  const double *ht, *hv;
  const double* sshv0;  // stored sshn_v (row jj = 0: the open boundary's)
  int jpi, jpj, pitch;
  // hybrid only: the shadow step's correction of a surrogate call, 4 floats
  // (ssh, u, v, unused) per T-cell in row-major order, added by every call
  // (null: none)
  const float* corr;
};
int ens_member_state(nemo_ens* e, int m, MemberState* out);
int ens_member_count(nemo_ens* e);
// Advances only the members with sel[m] != 0 by an even number n of steps.
int ens_step_subset(nemo_ens* e, int istp0, int n, const char* sel);
cudaStream_t ens_stream(nemo_ens* e);
int ens_device(nemo_ens* e);
// Tidal SSH a member's boundary row holds after step istp.
double ens_tide(nemo_ens* e, int m, int istp);
// A member's tidal amplitude.
double ens_amp(nemo_ens* e, int m);
}  // namespace nemo
