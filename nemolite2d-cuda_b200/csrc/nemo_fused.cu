// Fused NEMOLite2D step: continuity + momentum (u, v) + all boundary
// conditions + next in one pass over HBM (original/nemolite2d.f90:375-769).
//
// Work decomposition: one warp owns a strip of 30 T columns and marches north
// over a block of rows; lane l holds column c0+l-1, so lanes 0 and 31 are
// halo lanes whose results are only used by their neighbours.  Per row each
// lane loads its own sshn, un, vn, ht, hu, hv (one row ahead, prefetched),
// and the values of columns c-1 / c+1 come from warp shuffles: no shared
// memory, no block barriers.  The reference's `next` copies become a swap of
// the two state buffers.
//
// Every quantity the reference evaluates twice -- the upwind flux through a
// face shared by two velocity points, the velocity gradients, sshn_u/sshn_v
// -- is evaluated once (x-faces by the lane east of the face, y-faces
// carried in registers from the previous row).  Each reuse is an identical
// expression tree up to commutation of + and *, so with contraction off the
// results are bit-identical to the reference.
//
// Divisions by grid constants and by the static depths use the
// corrected-reciprocal quotient with host-formed RN(1/b) (RN(1/hu), RN(1/hv)
// are stored fields).  A row whose three rows of state hold a nonzero value
// below 2^-300 anywhere in the warp is computed with IEEE division instead
// (warp-uniform, so the common path stays branch-free); see qdiv.
//
// Row staging: PF = 2 (the default schedule) copies every row two rows
// ahead of its use into a per-warp ring in shared memory with cp.async, so
// DRAM latency is hidden without registers held for the prefetch; PF = 1
// prefetches into registers, PF = 0 loads each row one iteration ahead.
//
// Masks are those of the reference geometry (walls at ji=0, jpi+1 and
// jj=jpj+1, open boundary at jj=0), evaluated from the indices.
#include "nemo_step_dev.cuh"

namespace nemo {
namespace {
using namespace stepdev;

// NWARPS warps per CTA; MINB > 0 asks the compiler to fit MINB CTAs per SM
// (register cap 65536 / (32*NWARPS*MINB)).  PF: 1 prefetches row j+2 into
// registers while row j is computed; 0 loads row j+1 at the top of each
// iteration (fewer live registers).
template <int NWARPS, int MINB, int PF>
__global__ void __launch_bounds__(32 * NWARPS, MINB)
k_fused_step(Layout L, Consts C, FusedArgs A, int tile_y) {
  const int lane = threadIdx.x & 31;
  const int warp = (int)(blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5));
  const int c0 = 1 + COLS_PER_WARP * warp;
  if (c0 > L.jpi) return;  // whole warp idle
  const int J0 = 1 + (int)blockIdx.y * tile_y;
  if (J0 > L.jpj) return;
  const int J1 = min(J0 + tile_y - 1, L.jpj);
  if constexpr (PF >= 2) {
    constexpr int RD = ring_doubles<PF == 3>();
    __shared__ double ring[NWARPS * RD];
    run_strip_ring<PF == 3, 2>(L, C, A, c0, J0, J1, lane, ring + (threadIdx.x >> 5) * RD);
  } else {
    run_strip<PF>(L, C, A, c0, J0, J1, lane);
  }
}

}  // namespace

template <int NW, int MB, int PF>
static cudaError_t launch_variant(const Layout& L, const Consts& C, const FusedArgs& a, int tile_y,
                                  cudaStream_t s) {
  const int cols_per_cta = COLS_PER_WARP * NW;
  const int gx = (L.jpi + cols_per_cta - 1) / cols_per_cta;
  if (tile_y <= 0) {
    // single wave: as many row blocks as the resident CTA slots allow
    static int slots = 0;  // CTAs of this variant resident on the whole device
    if (slots == 0) {
      int dev = 0, sms = 0, per_sm = 0;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fused_step<NW, MB, PF>, 32 * NW, 0);
      slots = sms * (per_sm > 0 ? per_sm : 1);
    }
    int nrb = slots / gx;
    if (nrb < 1) nrb = 1;
    tile_y = (L.jpj + nrb - 1) / nrb;
  }
  dim3 grid((unsigned)gx, (unsigned)((L.jpj + tile_y - 1) / tile_y));
  k_fused_step<NW, MB, PF><<<grid, 32 * NW, 0, s>>>(L, C, a, tile_y);
  return cudaGetLastError();
}

// warps: 2, 4 or 8 per CTA; occ: register budget as resident warps per SM
// (0: compiler's choice, 16, 20, 24) with the register prefetch of the next
// row; a negative occ: the same budget without it; 100 + budget (116, 120):
// rows staged through the shared-memory ring; 200 + budget (216, 220): the
// ring with the reciprocal depths formed in the kernel.
cudaError_t launch_fused_step(const Layout& L, const Consts& C, const FusedArgs& a, int warps,
                              int occ, int tile_y, cudaStream_t s) {
  if (warps == 2) {
    switch (occ) {
      case 216: return launch_variant<2, 8, 3>(L, C, a, tile_y, s);
      case 220: return launch_variant<2, 10, 3>(L, C, a, tile_y, s);
      case 116: return launch_variant<2, 8, 2>(L, C, a, tile_y, s);
      case 120: return launch_variant<2, 10, 2>(L, C, a, tile_y, s);
      case 0: return launch_variant<2, 1, 1>(L, C, a, tile_y, s);
      case 16: return launch_variant<2, 8, 1>(L, C, a, tile_y, s);
      case 20: return launch_variant<2, 10, 1>(L, C, a, tile_y, s);
      case 24: return launch_variant<2, 12, 1>(L, C, a, tile_y, s);
      case -16: return launch_variant<2, 8, 0>(L, C, a, tile_y, s);
      case -20: return launch_variant<2, 10, 0>(L, C, a, tile_y, s);
      case -24: return launch_variant<2, 12, 0>(L, C, a, tile_y, s);
    }
  } else if (warps == 4) {
    switch (occ) {
      case 216: return launch_variant<4, 4, 3>(L, C, a, tile_y, s);
      case 220: return launch_variant<4, 5, 3>(L, C, a, tile_y, s);
      case 116: return launch_variant<4, 4, 2>(L, C, a, tile_y, s);
      case 120: return launch_variant<4, 5, 2>(L, C, a, tile_y, s);
      case 0: return launch_variant<4, 1, 1>(L, C, a, tile_y, s);
      case 16: return launch_variant<4, 4, 1>(L, C, a, tile_y, s);
      case 20: return launch_variant<4, 5, 1>(L, C, a, tile_y, s);
      case 24: return launch_variant<4, 6, 1>(L, C, a, tile_y, s);
      case -20: return launch_variant<4, 5, 0>(L, C, a, tile_y, s);
    }
  } else if (warps == 8) {
    switch (occ) {
      case 0: return launch_variant<8, 1, 1>(L, C, a, tile_y, s);
      case 16: return launch_variant<8, 2, 1>(L, C, a, tile_y, s);
      case 24: return launch_variant<8, 3, 1>(L, C, a, tile_y, s);
    }
  }
  return cudaErrorInvalidValue;
}

}  // namespace nemo

namespace nemo {
bool fused_variant_ok(int warps, int occ, bool nr_ok) {
  if ((occ == 216 || occ == 220) && (warps == 2 || warps == 4)) return nr_ok;
  if (warps == 2) return occ == 0 || occ == 16 || occ == 20 || occ == 24 || occ == -16 ||
                         occ == -20 || occ == -24 || occ == 116 || occ == 120;
  if (warps == 4) return occ == 0 || occ == 16 || occ == 20 || occ == 24 || occ == -20 || occ == 116 ||
                         occ == 120;
  if (warps == 8) return occ == 0 || occ == 16 || occ == 24;
  return false;
}
}  // namespace nemo
