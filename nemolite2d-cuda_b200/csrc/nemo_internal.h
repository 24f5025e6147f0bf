// Host-side internals shared by the library's translation units.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "nemo_alloc.h"
#include "nemo_b200.h"
#include "nemo_common.cuh"

namespace nemo {

// Device pointers of one state set (the reference's "n" or "a" fields).
struct StateSet {
  double* ssh;
  double* u;
  double* v;
};

struct RoutinePtrs {
  double *sshn, *un, *vn, *ssha, *ua, *va, *sshn_u, *sshn_v, *ht, *hu, *hv;
};

// A general grid (nemo_set_grid): the mask pt (1 water, 0 land, -1 open) and
// the metrics as arrays in the fields' layout; fcu, fcv = 2*omega*sin(gphi*d2r)
// at u and v points.  The per-routine launchers take a GridDev pointer, null
// for the reference's uniform grid (constants and the analytic mask).
struct GridDev {
  const signed char* pt;
  const double *e1t, *e2t, *e1u, *e2u, *e1v, *e2v, *e12t, *e12u, *e12v, *fcu, *fcv;
};

// ---- launchers (asynchronous on `s`) -------------------------------------
cudaError_t launch_depth(const Layout& L, double dep_const, int nbump, const double* ax,
                         const double* gy, double hmin, double hmax, double* ht,
                         double* hu, double* hv, cudaStream_t s);
// rhu = RN(1/hu), rhv = RN(1/hv) over the whole storage (0 where the depth is 0);
// adds to *mismatch (device) the number of depths whose recip_nr is not RN(1/h).
cudaError_t launch_recip(const Layout& L, const double* hu, const double* hv, double* rhu, double* rhv,
                         int* mismatch,
                         cudaStream_t s);
cudaError_t launch_init_sshn_uv(const Layout& L, const Consts& C, const double* sshn,
                                double* sshn_u, double* sshn_v, cudaStream_t s,
                                const GridDev* g = nullptr);
cudaError_t launch_continuity(const Layout& L, const Consts& C, const RoutinePtrs& p,
                              cudaStream_t s, const GridDev* g = nullptr);
cudaError_t launch_momentum_u(const Layout& L, const Consts& C, const RoutinePtrs& p,
                              cudaStream_t s, const GridDev* g = nullptr);
cudaError_t launch_momentum_v(const Layout& L, const Consts& C, const RoutinePtrs& p,
                              cudaStream_t s, const GridDev* g = nullptr);
cudaError_t launch_bc_ssh(const Layout& L, double value, double* ssha, cudaStream_t s,
                          const GridDev* g = nullptr);
cudaError_t launch_bc_solid_u(const Layout& L, double* ua, cudaStream_t s, const GridDev* g = nullptr);
cudaError_t launch_bc_solid_v(const Layout& L, double* va, cudaStream_t s, const GridDev* g = nullptr);
cudaError_t launch_bc_flather_u(const Layout& L, const RoutinePtrs& p, cudaStream_t s,
                                const GridDev* g = nullptr);
cudaError_t launch_bc_flather_v(const Layout& L, const RoutinePtrs& p, cudaStream_t s,
                                const GridDev* g = nullptr);
cudaError_t launch_copy_next(const Layout& L, const RoutinePtrs& p, cudaStream_t s);
// sshn and the cell-centred velocities as three dense [jpj][jpi] planes.
cudaError_t launch_record(const Layout& L, const double* sshn, const double* un, const double* vn, double* out,
                          cudaStream_t s);
cudaError_t launch_derive_sshn_uv(const Layout& L, const Consts& C, const double* sshn,
                                  double* sshn_u, double* sshn_v, cudaStream_t s,
                                  const GridDev* g = nullptr);

struct FusedArgs {
  const double *sshn, *un, *vn, *ht, *hu, *hv;
  const double *rhu, *rhv;  // RN(1/hu), RN(1/hv): divisors of the u and v updates
  const double* sshv0;  // stored sshn_v array (only its row jj=0 is read)
  double *ssha, *ua, *va;
  double tide;          // clamped SSH value for this step
};
// warps per CTA (2, 4, 8), register budget as resident warps per SM (0, 16,
// 20, 24; negative: same budget without the next-row register prefetch), rows
// per CTA (0: one wave).
cudaError_t launch_fused_step(const Layout& L, const Consts& C, const FusedArgs& a, int warps,
                              int occ, int tile_y, cudaStream_t s);
// nr_ok: the grid's depths passed launch_recip's check (variants 216, 220).
bool fused_variant_ok(int warps, int occ, bool nr_ok);

// Fused step of a general grid (nemo_fused_general.cu).  su_st, sv_st: the
// stored sshn_u / sshn_v, read where `next` leaves them unchanged.
struct GenArgs {
  const double *sshn, *un, *vn, *ht, *hu, *hv;
  const double *su_st, *sv_st;
  double *ssha, *ua, *va;
  double tide;
  GridDev g;
};
// One step: the fused kernel, then the Flather chains (flather_chains).
// ring: 0 (rows loaded where used), 3 or 4 (rows staged through a shared-memory
// ring of that many slots); tile_y: rows per CTA.
cudaError_t launch_fused_general(const Layout& L, const Consts& C, const GenArgs& a, const int4* chains,
                                 int nchains, int ring, int tile_y, cudaStream_t s);
// Flather points of the mask pt ((0:jpi+1, 0:jpj+1), leading dimension
// jpi+2) as independent chains: {ji, jj, kind, continues}.
void flather_chains(const int* pt, int jpi, int jpj, std::vector<int4>& out);

// Sums |f(1:jpi,1:jpj)| of nf fields into out[0..nf-1] (device), fixed order.
// row_partials: nf*jpj doubles of scratch.
cudaError_t launch_checksums(const Layout& L, const double* const* fields, int nf,
                             double* row_partials, double* out, cudaStream_t s);

// Host helpers.
void depth_tables(const nemo_params& p, double* ax, double* gy);  // sizes nbump*(2*jpi+2), nbump*(2*jpj+2)
double tide_value(const nemo_params& p, int istp);
Consts make_consts(const nemo_params& p);

}  // namespace nemo
