// Per-routine kernels: one thread per grid point, each a statement-for-
// statement rendering of one loop nest of original/nemolite2d.f90 (same
// bounds, CYCLE conditions and left-to-right evaluation).  They serve the
// routine-boundary API (continuity / momentum / bc / next called one by one,
// as cuda/nemolite2d.f90:486-489 does) and initialisation.
#include "nemo_internal.h"

namespace nemo {
namespace {

constexpr int BX = 32, BY = 8;

inline dim3 grid_for(int ni, int nj) {
  return dim3((unsigned)((ni + BX - 1) / BX), (unsigned)((nj + BY - 1) / BY));
}

// SIGN(a,b), gfortran semantics
__device__ __forceinline__ double fsign(double a, double b) { return copysign(fabs(a), b); }

// Grid accessors of the routine kernels: each metric at the point the
// reference indexes it.  UniGrid is the reference's uniform grid (the
// constants, the analytic mask), so its instantiations evaluate the same
// expressions as kernels written with the constants; ArrGrid reads a general
// grid's arrays (nemo_set_grid).
struct UniGrid {
  Consts C;
  int jpi, jpj;
  __device__ int pt(int a, int b) const { return ptmask(a, b, jpi, jpj); }
  __device__ double e1t(int, int) const { return C.e1t; }
  __device__ double e2t(int, int) const { return C.e2t; }
  __device__ double e1u(int, int) const { return C.e1u; }
  __device__ double e2u(int, int) const { return C.e2u; }
  __device__ double e1v(int, int) const { return C.e1v; }
  __device__ double e2v(int, int) const { return C.e2v; }
  __device__ double e12t(int, int) const { return C.e12t; }
  __device__ double e12u(int, int) const { return C.e12u; }
  __device__ double e12v(int, int) const { return C.e12v; }
  __device__ double fcu(int, int) const { return C.fcor; }
  __device__ double fcv(int, int) const { return C.fcor; }
};

struct ArrGrid {
  Layout L;
  GridDev d;
  __device__ int pt(int a, int b) const { return d.pt[L.idx(a, b)]; }
  __device__ double e1t(int a, int b) const { return d.e1t[L.idx(a, b)]; }
  __device__ double e2t(int a, int b) const { return d.e2t[L.idx(a, b)]; }
  __device__ double e1u(int a, int b) const { return d.e1u[L.idx(a, b)]; }
  __device__ double e2u(int a, int b) const { return d.e2u[L.idx(a, b)]; }
  __device__ double e1v(int a, int b) const { return d.e1v[L.idx(a, b)]; }
  __device__ double e2v(int a, int b) const { return d.e2v[L.idx(a, b)]; }
  __device__ double e12t(int a, int b) const { return d.e12t[L.idx(a, b)]; }
  __device__ double e12u(int a, int b) const { return d.e12u[L.idx(a, b)]; }
  __device__ double e12v(int a, int b) const { return d.e12v[L.idx(a, b)]; }
  __device__ double fcu(int a, int b) const { return d.fcu[L.idx(a, b)]; }
  __device__ double fcv(int a, int b) const { return d.fcv[L.idx(a, b)]; }
};

// Launches kernel K on stream st with the accessor of grid g (null: the
// uniform grid).
#define WITH_GRID(K, grid, block, st, L, C, g, ...)                                     \
  do {                                                                                  \
    if (g)                                                                              \
      K<ArrGrid><<<(grid), (block), 0, (st)>>>(L, ArrGrid{L, *(g)}, __VA_ARGS__);       \
    else                                                                                \
      K<UniGrid><<<(grid), (block), 0, (st)>>>(L, UniGrid{C, L.jpi, L.jpj}, __VA_ARGS__); \
  } while (0)

// Seeded bathymetry (no reference counterpart): depth at half-grid point
// (kx,ky) = clamp(H0 + sum_b ax[b][kx]*gy[b][ky]), summed in b order with
// separate roundings; uniform dep_const when nbump == 0 (:238-254).
__device__ double depth_at(int kx, int ky, int nkx, int nky, double dep_const, int nbump,
                           const double* ax, const double* gy, double hmin, double hmax) {
  if (nbump <= 0) return dep_const;
  double acc = 0.0;
  for (int b = 0; b < nbump; ++b)
    acc = __dadd_rn(acc, __dmul_rn(ax[(long)b * nkx + kx], gy[(long)b * nky + ky]));
  double h = __dadd_rn(dep_const, acc);
  h = h < hmin ? hmin : h;
  h = h > hmax ? hmax : h;
  return h;
}

__global__ void k_depth(Layout L, double dep_const, int nbump, const double* ax,
                        const double* gy, double hmin, double hmax, double* ht, double* hu,
                        double* hv) {
  int ji = blockIdx.x * BX + threadIdx.x;     // 0..jpi
  int jj = blockIdx.y * BY + threadIdx.y;     // 0..jpj
  if (ji > L.jpi || jj > L.jpj) return;
  int nkx = 2 * L.jpi + 2, nky = 2 * L.jpj + 2;
  if (ji >= 1 && jj >= 1)
    ht[L.idx(ji, jj)] = depth_at(2 * ji - 1, 2 * jj - 1, nkx, nky, dep_const, nbump, ax, gy, hmin, hmax);
  if (jj >= 1)
    hu[L.idx(ji, jj)] = depth_at(2 * ji, 2 * jj - 1, nkx, nky, dep_const, nbump, ax, gy, hmin, hmax);
  if (ji >= 1)
    hv[L.idx(ji, jj)] = depth_at(2 * ji - 1, 2 * jj, nkx, nky, dep_const, nbump, ax, gy, hmin, hmax);
}

// initialisation, original/nemolite2d.f90:337-353 (min/max-clamped averages)
template <class G>
__global__ void k_init_sshn_uv(Layout L, G g, const double* sshn, double* sshn_u, double* sshn_v) {
  int ji = blockIdx.x * BX + threadIdx.x;  // 0..jpi
  int jj = blockIdx.y * BY + threadIdx.y;  // 0..jpj
  const int jpi = L.jpi, jpj = L.jpj;
  if (ji > jpi || jj > jpj) return;
  if (jj >= 1) {
    int i1 = min(ji + 1, jpi), i2 = max(ji, 1);
    double r = g.e12t(i1, jj) * sshn[L.idx(i1, jj)] + g.e12t(i2, jj) * sshn[L.idx(i2, jj)];
    sshn_u[L.idx(ji, jj)] = 0.5 * r / g.e12u(ji, jj);
  }
  if (ji >= 1) {
    int j1 = min(jj + 1, jpj), j2 = max(jj, 1);
    double r = g.e12t(ji, j1) * sshn[L.idx(ji, j1)] + g.e12t(ji, j2) * sshn[L.idx(ji, j2)];
    sshn_v[L.idx(ji, jj)] = 0.5 * r / g.e12v(ji, jj);
  }
}

// continuity, :397-405
template <class G>
__global__ void k_continuity(Layout L, G g, Consts C, RoutinePtrs p) {
  int ji = 1 + blockIdx.x * BX + threadIdx.x;
  int jj = 1 + blockIdx.y * BY + threadIdx.y;
  if (ji > L.jpi || jj > L.jpj) return;
  double r1 = (p.sshn_u[L.idx(ji, jj)] + p.hu[L.idx(ji, jj)]) * p.un[L.idx(ji, jj)];
  double r2 = (p.sshn_u[L.idx(ji - 1, jj)] + p.hu[L.idx(ji - 1, jj)]) * p.un[L.idx(ji - 1, jj)];
  double r3 = (p.sshn_v[L.idx(ji, jj)] + p.hv[L.idx(ji, jj)]) * p.vn[L.idx(ji, jj)];
  double r4 = (p.sshn_v[L.idx(ji, jj - 1)] + p.hv[L.idx(ji, jj - 1)]) * p.vn[L.idx(ji, jj - 1)];
  p.ssha[L.idx(ji, jj)] = p.sshn[L.idx(ji, jj)] + (r2 - r1 + r4 - r3) * C.rdt / g.e12t(ji, jj);
}

// momentum, u equation, :431-517 (ssha_u is identically zero, :37, :315)
template <class G>
__global__ void k_momentum_u(Layout L, G g, Consts C, RoutinePtrs p) {
  int ji = 1 + blockIdx.x * BX + threadIdx.x;  // 1..jpi-1
  int jj = 1 + blockIdx.y * BY + threadIdx.y;  // 1..jpj
  const int jpi = L.jpi, jpj = L.jpj;
  if (ji > jpi - 1 || jj > jpj) return;
#define PT(a, b) g.pt((a), (b))
#define F(arr, a, b) p.arr[L.idx((a), (b))]
  if (PT(ji, jj) + PT(ji + 1, jj) <= 0) return;
  if (PT(ji, jj) <= 0 || PT(ji + 1, jj) <= 0) return;

  double u_e = 0.5 * (F(un, ji, jj) + F(un, ji + 1, jj)) * g.e2t(ji + 1, jj);
  double depe = F(ht, ji + 1, jj) + F(sshn, ji + 1, jj);
  double u_w = 0.5 * (F(un, ji, jj) + F(un, ji - 1, jj)) * g.e2t(ji, jj);
  double depw = F(ht, ji, jj) + F(sshn, ji, jj);

  double v_sc = 0.5 * (F(vn, ji, jj - 1) + F(vn, ji + 1, jj - 1));
  double v_s = 0.5 * v_sc * (g.e1v(ji, jj - 1) + g.e1v(ji + 1, jj - 1));
  double deps = 0.5 * (F(hv, ji, jj - 1) + F(sshn_v, ji, jj - 1) + F(hv, ji + 1, jj - 1) +
                       F(sshn_v, ji + 1, jj - 1));
  double v_nc = 0.5 * (F(vn, ji, jj) + F(vn, ji + 1, jj));
  double v_n = 0.5 * v_nc * (g.e1v(ji, jj) + g.e1v(ji + 1, jj));
  double depn = 0.5 * (F(hv, ji, jj) + F(sshn_v, ji, jj) + F(hv, ji + 1, jj) + F(sshn_v, ji + 1, jj));

  double uu_w = (0.5 - fsign(0.5, u_w)) * F(un, ji, jj) + (0.5 + fsign(0.5, u_w)) * F(un, ji - 1, jj);
  double uu_e = (0.5 + fsign(0.5, u_e)) * F(un, ji, jj) + (0.5 - fsign(0.5, u_e)) * F(un, ji + 1, jj);
  double uu_s, uu_n;
  if (PT(ji, jj - 1) <= 0 || PT(ji + 1, jj - 1) <= 0)
    uu_s = (0.5 - fsign(0.5, v_s)) * F(un, ji, jj);
  else
    uu_s = (0.5 - fsign(0.5, v_s)) * F(un, ji, jj) + (0.5 + fsign(0.5, v_s)) * F(un, ji, jj - 1);
  if (PT(ji, jj + 1) <= 0 || PT(ji + 1, jj + 1) <= 0)
    uu_n = (0.5 + fsign(0.5, v_n)) * F(un, ji, jj);
  else
    uu_n = (0.5 + fsign(0.5, v_n)) * F(un, ji, jj) + (0.5 - fsign(0.5, v_n)) * F(un, ji, jj + 1);

  double adv = uu_w * u_w * depw - uu_e * u_e * depe + uu_s * v_s * deps - uu_n * v_n * depn;

  double dudx_e = (F(un, ji + 1, jj) - F(un, ji, jj)) / g.e1t(ji + 1, jj) * (F(ht, ji + 1, jj) + F(sshn, ji + 1, jj));
  double dudx_w = (F(un, ji, jj) - F(un, ji - 1, jj)) / g.e1t(ji, jj) * (F(ht, ji, jj) + F(sshn, ji, jj));
  double dudy_s, dudy_n;
  if (PT(ji, jj - 1) <= 0 || PT(ji + 1, jj - 1) <= 0)
    dudy_s = 0.0;
  else
    dudy_s = (F(un, ji, jj) - F(un, ji, jj - 1)) / (g.e2u(ji, jj) + g.e2u(ji, jj - 1)) *
             (F(hu, ji, jj) + F(sshn_u, ji, jj) + F(hu, ji, jj - 1) + F(sshn_u, ji, jj - 1));
  if (PT(ji, jj + 1) <= 0 || PT(ji + 1, jj + 1) <= 0)
    dudy_n = 0.0;
  else
    dudy_n = (F(un, ji, jj + 1) - F(un, ji, jj)) / (g.e2u(ji, jj) + g.e2u(ji, jj + 1)) *
             (F(hu, ji, jj) + F(sshn_u, ji, jj) + F(hu, ji, jj + 1) + F(sshn_u, ji, jj + 1));

  double vis = (dudx_e - dudx_w) * g.e2u(ji, jj) + (dudy_n - dudy_s) * g.e1u(ji, jj) * 0.5;
  vis = C.visc * vis;
  double cor = 0.5 * (g.fcu(ji, jj) * (v_sc + v_nc)) * g.e12u(ji, jj) * (F(hu, ji, jj) + F(sshn_u, ji, jj));
  double hpg = -(C.g * (F(hu, ji, jj) + F(sshn_u, ji, jj)) * g.e2u(ji, jj) * (F(sshn, ji + 1, jj) - F(sshn, ji, jj)));
  F(ua, ji, jj) = (F(un, ji, jj) * (F(hu, ji, jj) + F(sshn_u, ji, jj)) +
                   C.rdt * (adv + vis + cor + hpg) / g.e12u(ji, jj)) /
                  (F(hu, ji, jj) + 0.0) / C.cfric;
}

// momentum, v equation, :520-609
template <class G>
__global__ void k_momentum_v(Layout L, G g, Consts C, RoutinePtrs p) {
  int ji = 1 + blockIdx.x * BX + threadIdx.x;  // 1..jpi
  int jj = 1 + blockIdx.y * BY + threadIdx.y;  // 1..jpj-1
  const int jpi = L.jpi, jpj = L.jpj;
  if (ji > jpi || jj > jpj - 1) return;
  // the reference tests pt(ji+1,jj) here (:523); kept verbatim
  if (PT(ji, jj) + PT(ji + 1, jj) <= 0) return;
  if (PT(ji, jj) <= 0 || PT(ji, jj + 1) <= 0) return;

  double v_n = 0.5 * (F(vn, ji, jj) + F(vn, ji, jj + 1)) * g.e1t(ji, jj + 1);
  double depn = F(ht, ji, jj + 1) + F(sshn, ji, jj + 1);
  double v_s = 0.5 * (F(vn, ji, jj) + F(vn, ji, jj - 1)) * g.e1t(ji, jj);
  double deps = F(ht, ji, jj) + F(sshn, ji, jj);

  double u_wc = 0.5 * (F(un, ji - 1, jj) + F(un, ji - 1, jj + 1));
  double u_w = 0.5 * u_wc * (g.e2u(ji - 1, jj) + g.e2u(ji - 1, jj + 1));
  double depw = 0.50 * (F(hu, ji - 1, jj) + F(sshn_u, ji - 1, jj) + F(hu, ji - 1, jj + 1) +
                        F(sshn_u, ji - 1, jj + 1));
  double u_ec = 0.5 * (F(un, ji, jj) + F(un, ji, jj + 1));
  double u_e = 0.5 * u_ec * (g.e2u(ji, jj) + g.e2u(ji, jj + 1));
  double depe = 0.50 * (F(hu, ji, jj) + F(sshn_u, ji, jj) + F(hu, ji, jj + 1) + F(sshn_u, ji, jj + 1));

  double vv_s = (0.5 - fsign(0.5, v_s)) * F(vn, ji, jj) + (0.5 + fsign(0.5, v_s)) * F(vn, ji, jj - 1);
  double vv_n = (0.5 + fsign(0.5, v_n)) * F(vn, ji, jj) + (0.5 - fsign(0.5, v_n)) * F(vn, ji, jj + 1);
  double vv_w, vv_e;
  if (PT(ji - 1, jj) <= 0 || PT(ji - 1, jj + 1) <= 0)
    vv_w = (0.5 - fsign(0.5, u_w)) * F(vn, ji, jj);
  else
    vv_w = (0.5 - fsign(0.5, u_w)) * F(vn, ji, jj) + (0.5 + fsign(0.5, u_w)) * F(vn, ji - 1, jj);
  if (PT(ji + 1, jj) <= 0 || PT(ji + 1, jj + 1) <= 0)
    vv_e = (0.5 + fsign(0.5, u_e)) * F(vn, ji, jj);
  else
    vv_e = (0.5 + fsign(0.5, u_e)) * F(vn, ji, jj) + (0.5 - fsign(0.5, u_e)) * F(vn, ji + 1, jj);

  double adv = vv_w * u_w * depw - vv_e * u_e * depe + vv_s * v_s * deps - vv_n * v_n * depn;

  double dvdy_n = (F(vn, ji, jj + 1) - F(vn, ji, jj)) / g.e2t(ji, jj + 1) * (F(ht, ji, jj + 1) + F(sshn, ji, jj + 1));
  double dvdy_s = (F(vn, ji, jj) - F(vn, ji, jj - 1)) / g.e2t(ji, jj) * (F(ht, ji, jj) + F(sshn, ji, jj));
  double dvdx_w, dvdx_e;
  if (PT(ji - 1, jj) <= 0 || PT(ji - 1, jj + 1) <= 0)
    dvdx_w = 0.0;
  else
    dvdx_w = (F(vn, ji, jj) - F(vn, ji - 1, jj)) / (g.e1v(ji, jj) + g.e1v(ji - 1, jj)) *
             (F(hv, ji, jj) + F(sshn_v, ji, jj) + F(hv, ji - 1, jj) + F(sshn_v, ji - 1, jj));
  if (PT(ji + 1, jj) <= 0 || PT(ji + 1, jj + 1) <= 0)
    dvdx_e = 0.0;
  else
    dvdx_e = (F(vn, ji + 1, jj) - F(vn, ji, jj)) / (g.e1v(ji, jj) + g.e1v(ji + 1, jj)) *
             (F(hv, ji, jj) + F(sshn_v, ji, jj) + F(hv, ji + 1, jj) + F(sshn_v, ji + 1, jj));

  double vis = (dvdy_n - dvdy_s) * g.e1v(ji, jj) + (dvdx_e - dvdx_w) * g.e2v(ji, jj) * 0.5;
  vis = C.visc * vis;
  double cor = -0.5 * (g.fcv(ji, jj) * (u_ec + u_wc)) * g.e12v(ji, jj) * (F(hv, ji, jj) + F(sshn_v, ji, jj));
  double hpg = -(C.g * (F(hv, ji, jj) + F(sshn_v, ji, jj)) * g.e1v(ji, jj) * (F(sshn, ji, jj + 1) - F(sshn, ji, jj)));
  F(va, ji, jj) = (F(vn, ji, jj) * (F(hv, ji, jj) + F(sshn_v, ji, jj)) +
                   C.rdt * (adv + vis + cor + hpg) / g.e12v(ji, jj)) /
                  ((F(hv, ji, jj) + 0.0)) / C.cfric;
}

// bc: clamped SSH, :631-644 (value = amp*sin(omega_tide*rtime) from the host)
template <class G>
__global__ void k_bc_ssh(Layout L, G g, double value, double* ssha) {
  int ji = 1 + blockIdx.x * BX + threadIdx.x;
  int jj = 1 + blockIdx.y * BY + threadIdx.y;
  const int jpi = L.jpi, jpj = L.jpj;
  if (ji > jpi || jj > jpj) return;
  if (PT(ji, jj) <= 0) return;
  if (PT(ji, jj - 1) < 0 || PT(ji, jj + 1) < 0 || PT(ji + 1, jj) < 0 || PT(ji - 1, jj) < 0)
    ssha[L.idx(ji, jj)] = value;
}

// bc: solid u, :648-652
template <class G>
__global__ void k_bc_solid_u(Layout L, G g, double* ua) {
  int ji = blockIdx.x * BX + threadIdx.x;      // 0..jpi
  int jj = 1 + blockIdx.y * BY + threadIdx.y;  // 1..jpj
  const int jpi = L.jpi, jpj = L.jpj;
  if (ji > jpi || jj > jpj) return;
  if (PT(ji, jj) * PT(ji + 1, jj) == 0) ua[L.idx(ji, jj)] = 0.0;
}

// bc: solid v, :656-660
template <class G>
__global__ void k_bc_solid_v(Layout L, G g, double* va) {
  int ji = 1 + blockIdx.x * BX + threadIdx.x;  // 1..jpi
  int jj = blockIdx.y * BY + threadIdx.y;      // 0..jpj
  const int jpi = L.jpi, jpj = L.jpj;
  if (ji > jpi || jj > jpj) return;
  if (PT(ji, jj) * PT(ji, jj + 1) == 0) va[L.idx(ji, jj)] = 0.0;
}

// bc: Flather u, :669-680.  The reference sweeps ji in order, in place; one
// thread per row keeps that order.
template <class G>
__global__ void k_bc_flather_u(Layout L, G g, RoutinePtrs p) {
  int jj = 1 + blockIdx.x * blockDim.x + threadIdx.x;  // 1..jpj
  const int jpi = L.jpi, jpj = L.jpj;
  if (jj > jpj) return;
  for (int ji = 0; ji <= jpi; ++ji) {
    if (PT(ji, jj) + PT(ji + 1, jj) <= -1) continue;
    if (PT(ji, jj) < 0) {
      int jiu = ji + 1;
      F(ua, ji, jj) = F(ua, jiu, jj) + sqrt(kG / F(hu, ji, jj)) * (F(sshn_u, ji, jj) - F(sshn_u, jiu, jj));
    } else if (PT(ji + 1, jj) < 0) {
      int jiu = ji - 1;
      F(ua, ji, jj) = F(ua, jiu, jj) + sqrt(kG / F(hu, ji, jj)) * (F(sshn_u, ji, jj) - F(sshn_u, jiu, jj));
    }
  }
}

// bc: Flather v, :684-695.  In-place dependence runs along jj, so one thread
// per column sweeps jj in the reference's order.
template <class G>
__global__ void k_bc_flather_v(Layout L, G g, RoutinePtrs p) {
  int ji = 1 + blockIdx.x * blockDim.x + threadIdx.x;  // 1..jpi
  const int jpi = L.jpi, jpj = L.jpj;
  if (ji > jpi) return;
  for (int jj = 0; jj <= jpj; ++jj) {
    if (PT(ji, jj) + PT(ji, jj + 1) <= -1) continue;
    if (PT(ji, jj) < 0) {
      int jiv = jj + 1;
      F(va, ji, jj) = F(va, ji, jiv) + sqrt(kG / F(hv, ji, jj)) * (F(sshn_v, ji, jj) - F(sshn_v, ji, jiv));
    } else if (PT(ji, jj + 1) < 0) {
      int jiv = jj - 1;
      F(va, ji, jj) = F(va, ji, jiv) + sqrt(kG / F(hv, ji, jj)) * (F(sshn_v, ji, jj) - F(sshn_v, ji, jiv));
    }
  }
}

// next, copies, :712-732
__global__ void k_copy_next(Layout L, RoutinePtrs p) {
  int ji = blockIdx.x * BX + threadIdx.x;  // 0..jpi
  int jj = blockIdx.y * BY + threadIdx.y;  // 0..jpj
  const int jpi = L.jpi, jpj = L.jpj;
  if (ji > jpi || jj > jpj) return;
  if (jj >= 1) F(un, ji, jj) = F(ua, ji, jj);
  if (ji >= 1) F(vn, ji, jj) = F(va, ji, jj);
  if (ji >= 1 && jj >= 1) F(sshn, ji, jj) = F(ssha, ji, jj);
}

// next, sshn_u/sshn_v re-interpolation, :736-764
template <class G>
__global__ void k_derive_sshn_uv(Layout L, G g, const double* sshn, double* sshn_u, double* sshn_v) {
  int ji = blockIdx.x * BX + threadIdx.x;  // 0..jpi
  int jj = blockIdx.y * BY + threadIdx.y;  // 0..jpj
  const int jpi = L.jpi, jpj = L.jpj;
  if (ji > jpi || jj > jpj) return;
  if (jj >= 1 && !(PT(ji, jj) + PT(ji + 1, jj) <= 0)) {
    double v;
    bool set = true;
    if (PT(ji, jj) * PT(ji + 1, jj) > 0) {
      double r = g.e12t(ji, jj) * sshn[L.idx(ji, jj)] + g.e12t(ji + 1, jj) * sshn[L.idx(ji + 1, jj)];
      v = 0.5 * r / g.e12u(ji, jj);
    } else if (PT(ji, jj) <= 0) {
      v = sshn[L.idx(ji + 1, jj)];
    } else if (PT(ji + 1, jj) <= 0) {
      v = sshn[L.idx(ji, jj)];
    } else {
      set = false;
      v = 0.0;
    }
    if (set) sshn_u[L.idx(ji, jj)] = v;
  }
  if (ji >= 1 && !(PT(ji, jj) + PT(ji, jj + 1) <= 0)) {
    double v;
    bool set = true;
    if (PT(ji, jj) * PT(ji, jj + 1) > 0) {
      double r = g.e12t(ji, jj) * sshn[L.idx(ji, jj)] + g.e12t(ji, jj + 1) * sshn[L.idx(ji, jj + 1)];
      v = 0.5 * r / g.e12v(ji, jj);
    } else if (PT(ji, jj) <= 0) {
      v = sshn[L.idx(ji, jj + 1)];
    } else if (PT(ji, jj + 1) <= 0) {
      v = sshn[L.idx(ji, jj)];
    } else {
      set = false;
      v = 0.0;
    }
    if (set) sshn_v[L.idx(ji, jj)] = v;
  }
}
#undef PT
#undef F

}  // namespace

cudaError_t launch_depth(const Layout& L, double dep_const, int nbump, const double* ax,
                         const double* gy, double hmin, double hmax, double* ht, double* hu,
                         double* hv, cudaStream_t s) {
  k_depth<<<grid_for(L.jpi + 1, L.jpj + 1), dim3(BX, BY), 0, s>>>(L, dep_const, nbump, ax, gy,
                                                                   hmin, hmax, ht, hu, hv);
  return cudaGetLastError();
}

// RN(1/hu), RN(1/hv) by IEEE division (0 where the depth is 0); counts the
// cells where recip_nr differs from it in `mismatch`.
__global__ void k_recip(long n, const double* __restrict__ hu, const double* __restrict__ hv,
                        double* __restrict__ rhu, double* __restrict__ rhv, int* __restrict__ mismatch) {
  int bad = 0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const double a = hu[i] + 0.0, b = hv[i] + 0.0;
    const double ra = a != 0.0 ? 1.0 / a : 0.0, rb = b != 0.0 ? 1.0 / b : 0.0;
    rhu[i] = ra;
    rhv[i] = rb;
    if (a != 0.0 && __double_as_longlong(recip_nr(a)) != __double_as_longlong(ra)) ++bad;
    if (b != 0.0 && __double_as_longlong(recip_nr(b)) != __double_as_longlong(rb)) ++bad;
  }
  if (bad) atomicAdd(mismatch, bad);
}

cudaError_t launch_recip(const Layout& L, const double* hu, const double* hv, double* rhu, double* rhv,
                         int* mismatch, cudaStream_t s) {
  const long n = L.elems();
  long g = (n + 255) / 256;
  if (g > 4096) g = 4096;
  k_recip<<<(unsigned)g, 256, 0, s>>>(n, hu, hv, rhu, rhv, mismatch);
  return cudaGetLastError();
}

// Output record (original/nemolite2d.f90:785-790): sshn, 0.5*(un(ji-1)+un(ji)),
// 0.5*(vn(jj-1)+vn(jj)) at every T-cell, as three dense [jpj][jpi] planes.
__global__ void k_record(Layout L, const double* __restrict__ sshn, const double* __restrict__ un,
                         const double* __restrict__ vn, double* __restrict__ out) {
  const int ji = 1 + blockIdx.x * BX + threadIdx.x;
  const int jj = 1 + blockIdx.y * BY + threadIdx.y;
  if (ji > L.jpi || jj > L.jpj) return;
  const long plane = (long)L.jpi * L.jpj;
  const long t = (long)(jj - 1) * L.jpi + (ji - 1);
  out[t] = sshn[L.idx(ji, jj)];
  out[plane + t] = 0.5 * (un[L.idx(ji - 1, jj)] + un[L.idx(ji, jj)]);
  out[2 * plane + t] = 0.5 * (vn[L.idx(ji, jj - 1)] + vn[L.idx(ji, jj)]);
}

cudaError_t launch_record(const Layout& L, const double* sshn, const double* un, const double* vn, double* out,
                          cudaStream_t s) {
  k_record<<<grid_for(L.jpi, L.jpj), dim3(BX, BY), 0, s>>>(L, sshn, un, vn, out);
  return cudaGetLastError();
}

cudaError_t launch_init_sshn_uv(const Layout& L, const Consts& C, const double* sshn,
                                double* sshn_u, double* sshn_v, cudaStream_t s, const GridDev* g) {
  WITH_GRID(k_init_sshn_uv, grid_for(L.jpi + 1, L.jpj + 1), dim3(BX, BY), s, L, C, g, sshn, sshn_u, sshn_v);
  return cudaGetLastError();
}

cudaError_t launch_continuity(const Layout& L, const Consts& C, const RoutinePtrs& p,
                              cudaStream_t s, const GridDev* g) {
  WITH_GRID(k_continuity, grid_for(L.jpi, L.jpj), dim3(BX, BY), s, L, C, g, C, p);
  return cudaGetLastError();
}

cudaError_t launch_momentum_u(const Layout& L, const Consts& C, const RoutinePtrs& p,
                              cudaStream_t s, const GridDev* g) {
  if (L.jpi < 2) return cudaSuccess;
  WITH_GRID(k_momentum_u, grid_for(L.jpi - 1, L.jpj), dim3(BX, BY), s, L, C, g, C, p);
  return cudaGetLastError();
}

cudaError_t launch_momentum_v(const Layout& L, const Consts& C, const RoutinePtrs& p,
                              cudaStream_t s, const GridDev* g) {
  if (L.jpj < 2) return cudaSuccess;
  WITH_GRID(k_momentum_v, grid_for(L.jpi, L.jpj - 1), dim3(BX, BY), s, L, C, g, C, p);
  return cudaGetLastError();
}

cudaError_t launch_bc_ssh(const Layout& L, double value, double* ssha, cudaStream_t s, const GridDev* g) {
  const Consts C{};  // the uniform grid's mask needs no constants
  WITH_GRID(k_bc_ssh, grid_for(L.jpi, L.jpj), dim3(BX, BY), s, L, C, g, value, ssha);
  return cudaGetLastError();
}

cudaError_t launch_bc_solid_u(const Layout& L, double* ua, cudaStream_t s, const GridDev* g) {
  const Consts C{};
  WITH_GRID(k_bc_solid_u, grid_for(L.jpi + 1, L.jpj), dim3(BX, BY), s, L, C, g, ua);
  return cudaGetLastError();
}

cudaError_t launch_bc_solid_v(const Layout& L, double* va, cudaStream_t s, const GridDev* g) {
  const Consts C{};
  WITH_GRID(k_bc_solid_v, grid_for(L.jpi, L.jpj + 1), dim3(BX, BY), s, L, C, g, va);
  return cudaGetLastError();
}

cudaError_t launch_bc_flather_u(const Layout& L, const RoutinePtrs& p, cudaStream_t s, const GridDev* g) {
  const Consts C{};
  WITH_GRID(k_bc_flather_u, (L.jpj + 127) / 128, 128, s, L, C, g, p);
  return cudaGetLastError();
}

cudaError_t launch_bc_flather_v(const Layout& L, const RoutinePtrs& p, cudaStream_t s, const GridDev* g) {
  const Consts C{};
  WITH_GRID(k_bc_flather_v, (L.jpi + 127) / 128, 128, s, L, C, g, p);
  return cudaGetLastError();
}

cudaError_t launch_copy_next(const Layout& L, const RoutinePtrs& p, cudaStream_t s) {
  k_copy_next<<<grid_for(L.jpi + 1, L.jpj + 1), dim3(BX, BY), 0, s>>>(L, p);
  return cudaGetLastError();
}

cudaError_t launch_derive_sshn_uv(const Layout& L, const Consts& C, const double* sshn,
                                  double* sshn_u, double* sshn_v, cudaStream_t s, const GridDev* g) {
  WITH_GRID(k_derive_sshn_uv, grid_for(L.jpi + 1, L.jpj + 1), dim3(BX, BY), s, L, C, g, sshn, sshn_u, sshn_v);
  return cudaGetLastError();
}

}  // namespace nemo
