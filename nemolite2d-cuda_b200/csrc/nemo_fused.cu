// Fused NEMOLite2D step: continuity + momentum (u, v) + all boundary
// conditions + next in one pass over HBM (original/nemolite2d.f90:375-769).
//
// Each thread owns a pair of T columns (i, i+1), i odd, so every load and
// store of its own columns is one 16-byte access, and marches north over a
// strip of rows.  Per row it reads the next row of sshn, un, vn, ht, hu, hv
// and writes ssha, ua, va of the current row into the other state buffer
// (the reference's `next` copies become a buffer swap).  Quantities the
// reference evaluates twice -- the upwind flux through a face shared by two
// velocity points, the velocity gradients, the interpolated sshn_u/sshn_v --
// are evaluated once here and carried: south-face values in registers from
// the previous row, the x-face between the two owned columns reused
// directly.  Each of these reuses is an identical expression tree (only
// commutations of + and * differ), so results are bit-identical to the
// reference when contraction is off.  Divisions by grid constants use the
// corrected-reciprocal quotient (div_const), which is the correctly rounded
// quotient; divisions by the depth fields stay IEEE divisions.
//
// Masks are the reference geometry's (walls at ji=0, jpi+1 and jj=jpj+1,
// open boundary at jj=0), evaluated from the indices.
#include "nemo_internal.h"

namespace nemo {
namespace {

struct Row {
  double s[4];   // sshn at i-1 .. i+2
  double u[4];   // un   at i-1 .. i+2
  double v[4];   // vn   at i-1 .. i+2
  double ht[3];  // ht   at i   .. i+2
  double hu[3];  // hu   at i-1 .. i+1
  double hv[4];  // hv   at i-1 .. i+2
};

__device__ __forceinline__ double ld1(const double* p) { return __ldg(p); }
__device__ __forceinline__ void ld2(const double* p, double& a, double& b) {
  double2 t = __ldg(reinterpret_cast<const double2*>(p));
  a = t.x;
  b = t.y;
}

__device__ __forceinline__ void load_row(Row& r, const FusedArgs& A, long base) {
  // base = index of (i, row); i odd so base is even (16-byte aligned)
  r.s[0] = ld1(A.sshn + base - 1);
  ld2(A.sshn + base, r.s[1], r.s[2]);
  r.s[3] = ld1(A.sshn + base + 2);
  r.u[0] = ld1(A.un + base - 1);
  ld2(A.un + base, r.u[1], r.u[2]);
  r.u[3] = ld1(A.un + base + 2);
  r.v[0] = ld1(A.vn + base - 1);
  ld2(A.vn + base, r.v[1], r.v[2]);
  r.v[3] = ld1(A.vn + base + 2);
  ld2(A.ht + base, r.ht[0], r.ht[1]);
  r.ht[2] = ld1(A.ht + base + 2);
  r.hu[0] = ld1(A.hu + base - 1);
  ld2(A.hu + base, r.hu[1], r.hu[2]);
  r.hv[0] = ld1(A.hv + base - 1);
  ld2(A.hv + base, r.hv[1], r.hv[2]);
  r.hv[3] = ld1(A.hv + base + 2);
}

// sshn_u at column c of a row from sshn(c), sshn(c+1) (:736-746)
__device__ __forceinline__ double interp_u(const Consts& C, int c, int jpi, double s0, double s1) {
  if (c == 0) return s1;
  if (c == jpi) return s0;
  return div_const(0.5 * (C.e12t * s0 + C.e12t * s1), C.e12u, C.r_e12u);
}
// sshn_v between rows jj and jj+1 (jj in 1..jpj; :752-763); jj == 0 is the
// stored open-boundary row and is handled by the caller.
__device__ __forceinline__ double interp_v(const Consts& C, int jj, int jpj, double s0, double s1) {
  if (jj == jpj) return s0;
  return div_const(0.5 * (C.e12t * s0 + C.e12t * s1), C.e12v, C.r_e12v);
}

__global__ void __launch_bounds__(128)
k_fused_step(Layout L, Consts C, FusedArgs A, int tile_y) {
  const int jpi = L.jpi, jpj = L.jpj;
  const int i = 1 + 2 * (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (i > jpi) return;
  const bool two = (i + 1 <= jpi);
  const int J0 = 1 + (int)blockIdx.y * tile_y;
  if (J0 > jpj) return;
  const int J1 = min(J0 + tile_y - 1, jpj);

  Row cur, nx;
  // ---- prologue: carried values for row J0 from rows J0-1 and J0 ---------
  double su_c[3], Hu_c[3];        // sshn_u and hu+sshn_u at row j, cols i-1..i+1
  double Fuy_s[2], dudy_s[2];     // u-eq south-face flux and dudy_s for row j
  double vnc_s[2];                // v_sc of u(c,j)
  double Fvy_s[2], Dvy_s[2];      // v-eq south-face flux and dvdy_s for row j
  double cf_s[2];                 // continuity south flux (sshn_v+hv)*vn at jj-1
  double sv0[2] = {0.0, 0.0}, hv0[2] = {0.0, 0.0};  // open boundary row (Flather)
  {
    Row pr;
    load_row(pr, A, L.idx(i, J0 - 1));
    load_row(cur, A, L.idx(i, J0));
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      su_c[k] = interp_u(C, i + k - 1, jpi, cur.s[k], cur.s[k + 1]);
      Hu_c[k] = cur.hu[k] + su_c[k];
    }
    double sv_p[4], Hv_p[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (J0 == 1)
        sv_p[k] = __ldg(A.sshv0 + L.idx(i + k - 1, 0));
      else
        sv_p[k] = interp_v(C, J0 - 1, jpj, pr.s[k], cur.s[k]);
      Hv_p[k] = pr.hv[k] + sv_p[k];
    }
#pragma unroll
    for (int l = 0; l < 2; ++l) {
      // corner (i+l, J0-1): south face of u(i+l, J0)
      double vnc = 0.5 * (pr.v[l + 1] + pr.v[l + 2]);
      double vn_ = 0.5 * vnc * C.two_dx;
      double dep = 0.5 * ((Hv_p[l + 1] + pr.hv[l + 2]) + sv_p[l + 2]);
      double uu = (J0 == 1) ? upwind_hi_only(vn_, cur.u[l + 1])
                            : upwind(vn_, pr.u[l + 1], cur.u[l + 1]);
      Fuy_s[l] = uu * vn_ * dep;
      vnc_s[l] = vnc;
      if (J0 == 1) {
        dudy_s[l] = 0.0;
      } else {
        double su_p = interp_u(C, i + l, jpi, pr.s[l + 1], pr.s[l + 2]);
        double gy = div_const(cur.u[l + 1] - pr.u[l + 1], C.two_dy, C.r_2dy);
        dudy_s[l] = gy * ((Hu_c[l + 1] + pr.hu[l + 1]) + su_p);
      }
      // T(i+l, J0): south face of v(i+l, J0)
      double vlo = pr.v[l + 1], vhi = cur.v[l + 1];
      double vs = 0.5 * (vhi + vlo) * C.e1t;
      double depc = cur.ht[l] + cur.s[l + 1];
      Fvy_s[l] = upwind(vs, vlo, vhi) * vs * depc;
      Dvy_s[l] = div_const(vhi - vlo, C.e2t, C.r_e2t) * depc;
      cf_s[l] = Hv_p[l + 1] * pr.v[l + 1];
      if (J0 == 1) {
        sv0[l] = sv_p[l + 1];
        hv0[l] = pr.hv[l + 1];
      }
    }
  }

  for (int j = J0; j <= J1; ++j) {
    load_row(nx, A, L.idx(i, j + 1));
    const bool south = (j == 1), north = (j == jpj);

    // sshn_v and hv+sshn_v at row j, cols i-1..i+2
    double sv[4], Hv[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      sv[k] = interp_v(C, j, jpj, cur.s[k], nx.s[k]);
      Hv[k] = cur.hv[k] + sv[k];
    }
    // sshn_u and hu+sshn_u at row j+1, cols i-1..i+1
    double su_n[3], Hu_n[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      su_n[k] = interp_u(C, i + k - 1, jpi, nx.s[k], nx.s[k + 1]);
      Hu_n[k] = nx.hu[k] + su_n[k];
    }

    // x-faces of the u equation at T(c,j), c = i .. i+2 (between u(c-1), u(c))
    double Fx[3], Dx[3];
#pragma unroll
    for (int l = 0; l < 3; ++l) {
      double ulo = cur.u[l], uhi = cur.u[l + 1];
      double uw = 0.5 * (uhi + ulo) * C.e2t;
      double dep = cur.ht[l] + cur.s[l + 1];
      Fx[l] = upwind(uw, ulo, uhi) * uw * dep;
      Dx[l] = div_const(uhi - ulo, C.e1t, C.r_e1t) * dep;
    }

    // corners (c, j), c = i-1 .. i+1: east face of v(c,j); north face of u(c,j)
    double Fvx[3], Gx[3], uec[3], Sn[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const int c = i + k - 1;
      uec[k] = 0.5 * (cur.u[k] + nx.u[k]);
      double ue = 0.5 * uec[k] * C.two_dy;
      Sn[k] = (Hu_c[k] + nx.hu[k]) + su_n[k];
      double depe = 0.5 * Sn[k];
      double vlo = cur.v[k], vhi = cur.v[k + 1];
      double uu = (c == 0) ? upwind_hi_only(ue, vhi)
                           : (c == jpi) ? upwind_lo_only(ue, vlo) : upwind(ue, vlo, vhi);
      Fvx[k] = uu * ue * depe;
      Gx[k] = div_const(vhi - vlo, C.two_dx, C.r_2dx);
    }
    double Fuy[2], Re[2], vnc[2], Gy[2];
#pragma unroll
    for (int l = 0; l < 2; ++l) {
      const int k = l + 1;  // corner index of column i+l
      vnc[l] = 0.5 * (cur.v[k] + cur.v[k + 1]);
      double vn_ = 0.5 * vnc[l] * C.two_dx;
      Re[l] = (Hv[k] + cur.hv[k + 1]) + sv[k + 1];
      double depn = 0.5 * Re[l];
      double ulo = cur.u[k], uhi = nx.u[k];
      double uu = north ? upwind_lo_only(vn_, ulo) : upwind(vn_, ulo, uhi);
      Fuy[l] = uu * vn_ * depn;
      Gy[l] = div_const(uhi - ulo, C.two_dy, C.r_2dy);
    }

    // v-eq faces at T(c, j+1), c = i, i+1 (between v(c,j) and v(c,j+1))
    double Fvy_n[2], Dvy_n[2];
#pragma unroll
    for (int l = 0; l < 2; ++l) {
      double vlo = cur.v[l + 1], vhi = nx.v[l + 1];
      double vs = 0.5 * (vhi + vlo) * C.e1t;
      double dep = nx.ht[l] + nx.s[l + 1];
      Fvy_n[l] = upwind(vs, vlo, vhi) * vs * dep;
      Dvy_n[l] = div_const(vhi - vlo, C.e2t, C.r_e2t) * dep;
    }

    double ssha[2], ua[2], va[2];
#pragma unroll
    for (int l = 0; l < 2; ++l) {
      const int c = i + l;
      // continuity (:399-403) and the clamped SSH row (:631-644)
      double r1 = Hu_c[l + 1] * cur.u[l + 1];
      double r2 = Hu_c[l] * cur.u[l];
      double r3 = Hv[l + 1] * cur.v[l + 1];
      double r4 = cf_s[l];
      double ssh = cur.s[l + 1] + div_const((r2 - r1 + r4 - r3) * C.rdt, C.e12t, C.r_e12t);
      ssha[l] = south ? A.tide : ssh;
      cf_s[l] = r3;

      // u equation (:439-514); u(jpi,j) is the east wall (:650)
      {
        double adv = Fx[l] - Fx[l + 1] + Fuy_s[l] - Fuy[l];
        double dudy_n = north ? 0.0 : Gy[l] * Sn[l + 1];
        double dudy_sl = south ? 0.0 : dudy_s[l];
        double vis = (Dx[l + 1] - Dx[l]) * C.e2u + (dudy_n - dudy_sl) * C.e1u * 0.5;
        vis = C.visc * vis;
        double Hu = Hu_c[l + 1];
        double cor = 0.5 * (C.fcor * (vnc_s[l] + vnc[l])) * C.e12u * Hu;
        double hpg = -(C.g * Hu * C.e2u * (cur.s[l + 2] - cur.s[l + 1]));
        double num = cur.u[l + 1] * Hu +
                     div_const(C.rdt * (adv + vis + cor + hpg), C.e12u, C.r_e12u);
        double q = num / (cur.hu[l + 1] + 0.0);
        ua[l] = (c == jpi) ? 0.0 : div_const(q, C.cfric, C.r_cfric);
      }
      // v equation (:527-606); v(c,jpj) is the north wall (:658)
      {
        double adv = Fvx[l] - Fvx[l + 1] + Fvy_s[l] - Fvy_n[l];
        double dvdx_e = (c == jpi) ? 0.0 : Gx[l + 1] * Re[l];
        double dvdx_w = (c == 1) ? 0.0 : Gx[l] * ((Hv[l + 1] + cur.hv[l]) + sv[l]);
        double vis = (Dvy_n[l] - Dvy_s[l]) * C.e1v + (dvdx_e - dvdx_w) * C.e2v * 0.5;
        vis = C.visc * vis;
        double Hv_ = Hv[l + 1];
        double cor = -(0.5 * (C.fcor * (uec[l + 1] + uec[l])) * C.e12v * Hv_);
        double hpg = -(C.g * Hv_ * C.e1v * (nx.s[l + 1] - cur.s[l + 1]));
        double num = cur.v[l + 1] * Hv_ +
                     div_const(C.rdt * (adv + vis + cor + hpg), C.e12v, C.r_e12v);
        double q = num / (cur.hv[l + 1] + 0.0);
        va[l] = north ? 0.0 : div_const(q, C.cfric, C.r_cfric);
      }
    }

    // ---- stores ----------------------------------------------------------
    const long o = L.idx(i, j);
    if (two) {
      *reinterpret_cast<double2*>(A.ssha + o) = make_double2(ssha[0], ssha[1]);
      *reinterpret_cast<double2*>(A.ua + o) = make_double2(ua[0], ua[1]);
      *reinterpret_cast<double2*>(A.va + o) = make_double2(va[0], va[1]);
    } else {
      A.ssha[o] = ssha[0];
      A.ua[o] = ua[0];
      A.va[o] = va[0];
    }
    if (i == 1) A.ua[o - 1] = 0.0;  // u(0,j), west wall (:650)
    if (south) {
      // Flather open boundary, v(c,0) = v(c,1) + sqrt(g/hv)*(sshn_v(c,0)-sshn_v(c,1))  (:684-695)
      const long o0 = L.idx(i, 0);
      double f0 = va[0] + sqrt(kG / hv0[0]) * (sv0[0] - sv[1]);
      double f1 = va[1] + sqrt(kG / hv0[1]) * (sv0[1] - sv[2]);
      if (two) {
        *reinterpret_cast<double2*>(A.va + o0) = make_double2(f0, f1);
      } else {
        A.va[o0] = f0;
      }
    }

    // ---- carry to row j+1 ------------------------------------------------
#pragma unroll
    for (int l = 0; l < 2; ++l) {
      Fuy_s[l] = Fuy[l];
      // dudy_s of u(c, j+1): ((un(j+1)-un(j))/(e2u+e2u)) * (Hu(j+1) + hu(j) + sshn_u(j))
      dudy_s[l] = Gy[l] * ((Hu_n[l + 1] + cur.hu[l + 1]) + su_c[l + 1]);
      vnc_s[l] = vnc[l];
      Fvy_s[l] = Fvy_n[l];
      Dvy_s[l] = Dvy_n[l];
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      su_c[k] = su_n[k];
      Hu_c[k] = Hu_n[k];
    }
    cur = nx;
  }
}

}  // namespace

cudaError_t launch_fused_step(const Layout& L, const Consts& C, const FusedArgs& a, int tile_x,
                              int tile_y, cudaStream_t s) {
  // tile_x = T columns per CTA (two per thread)
  int threads = tile_x / 2;
  if (threads < 32) threads = 32;
  if (threads > 128) threads = 128;
  int cols_per_cta = 2 * threads;
  dim3 grid((unsigned)((L.jpi + cols_per_cta - 1) / cols_per_cta),
            (unsigned)((L.jpj + tile_y - 1) / tile_y));
  k_fused_step<<<grid, threads, 0, s>>>(L, C, a, tile_y);
  return cudaGetLastError();
}

}  // namespace nemo
