// Device code of the fused NEMOLite2D step shared by the single-grid kernel
// (nemo_fused.cu) and the ensemble kernel (nemo_ensemble.cu): one warp
// advances a strip of 30 T columns over a block of rows.  See nemo_fused.cu
// for the design and the exactness argument.
#pragma once

#include "nemo_internal.h"

namespace nemo {
namespace stepdev {


constexpr unsigned FULL = 0xffffffffu;
constexpr int COLS_PER_WARP = 30;

struct Cell {
  double s, u, v, ht, hu, hv;
};

__device__ __forceinline__ void load_cell(Cell& x, const FusedArgs& A, long o) {
  x.s = __ldg(A.sshn + o);
  x.u = __ldg(A.un + o);
  x.v = __ldg(A.vn + o);
  x.ht = __ldg(A.ht + o);
  x.hu = __ldg(A.hu + o);
  x.hv = __ldg(A.hv + o);
}

__device__ __forceinline__ double dn(double x) { return __shfl_down_sync(FULL, x, 1); }
__device__ __forceinline__ double up(double x) { return __shfl_up_sync(FULL, x, 1); }

// Quotients of the fused step.  The strict (-fmad=false) build forms every
// quotient correctly rounded, as the reference's division does.  The default
// build, which the reference's tolerance (1e-12 relative max-norm) governs,
// relaxes the quotients whose rounding errors average out over the steps:
// qdiv_k forms a/b by a grid constant as a * RN(1/b) (one rounding more, two
// FP64 operations fewer), and no state row needs the range check.  The
// divisions that scale the new velocities every step (by the depth and by
// the friction factor) stay rounded: a fixed divisor's RN(1/b) errs the same
// way at every step, and that bias accumulated to 1.4e-12 over 2000 steps of
// the 128^2 case when those too took the one-multiply form (1.3e-14 without).
// The same reasoning lets the default build fold products of grid constants
// (0.5*x*e2t as x*(0.5*e2t), rdt*(...)/e12u as (...)*(rdt/e12u), the grid
// spacings of the viscous gradients into the viscosity coefficients, and
// the Coriolis and pressure-gradient coefficients; kFold below) and pick the
// upwind value with a plain select.  Carried face values then hold the
// folded (scaled) forms, so the IEEE-division rows (SAFE) exist only in the
// strict build.
#ifdef NEMO_STRICT_BUILD
constexpr bool kRoundedQuotients = true;
#else
constexpr bool kRoundedQuotients = false;
#endif
constexpr bool kFold = !kRoundedQuotients;

// upwind() of the strict build, a select in the default build (the two differ
// only in the sign of a zero result and in propagating a NaN from the unused
// side)
__device__ __forceinline__ double upw(double w, double lo, double hi) {
  if (kFold) return sign_clear(w) ? lo : hi;
  return upwind(w, lo, hi);
}

// a/b given rb = RN(1/b): the corrected-reciprocal quotient (see div_const),
// exact whenever the quotient is zero or at least 2^-959 in magnitude.  The
// range is guaranteed per row instead of per quotient (row_tiny): a row whose
// three rows of state hold no nonzero value below 2^-300 in magnitude has no
// nonzero quotient below 2^-959.  Every quotient of a row is a sum of terms
// with at most two state factors (velocity x velocity in the advective
// fluxes) times grid constants and depths (depth >= hmin > 0); a nonzero
// difference of state values >= 2^-300 is >= 2^-352 (their ulp), a product
// of two such >= 2^-704 with ulp >= 2^-756, and a nonzero sum of such terms
// keeps that grain; the remaining factors are grid constants, rdt, visc,
// the Coriolis parameter and depths (at 1 km spacing, rdt 20 s: together
// within 2^-45 of 1), so every nonzero quotient is >= 2^-810, leaving over
// 140 binades for other grids and coefficients.  Rows outside that
// guarantee take the IEEE division (SAFE).  An infinite or NaN operand gives
// a non-finite quotient on both paths.
template <bool SAFE>
__device__ __forceinline__ double qdiv(double a, double b, double rb, bool& bad) {
  (void)bad;
  if (SAFE) return a / b;
  double q = __dmul_rn(a, rb);
  double r = fma(-q, b, a);
  return -fma(-r, rb, -q);
}

// a/b for a grid-constant divisor b: rounded in the strict build, a * RN(1/b)
// in the default build.
template <bool SAFE>
__device__ __forceinline__ double qdiv_k(double a, double b, double rb, bool& bad) {
  if (!SAFE && !kRoundedQuotients) return a * rb;
  return qdiv<SAFE>(a, b, rb, bad);
}

// a/cfric: rounded in the strict build; in the default build from the two-part
// reciprocal, a * (r_cfric + r_cfric_lo) with one rounding, which is the
// rounded quotient except within about 2^-50 ulp of a rounding boundary (two
// FP64 operations instead of three).
template <bool SAFE>
__device__ __forceinline__ double qdiv_fric(double a, const Consts& C, bool& bad) {
  if (!SAFE && !kRoundedQuotients) return fma(a, C.r_cfric, a * C.r_cfric_lo);
  return qdiv<SAFE>(a, C.cfric, C.r_cfric, bad);
}

// Reciprocal depth for the corrected depth quotients of the ring strips:
// RN(1/b) (recip_nr, checked cell by cell at setup) in the strict build; one
// Newton step in the default build, where the quotient's residual step turns
// its 2^-46 error into a quotient that is still the rounded one except within
// about 2^-39 ulp of a rounding boundary.
__device__ __forceinline__ double recip_depth(double b) { return kFold ? recip_nr1(b) : recip_nr(b); }

// Nonzero with |x| < 2^-300 (biased exponent below 723).
__device__ __forceinline__ bool tiny(double x) {
  const unsigned hi2 = (unsigned)__double2hiint(x) << 1;
  const unsigned lo = (unsigned)__double2loint(x);
  return (hi2 < (723u << 21)) & ((hi2 | lo) != 0u);
}
// Only the rounded quotients need the range guarantee.
__device__ __forceinline__ bool row_tiny(const Cell& x) {
  return kRoundedQuotients && (tiny(x.s) | tiny(x.u) | tiny(x.v));
}
// Warp-wide: does any lane's row need the IEEE division form?
__device__ __forceinline__ unsigned any_tiny(const Cell& x) {
  return kRoundedQuotients && __any_sync(FULL, row_tiny(x)) ? 1u : 0u;
}

__device__ __forceinline__ double interp_u(const Consts& C, int c, int jpi, double s0, double s1,
                                          bool safe, bool& bad) {
  if (c == 0) return s1;
  if (c == jpi) return s0;
  if (kFold && !safe) return (s0 + s1) * C.k_su;
  double a = 0.5 * (C.e12t * s0 + C.e12t * s1);
  return safe ? qdiv<true>(a, C.e12u, C.r_e12u, bad) : qdiv_k<false>(a, C.e12u, C.r_e12u, bad);
}

__device__ __forceinline__ double interp_v(const Consts& C, int jj, int jpj, double s0, double s1,
                                          bool safe, bool& bad) {
  if (jj == jpj) return s0;
  if (kFold && !safe) return (s0 + s1) * C.k_sv;
  double a = 0.5 * (C.e12t * s0 + C.e12t * s1);
  return safe ? qdiv<true>(a, C.e12v, C.r_e12v, bad) : qdiv_k<false>(a, C.e12v, C.r_e12v, bad);
}

// Values carried from row j-1 to row j for one column.
struct Carry {
  double su, Hu;       // sshn_u and hu+sshn_u at (c, j)
  double s_e;          // sshn(c+1, j)
  double Fuy_s;        // upwind flux through the south face of u(c,j)
  double dudy_s;       // dudy_s of u(c,j)
  double vnc_s;        // v_sc of u(c,j)
  double Fvy_s;        // upwind flux through the south face of v(c,j)
  double Dvy_s;        // dvdy_s of v(c,j)
  double cf_s;         // (sshn_v + hv)*vn at (c, j-1)
};

struct RowOut {
  double ssha, ua, va, sv;
  Carry next;
};

// One row of the step for one lane: outputs at (c, j) and the carry to j+1.
// EDGE = false is the interior form: the caller guarantees that no lane of
// the warp sits on column 0, 1 or jpi and that j is neither 1 nor jpj, so
// every mask of the reference geometry is inactive.
// rhu, rhv: RN(1/hu), RN(1/hv) at (c, j).
template <bool SAFE, bool EDGE>
__device__ __forceinline__ void row(const Consts& C, int c, int j, int jpi, int jpj, double tide,
                                    const Cell& cur, const Cell& nx, const Carry& k, double rhu,
                                    double rhv, RowOut& o, bool& bad) {
  const bool south = EDGE && (j == 1), north = EDGE && (j == jpj);
  const bool west0 = EDGE && (c == 0), west1 = EDGE && (c == 1), east = EDGE && (c == jpi);
  // sshn_v at (c, j), sshn_u at (c, j+1)
  const double sv = EDGE ? interp_v(C, j, jpj, cur.s, nx.s, SAFE, bad)
                         : interp_v(C, 0, 1, cur.s, nx.s, SAFE, bad);
  const double Hv = cur.hv + sv;
  const double s_e_n = dn(nx.s);
  const double su_n = EDGE ? interp_u(C, c, jpi, nx.s, s_e_n, SAFE, bad)
                           : interp_u(C, 1, 0, nx.s, s_e_n, SAFE, bad);
  const double Hu_n = nx.hu + su_n;

  // x-face of the u equation at T(c,j), between u(c-1,j) and u(c,j)
  const double u_w = up(cur.u);
  const double uw = kFold ? (cur.u + u_w) * C.h_e2t : 0.5 * (cur.u + u_w) * C.e2t;
  const double dep = cur.ht + cur.s;
  const double Fx = upw(uw, u_w, cur.u) * uw * dep;
  const double Dx = kFold ? (cur.u - u_w) * dep : qdiv_k<SAFE>(cur.u - u_w, C.e1t, C.r_e1t, bad) * dep;

  // corner (c,j): east face of v(c,j), north face of u(c,j)
  const double uec = kFold ? cur.u + nx.u : 0.5 * (cur.u + nx.u);  // folded: twice
  const double ue = kFold ? uec * C.e_2dy : 0.5 * uec * C.two_dy;    // folded: half
  const double Sn = (k.Hu + nx.hu) + su_n;
  const double v_e = dn(cur.v);
  const double uuv = west0 ? upwind_hi_only(ue, v_e)
                          : east ? upwind_lo_only(ue, cur.v) : upw(ue, cur.v, v_e);
  const double Fvx = kFold ? uuv * ue * Sn : uuv * ue * (0.5 * Sn);
  const double Gx = kFold ? v_e - cur.v : qdiv_k<SAFE>(v_e - cur.v, C.two_dx, C.r_2dx, bad);
  const double vnc = kFold ? cur.v + v_e : 0.5 * (cur.v + v_e);  // folded: twice
  const double vn_ = kFold ? vnc * C.e_2dx : 0.5 * vnc * C.two_dx;  // folded: half
  const double Re = (Hv + dn(cur.hv)) + dn(sv);
  const double uuu = north ? upwind_lo_only(vn_, cur.u) : upw(vn_, cur.u, nx.u);
  const double Fuy = kFold ? uuu * vn_ * Re : uuu * vn_ * (0.5 * Re);
  const double Gy = kFold ? nx.u - cur.u : qdiv_k<SAFE>(nx.u - cur.u, C.two_dy, C.r_2dy, bad);

  // y-face of the v equation at T(c,j+1), between v(c,j) and v(c,j+1)
  const double vs = kFold ? (nx.v + cur.v) * C.h_e1t : 0.5 * (nx.v + cur.v) * C.e1t;
  const double depn = nx.ht + nx.s;
  const double Fvy_n = upw(vs, cur.v, nx.v) * vs * depn;
  const double Dvy_n = kFold ? (nx.v - cur.v) * depn : qdiv_k<SAFE>(nx.v - cur.v, C.e2t, C.r_e2t, bad) * depn;

  // continuity (:399-403), clamped SSH row (:631-644)
  const double r1 = k.Hu * cur.u;
  const double r2 = up(r1);
  const double r3 = Hv * cur.v;
  const double ssh = kFold ? cur.s + (r2 - r1 + k.cf_s - r3) * C.k_ssh
                                      : cur.s + qdiv_k<SAFE>((r2 - r1 + k.cf_s - r3) * C.rdt, C.e12t, C.r_e12t, bad);
  o.ssha = south ? tide : ssh;

  // u equation (:439-514); u(jpi,j) is the east wall (:650)
  {
    const double Fx_e = dn(Fx);
    const double Dx_e = dn(Dx);
    const double adv = Fx - Fx_e + k.Fuy_s - Fuy;
    const double dudy_n = north ? 0.0 : Gy * Sn;
    const double dudy_s = south ? 0.0 : k.dudy_s;
    double num;
    if (kFold) {
      const double vis = (Dx_e - Dx) * C.vis_u1 + (dudy_n - dudy_s) * C.vis_u2;
      const double corhpg = k.Hu * ((k.vnc_s + vnc) * C.cor_u + (k.s_e - cur.s) * C.hpg_u);
      num = cur.u * k.Hu + (adv + vis + corhpg) * C.k_u;
    } else {
      double vis = (Dx_e - Dx) * C.e2u + (dudy_n - dudy_s) * C.e1u * 0.5;
      vis = C.visc * vis;
      const double cor = 0.5 * (C.fcor * (k.vnc_s + vnc)) * C.e12u * k.Hu;
      const double hpg = -(C.g * k.Hu * C.e2u * (k.s_e - cur.s));
      num = cur.u * k.Hu + qdiv_k<SAFE>(C.rdt * (adv + vis + cor + hpg), C.e12u, C.r_e12u, bad);
    }
    const double q = qdiv<SAFE>(num, kFold ? cur.hu : cur.hu + 0.0, rhu, bad);
    o.ua = east ? 0.0 : qdiv_fric<SAFE>(q, C, bad);
  }
  // v equation (:527-606); v(c,jpj) is the north wall (:658)
  {
    const double Fvx_w = up(Fvx);
    const double Gx_w = up(Gx);
    const double hv_w = up(cur.hv);
    const double sv_w = up(sv);
    const double uec_w = up(uec);
    const double adv = Fvx_w - Fvx + k.Fvy_s - Fvy_n;
    const double dvdx_e = east ? 0.0 : Gx * Re;
    const double dvdx_w = west1 ? 0.0 : Gx_w * ((Hv + hv_w) + sv_w);
    double num;
    if (kFold) {
      const double vis = (Dvy_n - k.Dvy_s) * C.vis_v1 + (dvdx_e - dvdx_w) * C.vis_v2;
      const double corhpg = Hv * ((uec + uec_w) * C.cor_v + (nx.s - cur.s) * C.hpg_v);
      num = cur.v * Hv + (adv + vis + corhpg) * C.k_v;
    } else {
      double vis = (Dvy_n - k.Dvy_s) * C.e1v + (dvdx_e - dvdx_w) * C.e2v * 0.5;
      vis = C.visc * vis;
      const double cor = -(0.5 * (C.fcor * (uec + uec_w)) * C.e12v * Hv);
      const double hpg = -(C.g * Hv * C.e1v * (nx.s - cur.s));
      num = cur.v * Hv + qdiv_k<SAFE>(C.rdt * (adv + vis + cor + hpg), C.e12v, C.r_e12v, bad);
    }
    const double q = qdiv<SAFE>(num, kFold ? cur.hv : cur.hv + 0.0, rhv, bad);
    o.va = north ? 0.0 : qdiv_fric<SAFE>(q, C, bad);
  }
  o.sv = sv;
  // carry to row j+1
  o.next.su = su_n;
  o.next.Hu = Hu_n;
  o.next.s_e = s_e_n;
  o.next.Fuy_s = Fuy;
  o.next.dudy_s = Gy * ((Hu_n + cur.hu) + k.su);  // dudy_s of u(c,j+1)
  o.next.vnc_s = vnc;
  o.next.Fvy_s = Fvy_n;
  o.next.Dvy_s = Dvy_n;
  o.next.cf_s = r3;
}

// Carried values at row J0 from rows J0-1 (p) and J0 (q).
template <bool SAFE>
__device__ __forceinline__ void prologue(const Consts& C, int c, int J0, int jpi, int jpj,
                                         double sv_p_stored, const Cell& p, const Cell& q,
                                         Carry& k, double& sv_p, bool& bad) {
  k.s_e = dn(q.s);
  k.su = interp_u(C, c, jpi, q.s, k.s_e, SAFE, bad);
  k.Hu = q.hu + k.su;
  sv_p = (J0 == 1) ? sv_p_stored : interp_v(C, J0 - 1, jpj, p.s, q.s, SAFE, bad);
  const double Hv_p = p.hv + sv_p;
  // corner (c, J0-1): south face of u(c, J0)
  const double vnc = kFold ? p.v + dn(p.v) : 0.5 * (p.v + dn(p.v));
  const double vn_ = kFold ? vnc * C.e_2dx : 0.5 * vnc * C.two_dx;
  const double dep = kFold ? (Hv_p + dn(p.hv)) + dn(sv_p) : 0.5 * ((Hv_p + dn(p.hv)) + dn(sv_p));
  const double uu = (J0 == 1) ? upwind_hi_only(vn_, q.u) : upw(vn_, p.u, q.u);
  k.Fuy_s = uu * vn_ * dep;
  k.vnc_s = vnc;
  const double s_e_p = dn(p.s);
  if (J0 == 1) {
    k.dudy_s = 0.0;
  } else {
    const double su_p = interp_u(C, c, jpi, p.s, s_e_p, SAFE, bad);
    const double gy = kFold ? q.u - p.u : qdiv_k<SAFE>(q.u - p.u, C.two_dy, C.r_2dy, bad);
    k.dudy_s = gy * ((k.Hu + p.hu) + su_p);
  }
  // T(c, J0): south face of v(c, J0)
  const double vs = kFold ? (q.v + p.v) * C.h_e1t : 0.5 * (q.v + p.v) * C.e1t;
  const double depc = q.ht + q.s;
  k.Fvy_s = upw(vs, p.v, q.v) * vs * depc;
  k.Dvy_s = (kFold ? q.v - p.v : qdiv_k<SAFE>(q.v - p.v, C.e2t, C.r_e2t, bad)) * depc;
  k.cf_s = Hv_p * p.v;
}

// One warp's strip: columns c0 .. c0+29 (lanes 1..30), rows J0 .. J1 of the
// grid described by L, inputs/outputs in A.  All 32 lanes of the warp must
// call it together.  PF = 1 prefetches row j+2 into registers (run_strip_ring
// below stages rows through shared memory instead).
template <int PF>
__device__ __forceinline__ void run_strip(const Layout& L, const Consts& C, const FusedArgs& A,
                                          int c0, int J0, int J1, int lane) {
  const int jpi = L.jpi, jpj = L.jpj;
  const int c = c0 + lane - 1;
  const int cl = min(c, jpi + 1);  // lanes beyond the halo column read column jpi+1
  const bool store = (lane >= 1) && (lane <= COLS_PER_WARP) && (c <= jpi);

  // lanes span columns c0-1 .. c0+30; the interior row form applies when
  // none of them is 0, 1 or jpi
  const bool edge_warp = (c0 - 1 <= 1) || (c0 + COLS_PER_WARP >= jpi);

  Cell p, cur, nx;
  load_cell(p, A, L.idx(cl, J0 - 1));
  load_cell(cur, A, L.idx(cl, J0));
  const double sv_stored = (J0 == 1) ? __ldg(A.sshv0 + L.idx(cl, 0)) : 0.0;
  Carry k;
  double sv0;
  // warp-wide tiny-value flags: bit 0 row j+1 (set as it arrives), bit 1
  // row j, bit 2 row j-1; row j takes the IEEE form while any is set
  unsigned hist = (any_tiny(p) << 1) | any_tiny(cur);
  {
    bool bad = false;
    if (kRoundedQuotients && hist) prologue<true>(C, c, J0, jpi, jpj, sv_stored, p, cur, k, sv0, bad);
    else prologue<false>(C, c, J0, jpi, jpj, sv_stored, p, cur, k, sv0, bad);
  }
  if (PF) load_cell(nx, A, L.idx(cl, J0 + 1));

  const long pitch = L.pitch;
  long o_ld = L.idx(cl, J0 + 1 + PF);  // next row to load
  const long o_last = L.idx(cl, jpj + 1);
  long o_st = L.idx(c, J0);
  long o_cur = L.idx(cl, J0);
#pragma unroll 1
  for (int j = J0; j <= J1; ++j) {
    Cell pf;
    if (PF) {
      load_cell(pf, A, o_ld < o_last ? o_ld : o_last);  // row j+2 (clamped to jpj+1)
    } else {
      load_cell(nx, A, o_ld);  // row j+1 <= jpj+1
    }
    o_ld += pitch;
    // reciprocal depths of this row, loaded where they are used
    const double rhu = __ldg(A.rhu + o_cur);
    const double rhv = __ldg(A.rhv + o_cur);
    o_cur += pitch;

    RowOut o;
    bool bad = false;
    hist = ((hist << 1) | any_tiny(nx)) & 7u;
    if (kRoundedQuotients && hist) {
      row<true, true>(C, c, j, jpi, jpj, A.tide, cur, nx, k, rhu, rhv, o, bad);
    } else if (edge_warp || j == 1 || j == jpj) {
      row<false, true>(C, c, j, jpi, jpj, A.tide, cur, nx, k, rhu, rhv, o, bad);
    } else {
      row<false, false>(C, c, j, jpi, jpj, A.tide, cur, nx, k, rhu, rhv, o, bad);
    }
    if (store) {
      A.ssha[o_st] = o.ssha;
      A.ua[o_st] = o.ua;
      A.va[o_st] = o.va;
      if (edge_warp && c == 1) A.ua[o_st - 1] = 0.0;  // u(0,j), west wall (:650)
      if (j == 1) {
        // Flather open boundary (:684-695): v(c,0) = v(c,1) + sqrt(g/hv(c,0))*(sshn_v(c,0) - sshn_v(c,1))
        const double hv0 = __ldg(A.hv + o_st - pitch), sv0r = __ldg(A.sshv0 + o_st - pitch);
        A.va[o_st - pitch] = o.va + sqrt(kG / hv0) * (sv0r - o.sv);
      }
    }
    o_st += pitch;
    k = o.next;
    cur = nx;
    if (PF) nx = pf;
  }
}

// ---- shared-memory ring variant -------------------------------------------
// Rows are staged by cp.async into a per-warp ring of ring_slots<NR>() rows
// x 6 or 8 fields x 32 lanes (each lane copies and reads only its own
// column), ring_slots<NR>() - 1 rows ahead of their use, so DRAM latency is
// hidden without holding prefetched rows in registers.  Row r sits in slot
// r % slots; the copy of row j+ahead reuses the slot of row j-1, read into
// registers two iterations earlier.  NR: the reciprocal depths are formed in
// the kernel, so a row holds 6 fields instead of 8.
#ifndef NEMO_RING_NR
#define NEMO_RING_NR 4
#endif
template <bool NR>
__host__ __device__ constexpr int ring_slots() { return NR ? NEMO_RING_NR : 4; }
template <bool NR>
__host__ __device__ constexpr int ring_row() { return (NR ? 6 : 8) * 32; }  // doubles per staged row
template <bool NR>
__host__ __device__ constexpr int ring_doubles() { return ring_slots<NR>() * ring_row<NR>(); }

__device__ __forceinline__ void cp_async8(double* dst, const double* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// Wait until at most N of this thread's copy groups are pending.
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// NR: the reciprocal depths are formed in the kernel (recip_nr), not staged.
template <bool NR>
__device__ __forceinline__ void ring_issue(double* slot, const FusedArgs& A, long o) {
  cp_async8(slot + 0 * 32, A.sshn + o);
  cp_async8(slot + 1 * 32, A.un + o);
  cp_async8(slot + 2 * 32, A.vn + o);
  cp_async8(slot + 3 * 32, A.ht + o);
  cp_async8(slot + 4 * 32, A.hu + o);
  cp_async8(slot + 5 * 32, A.hv + o);
  if (!NR) {
    cp_async8(slot + 6 * 32, A.rhu + o);
    cp_async8(slot + 7 * 32, A.rhv + o);
  }
  cp_commit();
}

__device__ __forceinline__ void ring_cell(Cell& x, const double* slot) {
  x.s = slot[0 * 32];
  x.u = slot[1 * 32];
  x.v = slot[2 * 32];
  x.ht = slot[3 * 32];
  x.hu = slot[4 * 32];
  x.hv = slot[5 * 32];
}

// run_strip with rows staged through `ring` (this warp's ring_doubles<NR>(), in
// shared memory), its row loop unrolled UNROLL times.  NR = true forms RN(1/hu), RN(1/hv) with recip_nr instead
// of reading the stored fields: valid only for depths that launch_recip
// found to give exactly the stored values (16 fewer bytes per cell-step).
template <bool NR, int UNROLL>
__device__ __forceinline__ void run_strip_ring(const Layout& L, const Consts& C, const FusedArgs& A,
                                               int c0, int J0, int J1, int lane, double* ring) {
  const int jpi = L.jpi, jpj = L.jpj;
  const int c = c0 + lane - 1;
  const int cl = min(c, jpi + 1);
  const bool store = (lane >= 1) && (lane <= COLS_PER_WARP) && (c <= jpi);
  const bool edge_warp = (c0 - 1 <= 1) || (c0 + COLS_PER_WARP >= jpi);
  double* my = ring + lane;  // this lane's column of every ring row
  constexpr int RING = ring_slots<NR>(), AHEAD = RING - 1, RS = ring_row<NR>();

  const long pitch = L.pitch;
  // rows J0+1 .. J0+AHEAD-1 into the ring, and row J0 when its stored
  // reciprocal depths are read from there (rows J0-1 and J0 are loaded
  // directly below).  Rows past J1+1, which no iteration reads, are not
  // copied: their copy group stays empty, so the group counts of the waits
  // hold.
  const int r_stop = J1 + 1;
#pragma unroll
  for (int r = NR ? 1 : 0; r < AHEAD; ++r) {
    if (J0 + r <= r_stop)
      ring_issue<NR>(my + ((J0 + r) % RING) * RS, A, L.idx(cl, J0 + r));
    else
      cp_commit();
  }

  Cell p, cur, nx;
  load_cell(p, A, L.idx(cl, J0 - 1));
  load_cell(cur, A, L.idx(cl, J0));
  const double sv_stored = (J0 == 1) ? __ldg(A.sshv0 + L.idx(cl, 0)) : 0.0;
  Carry k;
  double sv0;
  unsigned hist = (any_tiny(p) << 1) | any_tiny(cur);
  {
    bool bad = false;
    if (kRoundedQuotients && hist) prologue<true>(C, c, J0, jpi, jpj, sv_stored, p, cur, k, sv0, bad);
    else prologue<false>(C, c, J0, jpi, jpj, sv_stored, p, cur, k, sv0, bad);
  }
  long o_ld = L.idx(cl, J0 + AHEAD);
  long o_st = L.idx(c, J0);
  int slot_j = J0 % RING;
// UNROLL = 2 keeps two rows in flight (the second row's independent work
// fills FP64 latency) where registers allow it without spills
#pragma unroll UNROLL
  for (int j = J0; j <= J1; ++j) {
    const int slot_n = slot_j == RING - 1 ? 0 : slot_j + 1;  // row j+1
    const int slot_f = slot_j == 0 ? RING - 1 : slot_j - 1;  // row j+AHEAD (was row j-1)
    if (j + AHEAD <= r_stop)
      ring_issue<NR>(my + slot_f * RS, A, o_ld);
    else
      cp_commit();
    o_ld += pitch;
    cp_wait<AHEAD - 1>();  // rows <= j+1 have landed
    ring_cell(nx, my + slot_n * RS);
    const double rhu = NR ? recip_depth(cur.hu + 0.0) : my[slot_j * RS + 6 * 32];
    const double rhv = NR ? recip_depth(cur.hv + 0.0) : my[slot_j * RS + 7 * 32];

    RowOut o;
    bool bad = false;
    hist = ((hist << 1) | any_tiny(nx)) & 7u;
    if (kRoundedQuotients && hist) {
      row<true, true>(C, c, j, jpi, jpj, A.tide, cur, nx, k, rhu, rhv, o, bad);
    } else if (edge_warp || j == 1 || j == jpj) {
      row<false, true>(C, c, j, jpi, jpj, A.tide, cur, nx, k, rhu, rhv, o, bad);
    } else {
      row<false, false>(C, c, j, jpi, jpj, A.tide, cur, nx, k, rhu, rhv, o, bad);
    }
    if (store) {
      A.ssha[o_st] = o.ssha;
      A.ua[o_st] = o.ua;
      A.va[o_st] = o.va;
      if (edge_warp && c == 1) A.ua[o_st - 1] = 0.0;
      if (j == 1) {  // Flather open boundary, as in run_strip
        const double hv0 = __ldg(A.hv + o_st - pitch), sv0r = __ldg(A.sshv0 + o_st - pitch);
        A.va[o_st - pitch] = o.va + sqrt(kG / hv0) * (sv0r - o.sv);
      }
    }
    o_st += pitch;
    k = o.next;
    cur = nx;
    slot_j = slot_n;
  }
  asm volatile("cp.async.wait_all;" ::: "memory");  // no copy may outlive the strip's ring use
}

}  // namespace stepdev
}  // namespace nemo
