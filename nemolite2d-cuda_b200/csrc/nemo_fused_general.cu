// Fused step for general grids (nemo_set_grid): masks with open water on any
// border and islands, per-point scale factors, latitudes and depths
// (original/nemolite2d.f90:390-769 with the grid arrays of :145-281).
//
// Two launches per step instead of the routine sequence's twelve:
//
//  k_fused_general -- one warp owns a strip of 30 T columns and marches north
//    over a block of rows, as the uniform fused kernel does (lane l holds
//    column c0+l-1; lanes 0 and 31 are halo lanes; columns c-1 / c+1 come
//    from warp shuffles, row j-1 from values carried in registers).  Per row
//    it forms continuity (:397-405) and the clamped SSH (:631-644) at T(c,j),
//    the u equation (:431-517) at u(c,j) and the v equation (:520-609) at
//    v(c,j) with every mask test of the reference read from pt, then the
//    solid walls (:648-660).  Points that no routine of the step writes (a u
//    point between two open cells; a v point whose east neighbour is open,
//    which the reference's test of pt(ji+1,jj) at :523 skips) keep their
//    value, which after a complete step is the current velocity.
//    sshn_u / sshn_v are derived from sshn on the fly with the branches of
//    `next` (:736-764); where that loop leaves them alone (both sides land or
//    open) the stored value is read, which nothing changes.
//  k_flather_general -- the Flather conditions (:669-695).  The reference
//    sweeps them in place; an open u point reads its neighbour before that
//    neighbour's own Flather update when the neighbour lies east of it, and
//    after it when west.  Only a one-cell channel between two open cells
//    chains two updates (an open point west of water, then that water point
//    with open water east of it), so the host lists the Flather points as
//    independent chains of at most two and one thread runs each chain in the
//    sweep's order.  The same holds for v along jj.
//
// Every quantity the reference evaluates twice (a face flux shared by two
// velocity points, dudx, dvdy, the velocity gradients across faces) is formed
// once where the two expression trees agree up to commutation of + and *;
// where the reference masks the two uses differently (the slip-wall forms)
// each use has its own value.  e12t, e12u, e12v are formed in the kernel as
// the products the reference stores (:263-279), zero outside their ranges.
// Quotients: IEEE division in the -fmad=false build (bit-exact with the
// oracle).  The default build, which the reference's 1e-12 tolerance governs,
// multiplies by Newton reciprocals of the scale factors (the grid-constant
// sites of the uniform kernel's default build), and keeps the two quotients
// that scale the new velocities every step rounded as that build does: the
// depth by the corrected quotient, the friction factor by the two-part
// reciprocal.
#include "nemo_step_dev.cuh"

namespace nemo {
namespace {
using stepdev::COLS_PER_WARP;
using stepdev::FULL;
using stepdev::dn;
using stepdev::up;
using stepdev::upw;

using stepdev::kRoundedQuotients;

// The default build's reciprocal of a scale factor or depth: the FP64
// approximate reciprocal (one special-function operation, no conversions)
// refined by two Newton-Raphson steps, y <- y + y(1 - b y), each of which
// squares the relative error; the result is within a few units in the last
// place.  b = 0 gives NaN, in lanes whose results are discarded.
__device__ __forceinline__ double grecip(double b) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(b));
  y = fma(y, fma(-b, y, 1.0), y);
  return fma(y, fma(-b, y, 1.0), y);
}
// a / b: the rounded quotient in the -fmad=false build; a * rb in the default
// build, rb a reciprocal of b (grecip(b), or for a factor b of a product
// b*d, d * grecip(b*d)), which the strict build never forms.
__device__ __forceinline__ double qr(double a, double b, double rb) {
  if (kRoundedQuotients) return a / b;
  return a * rb;
}
// a / b for a scale-factor divisor.
__device__ __forceinline__ double qm(double a, double b) { return qr(a, b, grecip(b)); }
// a / h for a static depth h: in the default build the quotient corrected by
// one residual step, q + (a - q h) r, which is the rounded quotient except
// within a tiny fraction of an ulp of a rounding boundary.
__device__ __forceinline__ double qh(double a, double h) {
  if (kRoundedQuotients) return a / h;
  bool bad = false;
  return stepdev::qdiv<false>(a, h, grecip(h), bad);
}
// a / cfric
__device__ __forceinline__ double qf(double a, const Consts& C) {
  if (kRoundedQuotients) return a / C.cfric;
  bool bad = false;
  return stepdev::qdiv_fric<false>(a, C, bad);
}

__device__ __forceinline__ int dni(int x) { return __shfl_down_sync(FULL, x, 1); }
__device__ __forceinline__ int upi(int x) { return __shfl_up_sync(FULL, x, 1); }

// Fields of row j+1 that row j needs.
struct GNext {
  double s, u, v, ht, hu, e1t, e2t, e1u, e2u;
  int pt;
};
// Fields of row j used only at row j.
struct GOwn {
  double hv, e1v, e2v, fcu, fcv;
};

__device__ __forceinline__ void load_next(GNext& x, const GenArgs& A, long o) {
  x.s = __ldg(A.sshn + o);
  x.u = __ldg(A.un + o);
  x.v = __ldg(A.vn + o);
  x.ht = __ldg(A.ht + o);
  x.hu = __ldg(A.hu + o);
  x.e1t = __ldg(A.g.e1t + o);
  x.e2t = __ldg(A.g.e2t + o);
  x.e1u = __ldg(A.g.e1u + o);
  x.e2u = __ldg(A.g.e2u + o);
  x.pt = A.g.pt[o];
}
__device__ __forceinline__ void load_own(GOwn& x, const GenArgs& A, long o) {
  x.hv = __ldg(A.hv + o);
  x.e1v = __ldg(A.g.e1v + o);
  x.e2v = __ldg(A.g.e2v + o);
  x.fcu = __ldg(A.g.fcu + o);
  x.fcv = __ldg(A.g.fcv + o);
}

// e12t as the reference stores it: e1t*e2t over (1:jpi, 1:jpj), zero elsewhere.
__device__ __forceinline__ double e12t_at(const GNext& x, int c, int r, int jpi, int jpj) {
  return (c >= 1 && c <= jpi && r >= 1 && r <= jpj) ? x.e1t * x.e2t : 0.0;
}

// sshn_u at (c, r) after `next` (:736-749); every lane of the warp calls it
// (shuffles).  e12u is e1u*e2u of (c, r), inside its range (0:jpi, 1:jpj)
// wherever the branch that uses it is taken.
// ru: the default build's reciprocal of e1u*e2u at (c, r).
__device__ __forceinline__ double sshn_u_at(const GNext& x, int c, int r, int jpi, int jpj,
                                            const double* stored, long o, double ru) {
  const int a = x.pt, b = dni(x.pt);
  const double s1 = dn(x.s);
  const double t0 = e12t_at(x, c, r, jpi, jpj);
  const double t1 = dn(t0);
  const double avg = qr(0.5 * (t0 * x.s + t1 * s1), x.e1u * x.e2u, ru);
  const double st = (a + b > 0) ? 0.0 : __ldg(stored + o);
  return (a + b > 0) ? ((a * b > 0) ? avg : ((a <= 0) ? s1 : x.s)) : st;
}

// sshn_v at (c, j) after `next` (:751-764) from rows j (x, own) and j+1 (y);
// rv: the default build's reciprocal of e1v*e2v at (c, j).
__device__ __forceinline__ double sshn_v_at(const GNext& x, const GOwn& w, const GNext& y, int c, int j,
                                            int jpi, int jpj, const double* stored, long o, double rv) {
  const int a = x.pt, b = y.pt;
  const double t0 = e12t_at(x, c, j, jpi, jpj), t1 = e12t_at(y, c, j + 1, jpi, jpj);
  const double avg = qr(0.5 * (t0 * x.s + t1 * y.s), w.e1v * w.e2v, rv);
  const double st = (a + b > 0) ? 0.0 : __ldg(stored + o);
  return (a + b > 0) ? ((a * b > 0) ? avg : ((a <= 0) ? y.s : x.s)) : st;
}

// Values carried from row j-1 to row j for one column.
struct GCarry {
  double su;      // sshn_u(c, j)
  double cf_s;    // (sshn_v + hv) * vn at (c, j-1)
  double Fuy_s;   // south-face flux of u(c, j), masked as u(c, j) sees it
  double vnc_s;   // v_sc of u(c, j)
  double dudy_s;  // dudy_s of u(c, j), masked as u(c, j) sees it
  double Fvy_s;   // south-face flux of v(c, j)
  double Dvy_s;   // dvdy_s of v(c, j)
  int pt_s;       // pt(c, j-1)
};

// Rows staged through a per-warp ring in shared memory: RG slots, each row
// issued RG-1 rows ahead of its use by cp.async, every lane copying its own
// column of each field (8 bytes).  A slot holds the 14 fields of one row (the
// 9 of GNext and the 5 of GOwn) field-major, 32 doubles per field with lane
// l's column at l; the int8 mask is loaded one row ahead into a register.
// RG = 0: every row is loaded at the top of the iteration that needs it.
constexpr int GF = 14;

__device__ __forceinline__ void ring_issue_g(double* my, const GenArgs& A, long o) {
  using stepdev::cp_async8;
  cp_async8(my + 0 * 32, A.sshn + o);
  cp_async8(my + 1 * 32, A.un + o);
  cp_async8(my + 2 * 32, A.vn + o);
  cp_async8(my + 3 * 32, A.ht + o);
  cp_async8(my + 4 * 32, A.hu + o);
  cp_async8(my + 5 * 32, A.g.e1t + o);
  cp_async8(my + 6 * 32, A.g.e2t + o);
  cp_async8(my + 7 * 32, A.g.e1u + o);
  cp_async8(my + 8 * 32, A.g.e2u + o);
  cp_async8(my + 9 * 32, A.hv + o);
  cp_async8(my + 10 * 32, A.g.e1v + o);
  cp_async8(my + 11 * 32, A.g.e2v + o);
  cp_async8(my + 12 * 32, A.g.fcu + o);
  cp_async8(my + 13 * 32, A.g.fcv + o);
  stepdev::cp_commit();
}
__device__ __forceinline__ void ring_next(GNext& x, const double* my, int pt) {
  x.s = my[0 * 32];
  x.u = my[1 * 32];
  x.v = my[2 * 32];
  x.ht = my[3 * 32];
  x.hu = my[4 * 32];
  x.e1t = my[5 * 32];
  x.e2t = my[6 * 32];
  x.e1u = my[7 * 32];
  x.e2u = my[8 * 32];
  x.pt = pt;
}
__device__ __forceinline__ void ring_own(GOwn& w, const double* my) {
  w.hv = my[9 * 32];
  w.e1v = my[10 * 32];
  w.e2v = my[11 * 32];
  w.fcu = my[12 * 32];
  w.fcv = my[13 * 32];
}
__device__ __forceinline__ int ring_step(int s, int rg) { return s + 1 == rg ? 0 : s + 1; }

#ifndef NEMO_GEN_MINB
#define NEMO_GEN_MINB 8  // resident CTAs per SM the register budget is fitted to
#endif
template <int RG>
__global__ void __launch_bounds__(64, NEMO_GEN_MINB)
k_fused_general(Layout L, Consts C, GenArgs A, int tile_y) {
  constexpr int AHEAD = RG > 0 ? RG - 1 : 0;
  __shared__ double ring_all[RG > 0 ? 2 * RG * GF * 32 : 1];
  const int lane = threadIdx.x & 31;
  const int warp = (int)(blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5));
  const int c0 = 1 + COLS_PER_WARP * warp;
  if (c0 > L.jpi) return;  // whole warp idle
  const int J0 = 1 + (int)blockIdx.y * tile_y;
  if (J0 > L.jpj) return;
  const int J1 = min(J0 + tile_y - 1, L.jpj);
  const int jpi = L.jpi, jpj = L.jpj;
  const int c = c0 + lane - 1;
  const int cl = min(c, jpi + 1);  // lanes beyond the halo column read column jpi+1
  // T and v points: columns 1..jpi; u points also column 0 (lane 0 of the
  // first strip)
  const bool store = (lane >= 1) && (lane <= COLS_PER_WARP) && (c <= jpi);
  const bool store_u = store || (c == 0);
  const long pitch = L.pitch;

  // ---- the ring: rows J0 .. J1+1 (row J0-1 is loaded directly); row J0+i
  // goes to slot i mod RG ----
  double* my = ring_all + (threadIdx.x >> 5) * (RG > 0 ? RG * GF * 32 : 0) + lane;
  const int r_stop = J1 + 1;  // the last row any iteration reads
  if constexpr (RG > 0) {
#pragma unroll
    for (int r = 0; r < AHEAD; ++r) {
      if (J0 + r <= r_stop) ring_issue_g(my + r * GF * 32, A, L.idx(cl, J0 + r));
      else stepdev::cp_commit();
    }
  }

  // ---- prologue: rows J0-1 (p) and J0 (q) ----
  GNext p, cur;
  GOwn pw;
  load_next(p, A, L.idx(cl, J0 - 1));
  load_own(pw, A, L.idx(cl, J0 - 1));
  int pt1 = 0;  // RG > 0: the mask of the next row to take out of the ring
  if constexpr (RG > 0) {
    const int pt0 = A.g.pt[L.idx(cl, J0)];
    pt1 = A.g.pt[L.idx(cl, J0 + 1)];
    stepdev::cp_wait<AHEAD - 1>();  // row J0 has landed in slot 0
    ring_next(cur, my, pt0);
  } else {
    load_next(cur, A, L.idx(cl, J0));
  }
  GCarry k;
  {
    const double su_p = sshn_u_at(p, c, J0 - 1, jpi, jpj, A.su_st, L.idx(cl, J0 - 1), grecip(p.e1u * p.e2u));
    k.su = sshn_u_at(cur, c, J0, jpi, jpj, A.su_st, L.idx(cl, J0), grecip(cur.e1u * cur.e2u));
    const double sv_p = sshn_v_at(p, pw, cur, c, J0 - 1, jpi, jpj, A.sv_st, L.idx(cl, J0 - 1),
                                  grecip(pw.e1v * pw.e2v));
    k.cf_s = (sv_p + pw.hv) * p.v;
    // corner (c, J0-1): the south face of u(c, J0)
    const double vnc = 0.5 * (p.v + dn(p.v));
    const double vfl = 0.5 * vnc * (pw.e1v + dn(pw.e1v));
    const double depc = 0.5 * (pw.hv + sv_p + dn(pw.hv) + dn(sv_p));
    // every lane shuffles (a shuffle inside the short-circuit would leave out
    // the lanes whose own cell is land or open)
    const int ppt_e = dni(p.pt);
    const bool ms = p.pt <= 0 || ppt_e <= 0;  // pt(ji,jj-1), pt(ji+1,jj-1) of u(c, J0)
    k.Fuy_s = (ms ? upwind_hi_only(vfl, cur.u) : upw(vfl, p.u, cur.u)) * vfl * depc;
    k.vnc_s = vnc;
    k.dudy_s = ms ? 0.0 : qm(cur.u - p.u, cur.e2u + p.e2u) * (cur.hu + k.su + p.hu + su_p);
    // T(c, J0): the south face of v(c, J0)
    const double vs = 0.5 * (cur.v + p.v) * cur.e1t;
    const double deps = cur.ht + cur.s;
    k.Fvy_s = upw(vs, p.v, cur.v) * vs * deps;
    k.Dvy_s = qm(cur.v - p.v, cur.e2t) * deps;
    k.pt_s = p.pt;
    if (J0 == 1 && store) {
      // v(c, 0): outside the momentum loop (:520); solid wall (:656-660) or
      // kept (Flather, in k_flather_general, may replace it)
      A.va[L.idx(c, 0)] = (p.pt * cur.pt == 0) ? 0.0 : p.v;
    }
  }

  // slots of rows j, j+1 and j+AHEAD (= the slot of row j-1)
  int s_w = 0, s_n = RG > 1 ? 1 : 0, s_i = RG > 0 ? RG - 1 : 0;
  long o_st = L.idx(c, J0);
#pragma unroll 1
  for (int j = J0; j <= J1; ++j) {
    GNext nx;
    GOwn w;
    if constexpr (RG > 0) {
      // row j+AHEAD into the slot of row j-1, the mask of row j+2 ahead
      if (j + AHEAD <= r_stop) ring_issue_g(my + s_i * GF * 32, A, L.idx(cl, j + AHEAD));
      else stepdev::cp_commit();
      const int pt2 = (j + 2 <= L.jpj + 1) ? A.g.pt[L.idx(cl, j + 2)] : 0;
      stepdev::cp_wait<AHEAD - 1>();  // rows <= j+1 have landed
      ring_next(nx, my + s_n * GF * 32, pt1);
      ring_own(w, my + s_w * GF * 32);
      pt1 = pt2;
      s_w = s_n;
      s_n = ring_step(s_n, RG);
      s_i = ring_step(s_i, RG);
    } else {
      load_next(nx, A, L.idx(cl, j + 1));  // row j+1 <= jpj+1
      load_own(w, A, L.idx(cl, j));
    }
    const int pt_e = dni(cur.pt), pt_w = upi(cur.pt);
    const int ptn_e = dni(nx.pt), ptn_w = upi(nx.pt);
    const double s_e = dn(cur.s);
    // default build: reciprocals of e1v*e2v and e1t*e2t at (c, j) (the
    // latter gives 1/e1t as e2t/(e1t*e2t))
    const double rv = grecip(w.e1v * w.e2v);
    const double rt = grecip(cur.e1t * cur.e2t);

    // sshn_v at (c, j), sshn_u at (c, j+1)
    const double sv = sshn_v_at(cur, w, nx, c, j, jpi, jpj, A.sv_st, L.idx(cl, j), rv);
    const double su_n = sshn_u_at(nx, c, j + 1, jpi, jpj, A.su_st, L.idx(cl, j + 1), grecip(nx.e1u * nx.e2u));

    // ---- continuity (:397-405) and the clamped SSH (:631-644) ----
    const double r1 = (k.su + cur.hu) * cur.u;
    const double r2 = up(r1);
    const double r3 = (sv + w.hv) * cur.v;
    double ssha = cur.s + qr((r2 - r1 + k.cf_s - r3) * C.rdt, e12t_at(cur, c, j, jpi, jpj), rt);
    if (cur.pt > 0 && (k.pt_s < 0 || nx.pt < 0 || pt_e < 0 || pt_w < 0)) ssha = A.tide;

    // ---- x-face at T(c,j), between u(c-1,j) and u(c,j) ----
    const double u_wn = up(cur.u);
    const double uw = 0.5 * (cur.u + u_wn) * cur.e2t;
    const double dep = cur.ht + cur.s;
    const double Fx = upw(uw, u_wn, cur.u) * uw * dep;
    const double Dx = qr(cur.u - u_wn, cur.e1t, cur.e2t * rt) * dep;

    // ---- corner (c,j): north face of u(c,j) / south face of u(c,j+1) ----
    const double v_e = dn(cur.v);
    const double vnc = 0.5 * (cur.v + v_e);
    const double vfl = 0.5 * vnc * (w.e1v + dn(w.e1v));
    const double depc = 0.5 * (w.hv + sv + dn(w.hv) + dn(sv));
    const bool mn = nx.pt <= 0 || ptn_e <= 0;   // u(c,j)'s test of row j+1
    const bool ms = cur.pt <= 0 || pt_e <= 0;   // u(c,j+1)'s test of row j
    const double Fuy_full = upw(vfl, cur.u, nx.u) * vfl * depc;
    const double Fuy_n = mn ? upwind_lo_only(vfl, cur.u) * vfl * depc : Fuy_full;
    const double Fuy_s_next = ms ? upwind_hi_only(vfl, nx.u) * vfl * depc : Fuy_full;
    const double Gy = qm(nx.u - cur.u, cur.e2u + nx.e2u);
    const double dudy_n = mn ? 0.0 : Gy * (cur.hu + k.su + nx.hu + su_n);
    const double dudy_s_next = ms ? 0.0 : Gy * (nx.hu + su_n + cur.hu + k.su);
    // ---- corner (c,j): east face of v(c,j) / west face of v(c+1,j) ----
    const double uec = 0.5 * (cur.u + nx.u);
    const double ufl = 0.5 * uec * (cur.e2u + nx.e2u);
    const double depcu = 0.5 * (cur.hu + k.su + nx.hu + su_n);
    const bool me = pt_e <= 0 || ptn_e <= 0;        // v(c,j)'s test of column c+1
    const bool mw_next = cur.pt <= 0 || nx.pt <= 0;  // v(c+1,j)'s test of column c
    const double Fvx_full = upw(ufl, cur.v, v_e) * ufl * depcu;
    const double Fvx_e = me ? upwind_lo_only(ufl, cur.v) * ufl * depcu : Fvx_full;
    const double Fvx_w_next = mw_next ? upwind_hi_only(ufl, v_e) * ufl * depcu : Fvx_full;
    const double hv_e = dn(w.hv), sv_e = dn(sv);
    const double Gx = qm(v_e - cur.v, w.e1v + dn(w.e1v));
    const double dvdx_e = me ? 0.0 : Gx * (w.hv + sv + hv_e + sv_e);
    const double dvdx_w_next = mw_next ? 0.0 : Gx * (hv_e + sv_e + w.hv + sv);
    // ---- y-face at T(c,j+1), between v(c,j) and v(c,j+1) ----
    const double vfn = 0.5 * (cur.v + nx.v) * nx.e1t;
    const double depn = nx.ht + nx.s;
    const double Fvy_n = upw(vfn, cur.v, nx.v) * vfn * depn;
    const double Dvy_n = qm(nx.v - cur.v, nx.e2t) * depn;

    // ---- u equation at u(c,j) (:431-517), solid walls (:648-652) ----
    // Both equations are evaluated in every lane and the result selected
    // afterwards: a lane outside an equation's mask still takes part in the
    // shuffles its neighbours' results need (a shuffle whose source lane has
    // branched away returns an undefined value), and the values it computes
    // for itself (quotients by the zero scale factors of the border ring
    // included) are discarded.
    const double Fx_e = dn(Fx), Dx_e = dn(Dx);
    double ua;
    {
      const double Hu = cur.hu + k.su;
      const double adv = Fx - Fx_e + k.Fuy_s - Fuy_n;
      double vis = (Dx_e - Dx) * cur.e2u + (dudy_n - k.dudy_s) * cur.e1u * 0.5;
      vis = C.visc * vis;
      const double e12u = cur.e1u * cur.e2u;
      const double cor = 0.5 * (w.fcu * (k.vnc_s + vnc)) * e12u * Hu;
      const double hpg = -(C.g * Hu * cur.e2u * (s_e - cur.s));
      const double um = qf(qh(cur.u * Hu + qm(C.rdt * (adv + vis + cor + hpg), e12u), cur.hu + 0.0), C);
      const bool mom = c >= 1 && c <= jpi - 1 && cur.pt > 0 && pt_e > 0;
      ua = mom ? um : ((cur.pt * pt_e == 0) ? 0.0 : cur.u);
    }

    // ---- v equation at v(c,j) (:520-609), solid walls (:656-660) ----
    const double Fvx_w = up(Fvx_w_next), dvdx_w = up(dvdx_w_next), uec_w = up(uec);
    double va;
    {
      const double Hv = w.hv + sv;
      const double adv = Fvx_w - Fvx_e + k.Fvy_s - Fvy_n;
      double vis = (Dvy_n - k.Dvy_s) * w.e1v + (dvdx_e - dvdx_w) * w.e2v * 0.5;
      vis = C.visc * vis;
      const double e12v = w.e1v * w.e2v;
      const double cor = -(0.5 * (w.fcv * (uec + uec_w)) * e12v * Hv);
      const double hpg = -(C.g * Hv * w.e1v * (nx.s - cur.s));
      const double vm = qf(qh(cur.v * Hv + qr(C.rdt * (adv + vis + cor + hpg), e12v, rv), w.hv + 0.0), C);
      const bool mom = j <= jpj - 1 && !(cur.pt + pt_e <= 0) && cur.pt > 0 && nx.pt > 0;
      va = mom ? vm : ((cur.pt * nx.pt == 0) ? 0.0 : cur.v);
    }

    if (store) {
      A.ssha[o_st] = ssha;
      A.va[o_st] = va;
    }
    if (store_u) A.ua[o_st] = ua;
    o_st += pitch;
    // carry to row j+1
    k.su = su_n;
    k.cf_s = r3;
    k.Fuy_s = Fuy_s_next;
    k.vnc_s = vnc;
    k.dudy_s = dudy_s_next;
    k.Fvy_s = Fvy_n;
    k.Dvy_s = Dvy_n;
    k.pt_s = cur.pt;
    cur = nx;
  }
  if constexpr (RG > 0) asm volatile("cp.async.wait_all;" ::: "memory");
}

// One Flather chain (see the file comment): x = ji, y = jj, z = kind (0: u,
// first branch; 1: u, second branch; 2: v, first; 3: v, second), w = 1 when
// the chain continues with the second-branch point next along the sweep.
// sshn_u / sshn_v at one point after `next`; outside the arrays' ranges
// ((0:jpi, 1:jpj), (1:jpi, 0:jpj)), where only masks the reference itself
// cannot run reach, the stored value.
__device__ __forceinline__ double sshn_u_pt(const Layout& L, const GenArgs& A, int ji, int jj) {
  const long o = L.idx(ji, jj);
  if (ji < 0 || ji > L.jpi || jj < 1 || jj > L.jpj) return A.su_st[o];
  const int a = A.g.pt[o], b = A.g.pt[o + 1];
  if (a + b > 0) {
    const double s0 = A.sshn[o], s1 = A.sshn[o + 1];
    if (a * b > 0) {
      const double t0 = (ji >= 1 && ji <= L.jpi) ? A.g.e1t[o] * A.g.e2t[o] : 0.0;
      const double t1 = (ji + 1 <= L.jpi) ? A.g.e1t[o + 1] * A.g.e2t[o + 1] : 0.0;
      return 0.5 * (t0 * s0 + t1 * s1) / (A.g.e1u[o] * A.g.e2u[o]);
    }
    if (a <= 0) return s1;
    return s0;
  }
  return A.su_st[o];
}
__device__ __forceinline__ double sshn_v_pt(const Layout& L, const GenArgs& A, int ji, int jj) {
  const long o = L.idx(ji, jj), on = o + L.pitch;
  if (ji < 1 || ji > L.jpi || jj < 0 || jj > L.jpj) return A.sv_st[o];
  const int a = A.g.pt[o], b = A.g.pt[on];
  if (a + b > 0) {
    const double s0 = A.sshn[o], s1 = A.sshn[on];
    if (a * b > 0) {
      const double t0 = (jj >= 1 && jj <= L.jpj) ? A.g.e1t[o] * A.g.e2t[o] : 0.0;
      const double t1 = (jj + 1 <= L.jpj) ? A.g.e1t[on] * A.g.e2t[on] : 0.0;
      return 0.5 * (t0 * s0 + t1 * s1) / (A.g.e1v[o] * A.g.e2v[o]);
    }
    if (a <= 0) return s1;
    return s0;
  }
  return A.sv_st[o];
}

__device__ __forceinline__ void flather_op(const Layout& L, const GenArgs& A, int ji, int jj, int kind) {
  if (kind < 2) {  // :673-679
    const int jiu = kind == 0 ? ji + 1 : ji - 1;
    const long o = L.idx(ji, jj);
    A.ua[o] = A.ua[L.idx(jiu, jj)] + sqrt(kG / A.hu[o]) * (sshn_u_pt(L, A, ji, jj) - sshn_u_pt(L, A, jiu, jj));
  } else {  // :688-694
    const int jjv = kind == 2 ? jj + 1 : jj - 1;
    const long o = L.idx(ji, jj);
    A.va[o] = A.va[L.idx(ji, jjv)] + sqrt(kG / A.hv[o]) * (sshn_v_pt(L, A, ji, jj) - sshn_v_pt(L, A, ji, jjv));
  }
}

__global__ void k_flather_general(Layout L, GenArgs A, const int4* __restrict__ chains, int n) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int4 ch = chains[t];
  flather_op(L, A, ch.x, ch.y, ch.z);
  if (ch.w) {  // the second-branch point after it in the sweep
    if (ch.z == 0) flather_op(L, A, ch.x + 1, ch.y, 1);
    else flather_op(L, A, ch.x, ch.y + 1, 3);
  }
}

}  // namespace

cudaError_t launch_fused_general(const Layout& L, const Consts& C, const GenArgs& a, const int4* chains,
                                 int nchains, int ring, int tile_y, cudaStream_t s) {
  constexpr int NW = 2;
  const int cols_per_cta = COLS_PER_WARP * NW;
  if (tile_y < 1) tile_y = 32;
  dim3 grid((unsigned)((L.jpi + cols_per_cta - 1) / cols_per_cta), (unsigned)((L.jpj + tile_y - 1) / tile_y));
  switch (ring) {
    case 0: k_fused_general<0><<<grid, 32 * NW, 0, s>>>(L, C, a, tile_y); break;
    case 3: k_fused_general<3><<<grid, 32 * NW, 0, s>>>(L, C, a, tile_y); break;
    case 4: k_fused_general<4><<<grid, 32 * NW, 0, s>>>(L, C, a, tile_y); break;
    default: return cudaErrorInvalidValue;
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || nchains == 0) return e;
  k_flather_general<<<(nchains + 127) / 128, 128, 0, s>>>(L, a, chains, nchains);
  return cudaGetLastError();
}

// The Flather points of a general grid as chains in the sweeps' order
// (original/nemolite2d.f90:669-695); pt over (0:jpi+1, 0:jpj+1), ld jpi+2.
void flather_chains(const int* pt, int jpi, int jpj, std::vector<int4>& out) {
  const long ld = jpi + 2;
  auto P = [&](int ji, int jj) { return pt[(long)jj * ld + ji]; };
  out.clear();
  // u: ji = 0..jpi, jj = 1..jpj
  for (int jj = 1; jj <= jpj; ++jj)
    for (int ji = 0; ji <= jpi; ++ji) {
      const int a = P(ji, jj), b = P(ji + 1, jj);
      if (a + b <= -1) continue;
      if (a < 0) {
        // a second-branch point right after it reads its new value
        const bool chain = ji + 1 <= jpi && P(ji + 1, jj) + P(ji + 2, jj) > -1 && P(ji + 1, jj) >= 0 &&
                           P(ji + 2, jj) < 0;
        out.push_back(make_int4(ji, jj, 0, chain ? 1 : 0));
        if (chain) ++ji;
      } else if (b < 0) {
        out.push_back(make_int4(ji, jj, 1, 0));
      }
    }
  // v: ji = 1..jpi, jj = 0..jpj
  for (int ji = 1; ji <= jpi; ++ji)
    for (int jj = 0; jj <= jpj; ++jj) {
      const int a = P(ji, jj), b = P(ji, jj + 1);
      if (a + b <= -1) continue;
      if (a < 0) {
        const bool chain = jj + 1 <= jpj && P(ji, jj + 1) + P(ji, jj + 2) > -1 && P(ji, jj + 1) >= 0 &&
                           P(ji, jj + 2) < 0;
        out.push_back(make_int4(ji, jj, 2, chain ? 1 : 0));
        if (chain) ++jj;
      } else if (b < 0) {
        out.push_back(make_int4(ji, jj, 3, 0));
      }
    }
}

}  // namespace nemo
