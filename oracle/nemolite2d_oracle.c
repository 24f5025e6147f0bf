/*
 * CPU oracle for the NEMOLite2D time-stepper -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of original/nemolite2d.f90 (the serial Fortran
 * model).  Every loop keeps the reference's bounds, CYCLE conditions and
 * left-to-right evaluation order; SIGN(a,b) is copysign(fabs(a),b) as
 * gfortran evaluates it (a negative zero B gives a negative result).
 * Build with -O2 -ffp-contract=off -fno-fast-math -fno-builtin so every
 * multiply and add rounds separately, as the Fortran source reads.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU legs use this file.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* original/nemolite2d.f90:15-18 */
static const double PI = 3.1415926535897932;
static const double G = 9.80665;
static const double OMEGA = 7.292116e-05;

static int g_threads = 1;

void oracle_set_threads(int n) { g_threads = n < 1 ? 1 : n; }
int oracle_get_threads(void) { return g_threads; }

struct oracle_model {
  oracle_params p;
  int jpi, jpj, ld;
  int* pt;
  double *e1t, *e2t, *e1u, *e2u, *e1v, *e2v, *e12t, *e12u, *e12v;
  double *gphiu, *gphiv, *xt, *yt, *ht, *hu, *hv;
  double *sshn, *sshn_u, *sshn_v, *ssha, *ssha_u, *ssha_v;
  double *un, *vn, *ua, *va;
};

#define I(ji, jj) ((long)(jj) * m->ld + (ji))

int oracle_jpi(const oracle_model* m) { return m->jpi; }
int oracle_jpj(const oracle_model* m) { return m->jpj; }

void oracle_default_params(oracle_params* p) {
  /* Defaults of setup, original/nemolite2d.f90:107-118 (jpiglo=258 -> 256). */
  memset(p, 0, sizeof(*p));
  p->jpi = 256;
  p->jpj = 256;
  p->dx = 1000.0;
  p->dy = 1000.0;
  p->dep_const = 100.0;
  p->nit000 = 1;
  p->nitend = 1000;
  p->irecord = 1;
  p->rdt = 10.0;
  p->cbfr = 0.001;
  p->visc = 100.0;
  p->amp_tide = 0.2;
  p->tide_phase = 0.0;
  p->lat = 50.0;
  p->nbump = 0;
  p->seed = 1234;
  p->bump_amp = 40.0;
  p->bump_wmin = 20.0e3;
  p->bump_wmax = 200.0e3;
  p->hmin = 10.0;
  p->hmax = 1.0e30;
}

/* ---- seeded Gaussian-bump bathymetry (no reference counterpart) --------
 * SplitMix64 (Steele, Lea & Flood 2014) drives the bump parameters; each
 * bump is separable, exp(-((x-xc)/w)^2) * exp(-((y-yc)/w)^2), tabulated on
 * the half-grid x_k = k*(dx/2).  depth = clamp(H0 + sum_b ax_b[kx]*gy_b[ky]),
 * summed b = 0,1,... with separate roundings.  The product library implements
 * the same rule independently; tests compare the two bit for bit. */
static uint64_t smix_next(uint64_t* s) {
  uint64_t z = (*s += 0x9E3779B97F4A7C15ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
static double smix_unif(uint64_t* s) {
  return (double)(smix_next(s) >> 11) * 0x1.0p-53;
}

static void bathymetry(oracle_model* m) {
  const oracle_params* p = &m->p;
  int jpi = m->jpi, jpj = m->jpj, nb = p->nbump;
  int nkx = 2 * jpi + 2, nky = 2 * jpj + 2;
  double* ax = (double*)malloc(sizeof(double) * (size_t)nb * nkx);
  double* gy = (double*)malloc(sizeof(double) * (size_t)nb * nky);
  uint64_t s = p->seed;
  double lx = (double)jpi * p->dx, ly = (double)jpj * p->dy;
  double hdx = 0.5 * p->dx, hdy = 0.5 * p->dy;
  for (int b = 0; b < nb; ++b) {
    double xc = smix_unif(&s) * lx;
    double yc = smix_unif(&s) * ly;
    double amp = p->bump_amp * (2.0 * smix_unif(&s) - 1.0);
    double w = p->bump_wmin + (p->bump_wmax - p->bump_wmin) * smix_unif(&s);
    for (int k = 0; k < nkx; ++k) {
      double t = ((double)k * hdx - xc) / w;
      ax[(size_t)b * nkx + k] = amp * exp(-(t * t));
    }
    for (int k = 0; k < nky; ++k) {
      double t = ((double)k * hdy - yc) / w;
      gy[(size_t)b * nky + k] = exp(-(t * t));
    }
  }
#define DEPTH(kx, ky, out)                                              \
  do {                                                                  \
    double acc_ = 0.0;                                                  \
    for (int b_ = 0; b_ < nb; ++b_)                                     \
      acc_ = acc_ + ax[(size_t)b_ * nkx + (kx)] * gy[(size_t)b_ * nky + (ky)]; \
    double h_ = p->dep_const + acc_;                                    \
    h_ = h_ < p->hmin ? p->hmin : h_;                                   \
    h_ = h_ > p->hmax ? p->hmax : h_;                                   \
    (out) = h_;                                                         \
  } while (0)
  for (int jj = 1; jj <= jpj; ++jj)
    for (int ji = 1; ji <= jpi; ++ji) DEPTH(2 * ji - 1, 2 * jj - 1, m->ht[I(ji, jj)]);
  for (int jj = 1; jj <= jpj; ++jj)
    for (int ji = 0; ji <= jpi; ++ji) DEPTH(2 * ji, 2 * jj - 1, m->hu[I(ji, jj)]);
  for (int jj = 0; jj <= jpj; ++jj)
    for (int ji = 1; ji <= jpi; ++ji) DEPTH(2 * ji - 1, 2 * jj, m->hv[I(ji, jj)]);
#undef DEPTH
  free(ax);
  free(gy);
}

static double* zalloc(long n) { return (double*)calloc((size_t)n, sizeof(double)); }

/* initialisation of sshn_u/sshn_v, :337-353 (min/max-clamped averages) */
static void init_sshn_uv(oracle_model* m) {
  const int jpi = m->jpi, jpj = m->jpj;
  for (int ji = 0; ji <= jpi; ++ji)
    for (int jj = 1; jj <= jpj; ++jj) {
      int i1 = ji + 1 < jpi ? ji + 1 : jpi;
      int i2 = ji > 1 ? ji : 1;
      double r = m->e12t[I(i1, jj)] * m->sshn[I(i1, jj)] + m->e12t[I(i2, jj)] * m->sshn[I(i2, jj)];
      m->sshn_u[I(ji, jj)] = 0.5 * r / m->e12u[I(ji, jj)];
    }
  for (int ji = 1; ji <= jpi; ++ji)
    for (int jj = 0; jj <= jpj; ++jj) {
      int j1 = jj + 1 < jpj ? jj + 1 : jpj;
      int j2 = jj > 1 ? jj : 1;
      double r = m->e12t[I(ji, j1)] * m->sshn[I(ji, j1)] + m->e12t[I(ji, j2)] * m->sshn[I(ji, j2)];
      m->sshn_v[I(ji, jj)] = 0.5 * r / m->e12v[I(ji, jj)];
    }
}

/* cell areas over the ranges :263-279 fill; zero elsewhere */
static void cell_areas(oracle_model* m) {
  const int jpi = m->jpi, jpj = m->jpj;
  const size_t n = (size_t)(jpi + 2) * (jpj + 2);
  memset(m->e12t, 0, n * sizeof(double));
  memset(m->e12u, 0, n * sizeof(double));
  memset(m->e12v, 0, n * sizeof(double));
  for (int jj = 1; jj <= jpj; ++jj)
    for (int ji = 1; ji <= jpi; ++ji) m->e12t[I(ji, jj)] = m->e1t[I(ji, jj)] * m->e2t[I(ji, jj)];
  for (int jj = 1; jj <= jpj; ++jj)
    for (int ji = 0; ji <= jpi; ++ji) m->e12u[I(ji, jj)] = m->e1u[I(ji, jj)] * m->e2u[I(ji, jj)];
  for (int jj = 0; jj <= jpj; ++jj)
    for (int ji = 1; ji <= jpi; ++ji) m->e12v[I(ji, jj)] = m->e1v[I(ji, jj)] * m->e2v[I(ji, jj)];
}

oracle_model* oracle_create(const oracle_params* p) {
  if (p->jpi < 2 || p->jpj < 2) return NULL;
  oracle_model* m = (oracle_model*)calloc(1, sizeof(oracle_model));
  m->p = *p;
  m->jpi = p->jpi;
  m->jpj = p->jpj;
  m->ld = p->jpi + 2;
  long n = (long)(p->jpi + 2) * (p->jpj + 2);
  /* allocation, :285-320: every array zero-initialised. */
  m->pt = (int*)calloc((size_t)n, sizeof(int));
  double** arrs[] = {&m->e1t, &m->e2t, &m->e1u, &m->e2u, &m->e1v, &m->e2v,
                     &m->e12t, &m->e12u, &m->e12v, &m->gphiu, &m->gphiv,
                     &m->xt, &m->yt, &m->ht, &m->hu, &m->hv, &m->sshn,
                     &m->sshn_u, &m->sshn_v, &m->ssha, &m->ssha_u, &m->ssha_v,
                     &m->un, &m->vn, &m->ua, &m->va};
  for (size_t k = 0; k < sizeof(arrs) / sizeof(arrs[0]); ++k) *arrs[k] = zalloc(n);

  int jpi = m->jpi, jpj = m->jpj;
  double dx = p->dx, dy = p->dy;
  /* grid, CASE(1), :184-202: masks */
  for (int jj = 0; jj <= jpj + 1; ++jj)
    for (int ji = 0; ji <= jpi + 1; ++ji) m->pt[I(ji, jj)] = 1;
  for (int jj = 0; jj <= jpj + 1; ++jj) {
    m->pt[I(0, jj)] = 0;
    m->pt[I(jpi + 1, jj)] = 0;
  }
  for (int ji = 0; ji <= jpi + 1; ++ji) m->pt[I(ji, jpj + 1)] = 0;
  for (int ji = 1; ji <= jpi; ++ji) m->pt[I(ji, 0)] = -1;
  /* :210-222 scale factors and latitude */
  for (int jj = 1; jj <= jpj; ++jj)
    for (int ji = 1; ji <= jpi; ++ji) { m->e1t[I(ji, jj)] = dx; m->e2t[I(ji, jj)] = dy; }
  for (int jj = 1; jj <= jpj; ++jj)
    for (int ji = 0; ji <= jpi; ++ji) {
      m->e1u[I(ji, jj)] = dx; m->e2u[I(ji, jj)] = dy; m->gphiu[I(ji, jj)] = p->lat;
    }
  for (int jj = 0; jj <= jpj; ++jj)
    for (int ji = 1; ji <= jpi; ++ji) {
      m->e1v[I(ji, jj)] = dx; m->e2v[I(ji, jj)] = dy; m->gphiv[I(ji, jj)] = p->lat;
    }
  /* :224-233 coordinates (cumulative sums, as the reference forms them) */
  for (int jj = 1; jj <= jpj; ++jj) m->xt[I(1, jj)] = 0.0 + 0.5 * m->e1t[I(1, jj)];
  for (int ji = 1; ji <= jpi; ++ji) m->yt[I(ji, 1)] = 0.0 + 0.5 * m->e2t[I(ji, 1)];
  for (int ji = 2; ji <= jpi; ++ji)
    for (int jj = 1; jj <= jpj; ++jj) m->xt[I(ji, jj)] = m->xt[I(ji - 1, jj)] + dx;
  for (int jj = 2; jj <= jpj; ++jj)
    for (int ji = 1; ji <= jpi; ++ji) m->yt[I(ji, jj)] = m->yt[I(ji, jj - 1)] + dy;
  /* :238-254 depth */
  if (p->nbump <= 0) {
    for (int jj = 1; jj <= jpj; ++jj)
      for (int ji = 1; ji <= jpi; ++ji) m->ht[I(ji, jj)] = p->dep_const;
    for (int jj = 1; jj <= jpj; ++jj)
      for (int ji = 0; ji <= jpi; ++ji) m->hu[I(ji, jj)] = p->dep_const;
    for (int jj = 0; jj <= jpj; ++jj)
      for (int ji = 1; ji <= jpi; ++ji) m->hv[I(ji, jj)] = p->dep_const;
  } else {
    bathymetry(m);
  }
  /* :263-279 cell areas */
  cell_areas(m);

  /* initialisation, :331-365 */
  for (int ji = 1; ji <= jpi; ++ji)
    for (int jj = 1; jj <= jpj; ++jj) m->sshn[I(ji, jj)] = 0.0;
  init_sshn_uv(m);
  for (int jj = 1; jj <= jpj; ++jj)
    for (int ji = 0; ji <= jpi; ++ji) m->un[I(ji, jj)] = 0.0;
  for (int jj = 0; jj <= jpj; ++jj)
    for (int ji = 1; ji <= jpi; ++ji) m->vn[I(ji, jj)] = 0.0;
  return m;
}

void oracle_destroy(oracle_model* m) {
  if (!m) return;
  double* arrs[] = {m->e1t, m->e2t, m->e1u, m->e2u, m->e1v, m->e2v, m->e12t,
                    m->e12u, m->e12v, m->gphiu, m->gphiv, m->xt, m->yt, m->ht,
                    m->hu, m->hv, m->sshn, m->sshn_u, m->sshn_v, m->ssha,
                    m->ssha_u, m->ssha_v, m->un, m->vn, m->ua, m->va};
  for (size_t k = 0; k < sizeof(arrs) / sizeof(arrs[0]); ++k) free(arrs[k]);
  free(m->pt);
  free(m);
}

/* SIGN(a, b) with gfortran semantics: |a| carrying the sign bit of b. */
static inline double fsign(double a, double b) { return copysign(fabs(a), b); }

/* continuity, original/nemolite2d.f90:397-405 */
void oracle_continuity(oracle_model* m) {
  const int jpi = m->jpi, jpj = m->jpj;
  const double rdt = m->p.rdt;
#pragma omp parallel for num_threads(g_threads) if (g_threads > 1) schedule(static)
  for (int jj = 1; jj <= jpj; ++jj)
    for (int ji = 1; ji <= jpi; ++ji) {
      double r1 = (m->sshn_u[I(ji, jj)] + m->hu[I(ji, jj)]) * m->un[I(ji, jj)];
      double r2 = (m->sshn_u[I(ji - 1, jj)] + m->hu[I(ji - 1, jj)]) * m->un[I(ji - 1, jj)];
      double r3 = (m->sshn_v[I(ji, jj)] + m->hv[I(ji, jj)]) * m->vn[I(ji, jj)];
      double r4 = (m->sshn_v[I(ji, jj - 1)] + m->hv[I(ji, jj - 1)]) * m->vn[I(ji, jj - 1)];
      m->ssha[I(ji, jj)] = m->sshn[I(ji, jj)] + (r2 - r1 + r4 - r3) * rdt / m->e12t[I(ji, jj)];
    }
}

/* momentum, u equation, original/nemolite2d.f90:431-517 */
void oracle_momentum_u(oracle_model* m) {
  const int jpi = m->jpi, jpj = m->jpj;
  const double rdt = m->p.rdt, cbfr = m->p.cbfr, visc = m->p.visc;
  const double d2r = PI / 180.0;
  const int* pt = m->pt;
  const double *un = m->un, *vn = m->vn, *sshn = m->sshn, *sshn_u = m->sshn_u,
               *sshn_v = m->sshn_v, *ht = m->ht, *hu = m->hu, *hv = m->hv;
#pragma omp parallel for num_threads(g_threads) if (g_threads > 1) schedule(static)
  for (int jj = 1; jj <= jpj; ++jj)
    for (int ji = 1; ji <= jpi - 1; ++ji) {
      if (pt[I(ji, jj)] + pt[I(ji + 1, jj)] <= 0) continue;
      if (pt[I(ji, jj)] <= 0 || pt[I(ji + 1, jj)] <= 0) continue;

      double u_e = 0.5 * (un[I(ji, jj)] + un[I(ji + 1, jj)]) * m->e2t[I(ji + 1, jj)];
      double depe = ht[I(ji + 1, jj)] + sshn[I(ji + 1, jj)];
      double u_w = 0.5 * (un[I(ji, jj)] + un[I(ji - 1, jj)]) * m->e2t[I(ji, jj)];
      double depw = ht[I(ji, jj)] + sshn[I(ji, jj)];

      double v_sc = 0.5 * (vn[I(ji, jj - 1)] + vn[I(ji + 1, jj - 1)]);
      double v_s = 0.5 * v_sc * (m->e1v[I(ji, jj - 1)] + m->e1v[I(ji + 1, jj - 1)]);
      double deps = 0.5 * (hv[I(ji, jj - 1)] + sshn_v[I(ji, jj - 1)] + hv[I(ji + 1, jj - 1)] +
                           sshn_v[I(ji + 1, jj - 1)]);
      double v_nc = 0.5 * (vn[I(ji, jj)] + vn[I(ji + 1, jj)]);
      double v_n = 0.5 * v_nc * (m->e1v[I(ji, jj)] + m->e1v[I(ji + 1, jj)]);
      double depn = 0.5 * (hv[I(ji, jj)] + sshn_v[I(ji, jj)] + hv[I(ji + 1, jj)] +
                           sshn_v[I(ji + 1, jj)]);

      double uu_w = (0.5 - fsign(0.5, u_w)) * un[I(ji, jj)] + (0.5 + fsign(0.5, u_w)) * un[I(ji - 1, jj)];
      double uu_e = (0.5 + fsign(0.5, u_e)) * un[I(ji, jj)] + (0.5 - fsign(0.5, u_e)) * un[I(ji + 1, jj)];
      double uu_s, uu_n;
      if (pt[I(ji, jj - 1)] <= 0 || pt[I(ji + 1, jj - 1)] <= 0)
        uu_s = (0.5 - fsign(0.5, v_s)) * un[I(ji, jj)];
      else
        uu_s = (0.5 - fsign(0.5, v_s)) * un[I(ji, jj)] + (0.5 + fsign(0.5, v_s)) * un[I(ji, jj - 1)];
      if (pt[I(ji, jj + 1)] <= 0 || pt[I(ji + 1, jj + 1)] <= 0)
        uu_n = (0.5 + fsign(0.5, v_n)) * un[I(ji, jj)];
      else
        uu_n = (0.5 + fsign(0.5, v_n)) * un[I(ji, jj)] + (0.5 - fsign(0.5, v_n)) * un[I(ji, jj + 1)];

      double adv = uu_w * u_w * depw - uu_e * u_e * depe + uu_s * v_s * deps - uu_n * v_n * depn;

      double dudx_e = (un[I(ji + 1, jj)] - un[I(ji, jj)]) / m->e1t[I(ji + 1, jj)] *
                      (ht[I(ji + 1, jj)] + sshn[I(ji + 1, jj)]);
      double dudx_w = (un[I(ji, jj)] - un[I(ji - 1, jj)]) / m->e1t[I(ji, jj)] *
                      (ht[I(ji, jj)] + sshn[I(ji, jj)]);
      double dudy_s, dudy_n;
      if (pt[I(ji, jj - 1)] <= 0 || pt[I(ji + 1, jj - 1)] <= 0)
        dudy_s = 0.0;
      else
        dudy_s = (un[I(ji, jj)] - un[I(ji, jj - 1)]) / (m->e2u[I(ji, jj)] + m->e2u[I(ji, jj - 1)]) *
                 (hu[I(ji, jj)] + sshn_u[I(ji, jj)] + hu[I(ji, jj - 1)] + sshn_u[I(ji, jj - 1)]);
      if (pt[I(ji, jj + 1)] <= 0 || pt[I(ji + 1, jj + 1)] <= 0)
        dudy_n = 0.0;
      else
        dudy_n = (un[I(ji, jj + 1)] - un[I(ji, jj)]) / (m->e2u[I(ji, jj)] + m->e2u[I(ji, jj + 1)]) *
                 (hu[I(ji, jj)] + sshn_u[I(ji, jj)] + hu[I(ji, jj + 1)] + sshn_u[I(ji, jj + 1)]);

      double vis = (dudx_e - dudx_w) * m->e2u[I(ji, jj)] + (dudy_n - dudy_s) * m->e1u[I(ji, jj)] * 0.5;
      vis = visc * vis;

      double cor = 0.5 * (2.0 * OMEGA * sin(m->gphiu[I(ji, jj)] * d2r) * (v_sc + v_nc)) *
                   m->e12u[I(ji, jj)] * (hu[I(ji, jj)] + sshn_u[I(ji, jj)]);
      /* Fortran -g*x*y*z is -(g*x*y*z); negation is exact either way. */
      double hpg = -(G * (hu[I(ji, jj)] + sshn_u[I(ji, jj)]) * m->e2u[I(ji, jj)] *
                     (sshn[I(ji + 1, jj)] - sshn[I(ji, jj)]));

      m->ua[I(ji, jj)] = (un[I(ji, jj)] * (hu[I(ji, jj)] + sshn_u[I(ji, jj)]) +
                          rdt * (adv + vis + cor + hpg) / m->e12u[I(ji, jj)]) /
                         (hu[I(ji, jj)] + m->ssha_u[I(ji, jj)]) / (1.0 + cbfr * rdt);
    }
}

/* momentum, v equation, original/nemolite2d.f90:520-609 */
void oracle_momentum_v(oracle_model* m) {
  const int jpi = m->jpi, jpj = m->jpj;
  const double rdt = m->p.rdt, cbfr = m->p.cbfr, visc = m->p.visc;
  const double d2r = PI / 180.0;
  const int* pt = m->pt;
  const double *un = m->un, *vn = m->vn, *sshn = m->sshn, *sshn_u = m->sshn_u,
               *sshn_v = m->sshn_v, *ht = m->ht, *hu = m->hu, *hv = m->hv;
#pragma omp parallel for num_threads(g_threads) if (g_threads > 1) schedule(static)
  for (int jj = 1; jj <= jpj - 1; ++jj)
    for (int ji = 1; ji <= jpi; ++ji) {
      /* The reference tests pt(ji+1,jj) here (:523); kept verbatim. */
      if (pt[I(ji, jj)] + pt[I(ji + 1, jj)] <= 0) continue;
      if (pt[I(ji, jj)] <= 0 || pt[I(ji, jj + 1)] <= 0) continue;

      double v_n = 0.5 * (vn[I(ji, jj)] + vn[I(ji, jj + 1)]) * m->e1t[I(ji, jj + 1)];
      double depn = ht[I(ji, jj + 1)] + sshn[I(ji, jj + 1)];
      double v_s = 0.5 * (vn[I(ji, jj)] + vn[I(ji, jj - 1)]) * m->e1t[I(ji, jj)];
      double deps = ht[I(ji, jj)] + sshn[I(ji, jj)];

      double u_wc = 0.5 * (un[I(ji - 1, jj)] + un[I(ji - 1, jj + 1)]);
      double u_w = 0.5 * u_wc * (m->e2u[I(ji - 1, jj)] + m->e2u[I(ji - 1, jj + 1)]);
      double depw = 0.50 * (hu[I(ji - 1, jj)] + sshn_u[I(ji - 1, jj)] + hu[I(ji - 1, jj + 1)] +
                            sshn_u[I(ji - 1, jj + 1)]);
      double u_ec = 0.5 * (un[I(ji, jj)] + un[I(ji, jj + 1)]);
      double u_e = 0.5 * u_ec * (m->e2u[I(ji, jj)] + m->e2u[I(ji, jj + 1)]);
      double depe = 0.50 * (hu[I(ji, jj)] + sshn_u[I(ji, jj)] + hu[I(ji, jj + 1)] +
                            sshn_u[I(ji, jj + 1)]);

      double vv_s = (0.5 - fsign(0.5, v_s)) * vn[I(ji, jj)] + (0.5 + fsign(0.5, v_s)) * vn[I(ji, jj - 1)];
      double vv_n = (0.5 + fsign(0.5, v_n)) * vn[I(ji, jj)] + (0.5 - fsign(0.5, v_n)) * vn[I(ji, jj + 1)];
      double vv_w, vv_e;
      if (pt[I(ji - 1, jj)] <= 0 || pt[I(ji - 1, jj + 1)] <= 0)
        vv_w = (0.5 - fsign(0.5, u_w)) * vn[I(ji, jj)];
      else
        vv_w = (0.5 - fsign(0.5, u_w)) * vn[I(ji, jj)] + (0.5 + fsign(0.5, u_w)) * vn[I(ji - 1, jj)];
      if (pt[I(ji + 1, jj)] <= 0 || pt[I(ji + 1, jj + 1)] <= 0)
        vv_e = (0.5 + fsign(0.5, u_e)) * vn[I(ji, jj)];
      else
        vv_e = (0.5 + fsign(0.5, u_e)) * vn[I(ji, jj)] + (0.5 - fsign(0.5, u_e)) * vn[I(ji + 1, jj)];

      double adv = vv_w * u_w * depw - vv_e * u_e * depe + vv_s * v_s * deps - vv_n * v_n * depn;

      double dvdy_n = (vn[I(ji, jj + 1)] - vn[I(ji, jj)]) / m->e2t[I(ji, jj + 1)] *
                      (ht[I(ji, jj + 1)] + sshn[I(ji, jj + 1)]);
      double dvdy_s = (vn[I(ji, jj)] - vn[I(ji, jj - 1)]) / m->e2t[I(ji, jj)] *
                      (ht[I(ji, jj)] + sshn[I(ji, jj)]);
      double dvdx_w, dvdx_e;
      if (pt[I(ji - 1, jj)] <= 0 || pt[I(ji - 1, jj + 1)] <= 0)
        dvdx_w = 0.0;
      else
        dvdx_w = (vn[I(ji, jj)] - vn[I(ji - 1, jj)]) / (m->e1v[I(ji, jj)] + m->e1v[I(ji - 1, jj)]) *
                 (hv[I(ji, jj)] + sshn_v[I(ji, jj)] + hv[I(ji - 1, jj)] + sshn_v[I(ji - 1, jj)]);
      if (pt[I(ji + 1, jj)] <= 0 || pt[I(ji + 1, jj + 1)] <= 0)
        dvdx_e = 0.0;
      else
        dvdx_e = (vn[I(ji + 1, jj)] - vn[I(ji, jj)]) / (m->e1v[I(ji, jj)] + m->e1v[I(ji + 1, jj)]) *
                 (hv[I(ji, jj)] + sshn_v[I(ji, jj)] + hv[I(ji + 1, jj)] + sshn_v[I(ji + 1, jj)]);

      double vis = (dvdy_n - dvdy_s) * m->e1v[I(ji, jj)] + (dvdx_e - dvdx_w) * m->e2v[I(ji, jj)] * 0.5;
      vis = visc * vis;

      double cor = -0.5 * (2.0 * OMEGA * sin(m->gphiv[I(ji, jj)] * d2r) * (u_ec + u_wc)) *
                   m->e12v[I(ji, jj)] * (hv[I(ji, jj)] + sshn_v[I(ji, jj)]);
      double hpg = -(G * (hv[I(ji, jj)] + sshn_v[I(ji, jj)]) * m->e1v[I(ji, jj)] *
                     (sshn[I(ji, jj + 1)] - sshn[I(ji, jj)]));

      m->va[I(ji, jj)] = (vn[I(ji, jj)] * (hv[I(ji, jj)] + sshn_v[I(ji, jj)]) +
                          rdt * (adv + vis + cor + hpg) / m->e12v[I(ji, jj)]) /
                         ((hv[I(ji, jj)] + m->ssha_v[I(ji, jj)])) / (1.0 + cbfr * rdt);
    }
}

void oracle_momentum(oracle_model* m) {
  oracle_momentum_u(m);
  oracle_momentum_v(m);
}

/* bc: clamped SSH, original/nemolite2d.f90:629-644.  The tidal amplitude and
 * phase are parameters (reference: 0.2 and 0). */
void oracle_bc_ssh(oracle_model* m, double rtime) {
  const int jpi = m->jpi, jpj = m->jpj;
  const int* pt = m->pt;
  double amp_tide = m->p.amp_tide;
  double omega_tide = 2.0 * 3.14159 / (12.42 * 3600.0);
  double val = amp_tide * sin(omega_tide * rtime + m->p.tide_phase);
  for (int jj = 1; jj <= jpj; ++jj)
    for (int ji = 1; ji <= jpi; ++ji) {
      if (pt[I(ji, jj)] <= 0) continue;
      if (pt[I(ji, jj - 1)] < 0)
        m->ssha[I(ji, jj)] = val;
      else if (pt[I(ji, jj + 1)] < 0)
        m->ssha[I(ji, jj)] = val;
      else if (pt[I(ji + 1, jj)] < 0)
        m->ssha[I(ji, jj)] = val;
      else if (pt[I(ji - 1, jj)] < 0)
        m->ssha[I(ji, jj)] = val;
    }
}

/* bc: solid u, :648-652 */
void oracle_bc_solid_u(oracle_model* m) {
  const int jpi = m->jpi, jpj = m->jpj;
  for (int jj = 1; jj <= jpj; ++jj)
    for (int ji = 0; ji <= jpi; ++ji)
      if (m->pt[I(ji, jj)] * m->pt[I(ji + 1, jj)] == 0) m->ua[I(ji, jj)] = 0.0;
}

/* bc: solid v, :656-660 */
void oracle_bc_solid_v(oracle_model* m) {
  const int jpi = m->jpi, jpj = m->jpj;
  for (int jj = 0; jj <= jpj; ++jj)
    for (int ji = 1; ji <= jpi; ++ji)
      if (m->pt[I(ji, jj)] * m->pt[I(ji, jj + 1)] == 0) m->va[I(ji, jj)] = 0.0;
}

/* bc: Flather u, :669-680 (sequential in-place sweep) */
void oracle_bc_flather_u(oracle_model* m) {
  const int jpi = m->jpi, jpj = m->jpj;
  for (int jj = 1; jj <= jpj; ++jj)
    for (int ji = 0; ji <= jpi; ++ji) {
      if (m->pt[I(ji, jj)] + m->pt[I(ji + 1, jj)] <= -1) continue;
      if (m->pt[I(ji, jj)] < 0) {
        int jiu = ji + 1;
        m->ua[I(ji, jj)] = m->ua[I(jiu, jj)] +
                           sqrt(G / m->hu[I(ji, jj)]) * (m->sshn_u[I(ji, jj)] - m->sshn_u[I(jiu, jj)]);
      } else if (m->pt[I(ji + 1, jj)] < 0) {
        int jiu = ji - 1;
        m->ua[I(ji, jj)] = m->ua[I(jiu, jj)] +
                           sqrt(G / m->hu[I(ji, jj)]) * (m->sshn_u[I(ji, jj)] - m->sshn_u[I(jiu, jj)]);
      }
    }
}

/* bc: Flather v, :684-695 */
void oracle_bc_flather_v(oracle_model* m) {
  const int jpi = m->jpi, jpj = m->jpj;
  for (int jj = 0; jj <= jpj; ++jj)
    for (int ji = 1; ji <= jpi; ++ji) {
      if (m->pt[I(ji, jj)] + m->pt[I(ji, jj + 1)] <= -1) continue;
      if (m->pt[I(ji, jj)] < 0) {
        int jiv = jj + 1;
        m->va[I(ji, jj)] = m->va[I(ji, jiv)] +
                           sqrt(G / m->hv[I(ji, jj)]) * (m->sshn_v[I(ji, jj)] - m->sshn_v[I(ji, jiv)]);
      } else if (m->pt[I(ji, jj + 1)] < 0) {
        int jiv = jj - 1;
        m->va[I(ji, jj)] = m->va[I(ji, jiv)] +
                           sqrt(G / m->hv[I(ji, jj)]) * (m->sshn_v[I(ji, jj)] - m->sshn_v[I(ji, jiv)]);
      }
    }
}

void oracle_bc(oracle_model* m, double rtime) {
  oracle_bc_ssh(m, rtime);
  oracle_bc_solid_u(m);
  oracle_bc_solid_v(m);
  oracle_bc_flather_u(m);
  oracle_bc_flather_v(m);
}

static void derive_sshn_uv(oracle_model* m) {
  const int jpi = m->jpi, jpj = m->jpj;
  const int* pt = m->pt;
  /* sshn_u, :736-748 */
#pragma omp parallel for num_threads(g_threads) if (g_threads > 1) schedule(static)
  for (int jj = 1; jj <= jpj; ++jj)
    for (int ji = 0; ji <= jpi; ++ji) {
      if (pt[I(ji, jj)] + pt[I(ji + 1, jj)] <= 0) continue;
      if (pt[I(ji, jj)] * pt[I(ji + 1, jj)] > 0) {
        double r = m->e12t[I(ji, jj)] * m->sshn[I(ji, jj)] + m->e12t[I(ji + 1, jj)] * m->sshn[I(ji + 1, jj)];
        m->sshn_u[I(ji, jj)] = 0.5 * r / m->e12u[I(ji, jj)];
      } else if (pt[I(ji, jj)] <= 0) {
        m->sshn_u[I(ji, jj)] = m->sshn[I(ji + 1, jj)];
      } else if (pt[I(ji + 1, jj)] <= 0) {
        m->sshn_u[I(ji, jj)] = m->sshn[I(ji, jj)];
      }
    }
  /* sshn_v, :752-764 */
#pragma omp parallel for num_threads(g_threads) if (g_threads > 1) schedule(static)
  for (int jj = 0; jj <= jpj; ++jj)
    for (int ji = 1; ji <= jpi; ++ji) {
      if (pt[I(ji, jj)] + pt[I(ji, jj + 1)] <= 0) continue;
      if (pt[I(ji, jj)] * pt[I(ji, jj + 1)] > 0) {
        double r = m->e12t[I(ji, jj)] * m->sshn[I(ji, jj)] + m->e12t[I(ji, jj + 1)] * m->sshn[I(ji, jj + 1)];
        m->sshn_v[I(ji, jj)] = 0.5 * r / m->e12v[I(ji, jj)];
      } else if (pt[I(ji, jj)] <= 0) {
        m->sshn_v[I(ji, jj)] = m->sshn[I(ji, jj + 1)];
      } else if (pt[I(ji, jj + 1)] <= 0) {
        m->sshn_v[I(ji, jj)] = m->sshn[I(ji, jj)];
      }
    }
}

/* next, original/nemolite2d.f90:712-764 */
void oracle_next(oracle_model* m) {
  const int jpi = m->jpi, jpj = m->jpj;
#pragma omp parallel for num_threads(g_threads) if (g_threads > 1) schedule(static)
  for (int jj = 1; jj <= jpj; ++jj)
    for (int ji = 0; ji <= jpi; ++ji) m->un[I(ji, jj)] = m->ua[I(ji, jj)];
#pragma omp parallel for num_threads(g_threads) if (g_threads > 1) schedule(static)
  for (int jj = 0; jj <= jpj; ++jj)
    for (int ji = 1; ji <= jpi; ++ji) m->vn[I(ji, jj)] = m->va[I(ji, jj)];
#pragma omp parallel for num_threads(g_threads) if (g_threads > 1) schedule(static)
  for (int jj = 1; jj <= jpj; ++jj)
    for (int ji = 1; ji <= jpi; ++ji) m->sshn[I(ji, jj)] = m->ssha[I(ji, jj)];
  derive_sshn_uv(m);
}

/* step, original/nemolite2d.f90:375-386 (output handled by callers). */
void oracle_step(oracle_model* m, int istp) {
  double rtime = (double)istp * m->p.rdt;
  oracle_continuity(m);
  oracle_momentum(m);
  oracle_bc(m, rtime);
  oracle_next(m);
}

void oracle_run(oracle_model* m, int istp0, int nsteps) {
  for (int k = 0; k < nsteps; ++k) oracle_step(m, istp0 + k);
}

/* ---- field access -------------------------------------------------------- */
static const double* field_ptr(const oracle_model* m, int f, int* i0, int* i1,
                               int* j0, int* j1) {
  const int jpi = m->jpi, jpj = m->jpj;
  *i0 = 1; *i1 = jpi; *j0 = 1; *j1 = jpj;
  switch (f) {
    case ORC_SSHN: return m->sshn;
    case ORC_SSHA: return m->ssha;
    case ORC_HT: return m->ht;
    case ORC_XT: return m->xt;
    case ORC_YT: return m->yt;
    case ORC_UN: *i0 = 0; return m->un;
    case ORC_UA: *i0 = 0; return m->ua;
    case ORC_SSHN_U: *i0 = 0; return m->sshn_u;
    case ORC_HU: *i0 = 0; return m->hu;
    case ORC_VN: *j0 = 0; return m->vn;
    case ORC_VA: *j0 = 0; return m->va;
    case ORC_SSHN_V: *j0 = 0; return m->sshn_v;
    case ORC_HV: *j0 = 0; return m->hv;
    default: return 0;
  }
}

long oracle_get_field(const oracle_model* m, int field, double* out) {
  int i0, i1, j0, j1;
  const double* a = field_ptr(m, field, &i0, &i1, &j0, &j1);
  if (!a) return -1;
  long k = 0;
  for (int jj = j0; jj <= j1; ++jj)
    for (int ji = i0; ji <= i1; ++ji) out[k++] = a[I(ji, jj)];
  return k;
}

int oracle_set_state(oracle_model* m, const double* sshn, const double* un,
                     const double* vn) {
  const int jpi = m->jpi, jpj = m->jpj;
  long k = 0;
  for (int jj = 1; jj <= jpj; ++jj)
    for (int ji = 1; ji <= jpi; ++ji) m->sshn[I(ji, jj)] = sshn[k++];
  k = 0;
  for (int jj = 1; jj <= jpj; ++jj)
    for (int ji = 0; ji <= jpi; ++ji) m->un[I(ji, jj)] = un[k++];
  k = 0;
  for (int jj = 0; jj <= jpj; ++jj)
    for (int ji = 1; ji <= jpi; ++ji) m->vn[I(ji, jj)] = vn[k++];
  /* the state as after a complete step, where `next` (:712-732) has made the
   * after-step fields equal to the current ones */
  for (int jj = 1; jj <= jpj; ++jj)
    for (int ji = 1; ji <= jpi; ++ji) m->ssha[I(ji, jj)] = m->sshn[I(ji, jj)];
  for (int jj = 1; jj <= jpj; ++jj)
    for (int ji = 0; ji <= jpi; ++ji) m->ua[I(ji, jj)] = m->un[I(ji, jj)];
  for (int jj = 0; jj <= jpj; ++jj)
    for (int ji = 1; ji <= jpi; ++ji) m->va[I(ji, jj)] = m->vn[I(ji, jj)];
  derive_sshn_uv(m);
  return 0;
}

int oracle_set_grid(oracle_model* m, const int* pt, const double* e1t, const double* e2t,
                    const double* e1u, const double* e2u, const double* e1v, const double* e2v,
                    const double* gphiu, const double* gphiv, const double* ht, const double* hu,
                    const double* hv) {
  const size_t n = (size_t)(m->jpi + 2) * (m->jpj + 2);
  for (size_t k = 0; k < n; ++k)
    if (pt[k] < -1 || pt[k] > 1) return -1;
  memcpy(m->pt, pt, n * sizeof(int));
  const double* src[] = {e1t, e2t, e1u, e2u, e1v, e2v, gphiu, gphiv, ht, hu, hv};
  double* dst[] = {m->e1t, m->e2t, m->e1u, m->e2u, m->e1v, m->e2v, m->gphiu, m->gphiv, m->ht, m->hu, m->hv};
  for (int k = 0; k < 11; ++k)
    if (src[k]) memcpy(dst[k], src[k], n * sizeof(double));
  cell_areas(m);
  init_sshn_uv(m);
  return 0;
}

/* ---- checksums ----------------------------------------------------------- */
double oracle_checksum_seq(const oracle_model* m, int field) {
  int i0, i1, j0, j1;
  const double* a = field_ptr(m, field, &i0, &i1, &j0, &j1);
  if (!a) return NAN;
  double s = 0.0;
  for (int jj = 1; jj <= m->jpj; ++jj)
    for (int ji = 1; ji <= m->jpi; ++ji) s = s + fabs(a[I(ji, jj)]);
  return s;
}

/* Fixed reduction order of the device checksum: a 256-wide strided partial
 * per lane (ascending index), then an xor butterfly over 32 lanes (offsets
 * 16..1) and over the 8 warp results (offsets 4..1).  Applied to each row,
 * then to the column of row sums. */
#define CK_THREADS 256
static double block_reduce(const double* v, long n, long stride) {
  double lane[CK_THREADS];
  for (int t = 0; t < CK_THREADS; ++t) {
    double acc = 0.0;
    for (long k = t; k < n; k += CK_THREADS) acc = acc + v[k * stride];
    lane[t] = acc;
  }
  double warp[CK_THREADS / 32];
  for (int w = 0; w < CK_THREADS / 32; ++w) {
    double x[32], y[32];
    for (int l = 0; l < 32; ++l) x[l] = lane[w * 32 + l];
    for (int off = 16; off >= 1; off >>= 1) {
      for (int l = 0; l < 32; ++l) y[l] = x[l] + x[l ^ off];
      for (int l = 0; l < 32; ++l) x[l] = y[l];
    }
    warp[w] = x[0];
  }
  double x[8], y[8];
  for (int l = 0; l < 8; ++l) x[l] = warp[l];
  for (int off = 4; off >= 1; off >>= 1) {
    for (int l = 0; l < 8; ++l) y[l] = x[l] + x[l ^ off];
    for (int l = 0; l < 8; ++l) x[l] = y[l];
  }
  return x[0];
}

double oracle_tree_sum_abs(const double* a, int nx, int ny, int ld) {
  double* rows = (double*)malloc(sizeof(double) * (size_t)(ny > 0 ? ny : 1));
  double* absrow = (double*)malloc(sizeof(double) * (size_t)(nx > 0 ? nx : 1));
  for (int j = 0; j < ny; ++j) {
    for (int i = 0; i < nx; ++i) absrow[i] = fabs(a[(long)j * ld + i]);
    rows[j] = block_reduce(absrow, nx, 1);
  }
  double s = block_reduce(rows, ny, 1);
  free(rows);
  free(absrow);
  return s;
}

double oracle_checksum_tree(const oracle_model* m, int field) {
  int i0, i1, j0, j1;
  const double* a = field_ptr(m, field, &i0, &i1, &j0, &j1);
  if (!a) return NAN;
  /* region (1:jpi,1:jpj) of the superset array */
  return oracle_tree_sum_abs(a + I(1, 1), m->jpi, m->jpj, m->ld);
}
