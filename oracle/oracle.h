/*
 * CPU oracle for the NEMOLite2D time-stepper.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the serial
 * Fortran model original/nemolite2d.f90 (routines setup..finalisation,
 * lines 96-830).  Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / reference legs may load it, and only as the checker or the
 * timed CPU baseline.  The product library never links or calls it.
 *
 * Parity pin: the restatement is checked bit-for-bit against golden vectors
 * produced by executing the reference's own Fortran source text
 * (tests/golden/make_golden.py translates original/nemolite2d.f90 routine by
 * routine and runs it in IEEE double, left to right, no contraction).
 *
 * Layout: every 2-D array is stored over the superset index range
 * (0:jpi+1, 0:jpj+1), column-major (ji fastest), so each Fortran array with
 * bounds (1:jpi,1:jpj), (0:jpi,1:jpj) or (1:jpi,0:jpj) is addressed with its
 * own Fortran indices.
 */
#ifndef NEMO_ORACLE_H
#define NEMO_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Field identifiers; identical numbering to the product's C ABI. */
enum {
  ORC_SSHN = 0, ORC_UN = 1, ORC_VN = 2,
  ORC_SSHA = 3, ORC_UA = 4, ORC_VA = 5,
  ORC_SSHN_U = 6, ORC_SSHN_V = 7,
  ORC_HT = 8, ORC_HU = 9, ORC_HV = 10,
  ORC_XT = 11, ORC_YT = 12
};

typedef struct oracle_params {
  /* &namctl keys, original/nemolite2d.f90:100-118 (jpi/jpj already reduced
   * by 2 as setup does at :133-137). */
  int jpi, jpj;
  double dx, dy, dep_const;
  int nit000, nitend, irecord;
  double rdt, cbfr, visc;
  /* Extensions.  Defaults reproduce the reference exactly. */
  double amp_tide;   /* original/nemolite2d.f90:629 hard-codes 0.2 */
  double tide_phase; /* 0: sin(omega_tide*rtime) */
  double lat;        /* gphiu/gphiv latitude, :220-222 hard-codes 50 */
  int nbump;         /* 0: uniform depth dep_const (:238-254) */
  uint64_t seed;
  double bump_amp, bump_wmin, bump_wmax, hmin, hmax;
} oracle_params;

typedef struct oracle_model oracle_model;

void oracle_default_params(oracle_params* p);
void oracle_set_threads(int n);
int oracle_get_threads(void);

/* grid + allocation + initialisation (original/nemolite2d.f90:145-371). */
oracle_model* oracle_create(const oracle_params* p);
void oracle_destroy(oracle_model* m);

/* The four per-step routines, original/nemolite2d.f90:390-769. */
void oracle_continuity(oracle_model* m);
void oracle_momentum(oracle_model* m);
void oracle_momentum_u(oracle_model* m);
void oracle_momentum_v(oracle_model* m);
void oracle_bc(oracle_model* m, double rtime);
void oracle_bc_ssh(oracle_model* m, double rtime);
void oracle_bc_solid_u(oracle_model* m);
void oracle_bc_solid_v(oracle_model* m);
void oracle_bc_flather_u(oracle_model* m);
void oracle_bc_flather_v(oracle_model* m);
void oracle_next(oracle_model* m);
/* step (:375-386) without output: rtime = istp*rdt, then the four routines. */
void oracle_step(oracle_model* m, int istp);
void oracle_run(oracle_model* m, int istp0, int nsteps);

/* Copy a field's Fortran-bounded region into a dense column-major array.
 * Extents: T (jpi,jpj), U (jpi+1,jpj), V (jpi,jpj+1).  Returns count or -1. */
long oracle_get_field(const oracle_model* m, int field, double* out);
/* Replace sshn/un/vn (dense, same extents), set ssha/ua/va to the same
 * values (the state as after a complete step, where `next` has copied them,
 * :712-732) and re-derive sshn_u/sshn_v with the post-`next` interpolation
 * (:736-764). */
int oracle_set_state(oracle_model* m, const double* sshn, const double* un,
                     const double* vn);

/* Replace the grid of original/nemolite2d.f90's `grid` routine (:145-281)
 * by general arrays, each over (0:jpi+1, 0:jpj+1), column-major, ld jpi+2:
 * the mask pt (1 water, 0 land, -1 open water outside the domain), the scale
 * factors e1t..e2v, the latitudes gphiu/gphiv (degrees) and, when not NULL,
 * the depths ht/hu/hv.  The cell areas are re-formed over the ranges :263-279
 * fill (zero elsewhere, as allocated), and sshn_u/sshn_v are re-initialised
 * from the current sshn (:337-353).  Returns -1 for a pt value outside
 * {-1, 0, 1}. */
int oracle_set_grid(oracle_model* m, const int* pt, const double* e1t, const double* e2t,
                    const double* e1u, const double* e2u, const double* e1v, const double* e2v,
                    const double* gphiu, const double* gphiv, const double* ht, const double* hu,
                    const double* hv);

/* SUM(ABS(f(1:jpi,1:jpj))) in the reference's column-major order
 * (field_mod.f90:951). */
double oracle_checksum_seq(const oracle_model* m, int field);
/* The same sum in the device checksum kernel's fixed reduction order. */
double oracle_checksum_tree(const oracle_model* m, int field);
/* Tree order over an arbitrary dense (nx,ny) column-major array. */
double oracle_tree_sum_abs(const double* a, int nx, int ny, int ld);

int oracle_jpi(const oracle_model* m);
int oracle_jpj(const oracle_model* m);

#ifdef __cplusplus
}
#endif
#endif
