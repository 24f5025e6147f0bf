// C ABI of the NEMOLite2D stepper: context lifecycle, the per-routine
// boundary, the fused path, checksums and field copies, plus the drop-in
// cuda_*_ symbols of the reference library (cuda/cuda_nemolite2d.cu:234-270).
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <atomic>
#include <cmath>
#include <fstream>
#include <new>
#include <sstream>
#include <string>
#include <vector>

#include "nemo_internal.h"

using namespace nemo;

struct nemo_ctx {
  nemo_params p;
  Layout L;
  Consts C;
  int device;
  cudaStream_t stream;
  bool own_stream;
  double* slab;
  StateSet set[2];
  int n_idx;              // set[n_idx] holds sshn/un/vn, set[1-n_idx] ssha/ua/va
  double *sshn_u, *sshn_v, *ht, *hu, *hv;
  double *rhu, *rhv;      // RN(1/hu), RN(1/hv) for the fused step
  double* ck_partials;    // 4*jpj
  double* ck_out;         // 4
  double* ck_host;        // pinned, 4
  bool a_mirrors_n;       // after a fused step the reference's a-fields equal n
  bool uv_stale;          // stored sshn_u/sshn_v lag behind sshn
  bool recip_nr_ok;       // in-kernel reciprocal depths equal the stored ones
  nemo_schedule sched;
  // general grid (nemo_set_grid): mask and metrics on the device; the
  // routine kernels read them and steps run the routine sequence
  bool general = false;
  void* gslab = nullptr;
  GridDev grid{};
  int4* gchains = nullptr;   // Flather chains of the general grid
  int n_gchains = 0;
  // the general grid's fused kernel: warps 2, occupancy = ring slots (0, 3, 4),
  // rows per CTA
  nemo_schedule gsched{2, 3, 32};
  // output records (nemo_record): staging buffer, side stream and events
  double* rec_dev = nullptr;
  cudaStream_t rec_stream = nullptr;
  cudaEvent_t rec_state = nullptr, rec_staged = nullptr, rec_copied = nullptr;
};

namespace {

#define CK(call)                                     \
  do {                                               \
    cudaError_t e_ = (call);                         \
    if (e_ != cudaSuccess) return status_from(e_);   \
  } while (0)

int status_from(cudaError_t e) {
  if (e == cudaSuccess) return NEMO_OK;
  if (e == cudaErrorMemoryAllocation) return NEMO_ERR_ALLOC;
  return NEMO_ERR_CUDA;
}

int set_device(nemo_ctx* c) {
  if (c->device >= 0) CK(cudaSetDevice(c->device));
  return NEMO_OK;
}

const GridDev* gridp(const nemo_ctx* c) { return c->general ? &c->grid : nullptr; }

StateSet& nset(nemo_ctx* c) { return c->set[c->n_idx]; }
StateSet& aset(nemo_ctx* c) { return c->set[1 - c->n_idx]; }

RoutinePtrs rptrs(nemo_ctx* c) {
  RoutinePtrs r;
  r.sshn = nset(c).ssh;
  r.un = nset(c).u;
  r.vn = nset(c).v;
  r.ssha = aset(c).ssh;
  r.ua = aset(c).u;
  r.va = aset(c).v;
  r.sshn_u = c->sshn_u;
  r.sshn_v = c->sshn_v;
  r.ht = c->ht;
  r.hu = c->hu;
  r.hv = c->hv;
  return r;
}

size_t field_bytes(const Layout& L) { return (size_t)L.elems() * sizeof(double); }

// Before a per-routine kernel: bring stored sshn_u/sshn_v up to date, and
// materialise the a-fields if the last step was fused.
int prepare_routine(nemo_ctx* c, bool writes_a) {
  if (c->uv_stale) {
    CK(launch_derive_sshn_uv(c->L, c->C, nset(c).ssh, c->sshn_u, c->sshn_v, c->stream, gridp(c)));
    c->uv_stale = false;
  }
  if (writes_a && c->a_mirrors_n) {
    size_t b = field_bytes(c->L);
    CK(cudaMemcpyAsync(aset(c).ssh, nset(c).ssh, b, cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(aset(c).u, nset(c).u, b, cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(aset(c).v, nset(c).v, b, cudaMemcpyDeviceToDevice, c->stream));
    c->a_mirrors_n = false;
  }
  return NEMO_OK;
}

// Fortran bounds of each field: x from i0 (nx points), y from j0 (ny points).
bool field_window(const nemo_ctx* c, int f, int* i0, int* nx, int* j0, int* ny) {
  const int jpi = c->L.jpi, jpj = c->L.jpj;
  *i0 = 1; *nx = jpi; *j0 = 1; *ny = jpj;
  switch (f) {
    case NEMO_SSHN: case NEMO_SSHA: case NEMO_HT: case NEMO_XT: case NEMO_YT: return true;
    case NEMO_UN: case NEMO_UA: case NEMO_SSHN_U: case NEMO_HU: *i0 = 0; *nx = jpi + 1; return true;
    case NEMO_VN: case NEMO_VA: case NEMO_SSHN_V: case NEMO_HV: *j0 = 0; *ny = jpj + 1; return true;
    default: return false;
  }
}

double* field_storage(nemo_ctx* c, int f) {
  switch (f) {
    case NEMO_SSHN: return nset(c).ssh;
    case NEMO_UN: return nset(c).u;
    case NEMO_VN: return nset(c).v;
    case NEMO_SSHA: return c->a_mirrors_n ? nset(c).ssh : aset(c).ssh;
    case NEMO_UA: return c->a_mirrors_n ? nset(c).u : aset(c).u;
    case NEMO_VA: return c->a_mirrors_n ? nset(c).v : aset(c).v;
    case NEMO_SSHN_U: return c->sshn_u;
    case NEMO_SSHN_V: return c->sshn_v;
    case NEMO_HT: return c->ht;
    case NEMO_HU: return c->hu;
    case NEMO_HV: return c->hv;
    default: return nullptr;
  }
}

bool valid_params(const nemo_params* p) {
  if (!p) return false;
  if (p->jpi < 2 || p->jpj < 2 || p->jpi > (1 << 17) || p->jpj > (1 << 17)) return false;
  if (!(p->dx > 0.0) || !(p->dy > 0.0) || !(p->rdt > 0.0)) return false;
  if (p->nbump < 0 || p->nbump > 4096) return false;
  if (p->nbump > 0 && !(p->bump_wmin > 0.0 && p->bump_wmax >= p->bump_wmin)) return false;
  return true;
}

}  // namespace

namespace nemo {

Consts make_consts(const nemo_params& p) {
  Consts C;
  // original/nemolite2d.f90:210-217 (uniform grid) and :263-279 (areas)
  C.e1t = C.e1u = C.e1v = p.dx;
  C.e2t = C.e2u = C.e2v = p.dy;
  C.e12t = C.e1t * C.e2t;
  C.e12u = C.e1u * C.e2u;
  C.e12v = C.e1v * C.e2v;
  C.two_dx = C.e1v + C.e1v;
  C.two_dy = C.e2u + C.e2u;
  C.rdt = p.rdt;
  C.visc = p.visc;
  C.g = kG;
  const double d2r = kPi / 180.0;
  C.fcor = 2.0 * kOmega * sin(p.lat * d2r);
  C.cfric = 1.0 + p.cbfr * p.rdt;
  C.r_e1t = 1.0 / C.e1t;
  C.r_e2t = 1.0 / C.e2t;
  C.r_e12t = 1.0 / C.e12t;
  C.r_e12u = 1.0 / C.e12u;
  C.r_e12v = 1.0 / C.e12v;
  C.r_2dx = 1.0 / C.two_dx;
  C.r_2dy = 1.0 / C.two_dy;
  C.r_cfric = 1.0 / C.cfric;
  C.r_cfric_lo = fma(-C.cfric, C.r_cfric, 1.0) / C.cfric;  // the residual is exact
  C.k_su = (0.5 * C.e12t) / C.e12u;
  C.k_sv = (0.5 * C.e12t) / C.e12v;
  C.h_e2t = 0.5 * C.e2t;
  C.h_e1t = 0.5 * C.e1t;
  C.e_2dy = 0.125 * C.two_dy;
  C.e_2dx = 0.125 * C.two_dx;
  C.k_ssh = C.rdt / C.e12t;
  C.k_u = C.rdt / C.e12u;
  C.k_v = C.rdt / C.e12v;
  C.vis_u1 = C.visc * C.e2u / C.e1t;
  C.vis_u2 = C.visc * (0.5 * C.e1u) / C.two_dy;
  C.vis_v1 = C.visc * C.e1v / C.e2t;
  C.vis_v2 = C.visc * (0.5 * C.e2v) / C.two_dx;
  C.cor_u = (0.25 * C.fcor) * C.e12u;
  C.cor_v = -((0.25 * C.fcor) * C.e12v);
  C.hpg_u = -(C.g * C.e2u);
  C.hpg_v = -(C.g * C.e1v);
  return C;
}

// amp*sin(omega_tide*rtime + phase), omega_tide as original/nemolite2d.f90:630
double tide_value(const nemo_params& p, int istp) {
  const double omega_tide = 2.0 * 3.14159 / (12.42 * 3600.0);
  double rtime = (double)istp * p.rdt;
  return p.amp_tide * sin(omega_tide * rtime + p.tide_phase);
}

static double tide_at_time(const nemo_params& p, double rtime) {
  const double omega_tide = 2.0 * 3.14159 / (12.42 * 3600.0);
  return p.amp_tide * sin(omega_tide * rtime + p.tide_phase);
}

// Seeded Gaussian bumps: SplitMix64 (Steele, Lea & Flood 2014) draws centre,
// amplitude and width of each bump; each bump is separable and tabulated on
// the half-grid x_k = k*dx/2 with the host libm exp.
static uint64_t smix_next(uint64_t* s) {
  uint64_t z = (*s += 0x9E3779B97F4A7C15ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
static double smix_unif(uint64_t* s) { return (double)(smix_next(s) >> 11) * 0x1.0p-53; }

void depth_tables(const nemo_params& p, double* ax, double* gy) {
  const int nkx = 2 * p.jpi + 2, nky = 2 * p.jpj + 2;
  uint64_t s = p.seed;
  const double lx = (double)p.jpi * p.dx, ly = (double)p.jpj * p.dy;
  const double hdx = 0.5 * p.dx, hdy = 0.5 * p.dy;
  for (int b = 0; b < p.nbump; ++b) {
    double xc = smix_unif(&s) * lx;
    double yc = smix_unif(&s) * ly;
    double amp = p.bump_amp * (2.0 * smix_unif(&s) - 1.0);
    double w = p.bump_wmin + (p.bump_wmax - p.bump_wmin) * smix_unif(&s);
    for (int k = 0; k < nkx; ++k) {
      double t = ((double)k * hdx - xc) / w;
      ax[(size_t)b * nkx + k] = amp * exp(-(t * t));
    }
    for (int k = 0; k < nky; ++k) {
      double t = ((double)k * hdy - yc) / w;
      gy[(size_t)b * nky + k] = exp(-(t * t));
    }
  }
}

}  // namespace nemo

// ---- schedule cache (NEMO_TUNE_CACHE) ---------------------------------------
// One line per (GPU, grid): "<gpu>:<jpi>x<jpj> warps occupancy rows ms".
namespace {

std::string tune_key(const nemo_ctx* c) {
  cudaDeviceProp prop;
  int dev = 0;
  cudaGetDevice(&dev);
  std::string name = "gpu";
  if (cudaGetDeviceProperties(&prop, dev) == cudaSuccess) name = prop.name;
  for (auto& ch : name)
    if (ch == ' ' || ch == ':') ch = '_';
  std::ostringstream k;
  k << name << ":" << c->L.jpi << "x" << c->L.jpj;
  return k.str();
}

bool tune_lookup(const nemo_ctx* c, nemo_schedule* s) {
  const char* path = getenv("NEMO_TUNE_CACHE");
  if (!path || !*path) return false;
  std::ifstream f(path);
  if (!f) return false;
  const std::string key = tune_key(c);
  std::string line;
  bool found = false;
  while (std::getline(f, line)) {
    std::istringstream ls(line);
    std::string k;
    nemo_schedule t;
    double ms;
    if (ls >> k >> t.warps >> t.occupancy >> t.rows >> ms && k == key &&
        fused_variant_ok(t.warps, t.occupancy, c->recip_nr_ok)) {
      *s = t;
      found = true;  // the last entry for a key wins
    }
  }
  return found;
}

void tune_store(const nemo_ctx* c, const nemo_schedule& s, double ms) {
  const char* path = getenv("NEMO_TUNE_CACHE");
  if (!path || !*path) return;
  std::ofstream f(path, std::ios::app);
  if (f) f << tune_key(c) << " " << s.warps << " " << s.occupancy << " " << s.rows << " " << ms << "\n";
}

}  // namespace

namespace nemo {
// Countdown of nemo_debug_fail_alloc: 0 is off; n > 0 makes the n-th
// allocation from now fail.
static std::atomic<int> g_alloc_countdown{0};

bool alloc_should_fail() {
  int c = g_alloc_countdown.load(std::memory_order_relaxed);
  while (c > 0) {
    if (g_alloc_countdown.compare_exchange_weak(c, c - 1, std::memory_order_relaxed)) return c == 1;
  }
  return false;
}
}  // namespace nemo

extern "C" {

int nemo_default_params(nemo_params* p) {
  if (!p) return NEMO_ERR_INVALID;
  memset(p, 0, sizeof(*p));
  // original/nemolite2d.f90:107-118 (jpiglo = jpjglo = 258)
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
  p->stream = nullptr;
  p->device = -1;
  return NEMO_OK;
}

int nemo_destroy(nemo_ctx* c) {
  if (!c) return NEMO_ERR_INVALID;
  if (c->device >= 0) cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->rec_stream) cudaStreamSynchronize(c->rec_stream);
  if (c->slab) cudaFree(c->slab);
  if (c->ck_host) cudaFreeHost(c->ck_host);
  if (c->rec_dev) cudaFree(c->rec_dev);
  if (c->rec_state) cudaEventDestroy(c->rec_state);
  if (c->rec_staged) cudaEventDestroy(c->rec_staged);
  if (c->rec_copied) cudaEventDestroy(c->rec_copied);
  if (c->rec_stream) cudaStreamDestroy(c->rec_stream);
  if (c->gslab) cudaFree(c->gslab);
  if (c->gchains) cudaFree(c->gchains);
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return NEMO_OK;
}

int nemo_create(const nemo_params* p, nemo_ctx** out) {
  if (!out) return NEMO_ERR_INVALID;
  *out = nullptr;
  if (!valid_params(p)) return NEMO_ERR_INVALID;
  nemo_ctx* c = new (std::nothrow) nemo_ctx();
  if (!c) return NEMO_ERR_ALLOC;
  c->p = *p;
  c->device = p->device;
  c->L.jpi = p->jpi;
  c->L.jpj = p->jpj;
  c->L.pitch = layout_pitch(p->jpi);
  c->L.rows = (long)p->jpj + 3;
  c->C = make_consts(*p);
  c->sched.warps = 2;
  c->sched.occupancy = 216;  // 116 when the depths fail the reciprocal check below
  c->sched.rows = 32;
  c->recip_nr_ok = false;
  int st = set_device(c);
  if (st) { delete c; return st; }
  cudaError_t e;
  if (p->stream) {
    c->stream = (cudaStream_t)p->stream;
    c->own_stream = false;
  } else {
    e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) { delete c; return status_from(e); }
    c->own_stream = true;
  }
  const size_t fe = (size_t)c->L.elems();
  const size_t ck = 4 * (size_t)p->jpj + 4;
  const size_t total = 13 * fe + ck;
  e = nemo::dev_alloc(&c->slab, total * sizeof(double));
  if (e != cudaSuccess) { c->slab = nullptr; nemo_destroy(c); cudaGetLastError(); return NEMO_ERR_ALLOC; }
  e = nemo::host_alloc(&c->ck_host, 4 * sizeof(double));
  if (e != cudaSuccess) { c->ck_host = nullptr; nemo_destroy(c); cudaGetLastError(); return NEMO_ERR_ALLOC; }
  double* q = c->slab;
  for (int s = 0; s < 2; ++s) {
    c->set[s].ssh = q; q += fe;
    c->set[s].u = q; q += fe;
    c->set[s].v = q; q += fe;
  }
  c->sshn_u = q; q += fe;
  c->sshn_v = q; q += fe;
  c->ht = q; q += fe;
  c->hu = q; q += fe;
  c->hv = q; q += fe;
  c->rhu = q; q += fe;
  c->rhv = q; q += fe;
  c->ck_partials = q; q += 4 * (size_t)p->jpj;
  c->ck_out = q;
  c->n_idx = 0;
  c->a_mirrors_n = false;
  c->uv_stale = false;

  // allocation (:310-318): everything starts at zero
  e = cudaMemsetAsync(c->slab, 0, total * sizeof(double), c->stream);
  if (e != cudaSuccess) { nemo_destroy(c); return status_from(e); }
  // grid: depth (:238-254 or seeded bumps)
  double* tab = nullptr;
  if (p->nbump > 0) {
    const size_t nax = (size_t)p->nbump * (2 * p->jpi + 2), ngy = (size_t)p->nbump * (2 * p->jpj + 2);
    std::vector<double> h(nax + ngy);
    depth_tables(*p, h.data(), h.data() + nax);
    e = nemo::dev_alloc(&tab, (nax + ngy) * sizeof(double));
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(tab, h.data(), (nax + ngy) * sizeof(double), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess)
      e = launch_depth(c->L, p->dep_const, p->nbump, tab, tab + nax, p->hmin, p->hmax, c->ht, c->hu, c->hv, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (tab) cudaFree(tab);
  } else {
    e = launch_depth(c->L, p->dep_const, 0, nullptr, nullptr, p->hmin, p->hmax, c->ht, c->hu, c->hv, c->stream);
  }
  // reciprocal depths, and whether recip_nr reproduces them on every cell
  // (the checksum scratch holds the mismatch count; it is not in use yet)
  int* d_bad = reinterpret_cast<int*>(c->ck_partials);
  int h_bad = -1;
  if (e == cudaSuccess) e = cudaMemsetAsync(d_bad, 0, sizeof(int), c->stream);
  if (e == cudaSuccess) e = launch_recip(c->L, c->hu, c->hv, c->rhu, c->rhv, d_bad, c->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h_bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  c->recip_nr_ok = (e == cudaSuccess && h_bad == 0);
  if (!c->recip_nr_ok) c->sched.occupancy = 116;
  // initialisation (:331-365): sshn = un = vn = 0, sshn_u/sshn_v averaged
  if (e == cudaSuccess)
    e = launch_init_sshn_uv(c->L, c->C, nset(c).ssh, c->sshn_u, c->sshn_v, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) { nemo_destroy(c); return status_from(e); }
  nemo_schedule cached;
  if (tune_lookup(c, &cached)) c->sched = cached;
  *out = c;
  return NEMO_OK;
}

int nemo_continuity(nemo_ctx* c) {
  if (!c) return NEMO_ERR_STATE;
  int st = set_device(c); if (st) return st;
  st = prepare_routine(c, true); if (st) return st;
  CK(launch_continuity(c->L, c->C, rptrs(c), c->stream, gridp(c)));
  return NEMO_OK;
}

int nemo_momentum_u(nemo_ctx* c) {
  if (!c) return NEMO_ERR_STATE;
  int st = set_device(c); if (st) return st;
  st = prepare_routine(c, true); if (st) return st;
  CK(launch_momentum_u(c->L, c->C, rptrs(c), c->stream, gridp(c)));
  return NEMO_OK;
}

int nemo_momentum_v(nemo_ctx* c) {
  if (!c) return NEMO_ERR_STATE;
  int st = set_device(c); if (st) return st;
  st = prepare_routine(c, true); if (st) return st;
  CK(launch_momentum_v(c->L, c->C, rptrs(c), c->stream, gridp(c)));
  return NEMO_OK;
}

int nemo_momentum(nemo_ctx* c) {
  int st = nemo_momentum_u(c);
  return st ? st : nemo_momentum_v(c);
}

int nemo_bc_ssh(nemo_ctx* c, double rtime) {
  if (!c) return NEMO_ERR_STATE;
  int st = set_device(c); if (st) return st;
  st = prepare_routine(c, true); if (st) return st;
  CK(launch_bc_ssh(c->L, tide_at_time(c->p, rtime), aset(c).ssh, c->stream, gridp(c)));
  return NEMO_OK;
}

int nemo_bc_solid_u(nemo_ctx* c) {
  if (!c) return NEMO_ERR_STATE;
  int st = set_device(c); if (st) return st;
  st = prepare_routine(c, true); if (st) return st;
  CK(launch_bc_solid_u(c->L, aset(c).u, c->stream, gridp(c)));
  return NEMO_OK;
}

int nemo_bc_solid_v(nemo_ctx* c) {
  if (!c) return NEMO_ERR_STATE;
  int st = set_device(c); if (st) return st;
  st = prepare_routine(c, true); if (st) return st;
  CK(launch_bc_solid_v(c->L, aset(c).v, c->stream, gridp(c)));
  return NEMO_OK;
}

int nemo_bc_flather_u(nemo_ctx* c) {
  if (!c) return NEMO_ERR_STATE;
  int st = set_device(c); if (st) return st;
  st = prepare_routine(c, true); if (st) return st;
  CK(launch_bc_flather_u(c->L, rptrs(c), c->stream, gridp(c)));
  return NEMO_OK;
}

int nemo_bc_flather_v(nemo_ctx* c) {
  if (!c) return NEMO_ERR_STATE;
  int st = set_device(c); if (st) return st;
  st = prepare_routine(c, true); if (st) return st;
  CK(launch_bc_flather_v(c->L, rptrs(c), c->stream, gridp(c)));
  return NEMO_OK;
}

int nemo_bc(nemo_ctx* c, double rtime) {
  int st;
  if ((st = nemo_bc_ssh(c, rtime))) return st;
  if ((st = nemo_bc_solid_u(c))) return st;
  if ((st = nemo_bc_solid_v(c))) return st;
  if ((st = nemo_bc_flather_u(c))) return st;
  return nemo_bc_flather_v(c);
}

int nemo_next(nemo_ctx* c) {
  if (!c) return NEMO_ERR_STATE;
  int st = set_device(c); if (st) return st;
  st = prepare_routine(c, true); if (st) return st;
  CK(launch_copy_next(c->L, rptrs(c), c->stream));
  CK(launch_derive_sshn_uv(c->L, c->C, nset(c).ssh, c->sshn_u, c->sshn_v, c->stream, gridp(c)));
  return NEMO_OK;
}

int nemo_step(nemo_ctx* c, int istp) {
  if (!c) return NEMO_ERR_STATE;
  double rtime = (double)istp * c->p.rdt;  // original/nemolite2d.f90:378
  int st;
  if ((st = nemo_continuity(c))) return st;
  if ((st = nemo_momentum(c))) return st;
  if ((st = nemo_bc(c, rtime))) return st;
  return nemo_next(c);
}

int nemo_step_n(nemo_ctx* c, int istp0, int n) {
  if (!c) return NEMO_ERR_STATE;
  if (n < 0) return NEMO_ERR_INVALID;
  if (n == 0) return NEMO_OK;
  int st = set_device(c); if (st) return st;
  if (c->general) {  // the general grid's fused kernel and its Flather chains
    for (int k = 0; k < n; ++k) {
      GenArgs a;
      a.sshn = nset(c).ssh;
      a.un = nset(c).u;
      a.vn = nset(c).v;
      a.ht = c->ht;
      a.hu = c->hu;
      a.hv = c->hv;
      a.su_st = c->sshn_u;
      a.sv_st = c->sshn_v;
      a.ssha = aset(c).ssh;
      a.ua = aset(c).u;
      a.va = aset(c).v;
      a.tide = tide_value(c->p, istp0 + k);
      a.g = c->grid;
      CK(launch_fused_general(c->L, c->C, a, c->gchains, c->n_gchains, c->gsched.occupancy, c->gsched.rows,
                              c->stream));
      c->n_idx = 1 - c->n_idx;
    }
    c->a_mirrors_n = true;
    c->uv_stale = true;
    return NEMO_OK;
  }
  for (int k = 0; k < n; ++k) {
    FusedArgs a;
    a.sshn = nset(c).ssh;
    a.un = nset(c).u;
    a.vn = nset(c).v;
    a.ht = c->ht;
    a.hu = c->hu;
    a.hv = c->hv;
    a.rhu = c->rhu;
    a.rhv = c->rhv;
    a.sshv0 = c->sshn_v;
    a.ssha = aset(c).ssh;
    a.ua = aset(c).u;
    a.va = aset(c).v;
    a.tide = tide_value(c->p, istp0 + k);
    CK(launch_fused_step(c->L, c->C, a, c->sched.warps, c->sched.occupancy, c->sched.rows,
                         c->stream));
    c->n_idx = 1 - c->n_idx;  // next: the new state becomes "now"
  }
  c->a_mirrors_n = true;
  c->uv_stale = true;
  return NEMO_OK;
}

int nemo_checksum(nemo_ctx* c, int field, double* out) {
  if (!c || !out) return NEMO_ERR_INVALID;
  double* f = field_storage(c, field);
  if (!f || field == NEMO_XT || field == NEMO_YT) return NEMO_ERR_INVALID;
  int st = set_device(c); if (st) return st;
  if ((field == NEMO_SSHN_U || field == NEMO_SSHN_V) && (st = prepare_routine(c, false))) return st;
  const double* fl[1] = {f};
  CK(launch_checksums(c->L, fl, 1, c->ck_partials, c->ck_out, c->stream));
  CK(cudaMemcpyAsync(c->ck_host, c->ck_out, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  *out = c->ck_host[0];
  return NEMO_OK;
}

int nemo_checksums(nemo_ctx* c, double out[3]) {
  if (!c || !out) return NEMO_ERR_INVALID;
  int st = set_device(c); if (st) return st;
  const double* fl[3] = {nset(c).ssh, nset(c).u, nset(c).v};
  CK(launch_checksums(c->L, fl, 3, c->ck_partials, c->ck_out, c->stream));
  CK(cudaMemcpyAsync(c->ck_host, c->ck_out, 3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  for (int k = 0; k < 3; ++k) out[k] = c->ck_host[k];
  return NEMO_OK;
}

int nemo_record(nemo_ctx* c, double* host) {
  if (!c || !host) return NEMO_ERR_INVALID;
  int st = set_device(c); if (st) return st;
  if (!c->rec_dev) {
    CK(nemo::dev_alloc(&c->rec_dev, 3 * (size_t)c->L.jpi * c->L.jpj * sizeof(double)));
    CK(cudaStreamCreateWithFlags(&c->rec_stream, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&c->rec_state, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&c->rec_staged, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&c->rec_copied, cudaEventDisableTiming));
  }
  // the staging kernel reads the state after the steps queued so far; the
  // context's stream waits only for that kernel, the copy overlaps later steps
  // (in stream order after the previous record's copy, so the buffer is free)
  CK(cudaEventRecord(c->rec_state, c->stream));
  CK(cudaStreamWaitEvent(c->rec_stream, c->rec_state, 0));
  CK(launch_record(c->L, nset(c).ssh, nset(c).u, nset(c).v, c->rec_dev, c->rec_stream));
  CK(cudaEventRecord(c->rec_staged, c->rec_stream));
  CK(cudaStreamWaitEvent(c->stream, c->rec_staged, 0));
  CK(cudaMemcpyAsync(host, c->rec_dev, 3 * (size_t)c->L.jpi * c->L.jpj * sizeof(double), cudaMemcpyDeviceToHost,
                     c->rec_stream));
  CK(cudaEventRecord(c->rec_copied, c->rec_stream));
  return NEMO_OK;
}

int nemo_host_alloc(size_t bytes, void** ptr) {
  if (!ptr || bytes == 0) return NEMO_ERR_INVALID;
  *ptr = nullptr;
  cudaError_t e = nemo::host_alloc(ptr, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *ptr = nullptr;
    return e == cudaErrorMemoryAllocation ? NEMO_ERR_ALLOC : NEMO_ERR_CUDA;
  }
  return NEMO_OK;
}

int nemo_host_free(void* ptr) {
  if (!ptr) return NEMO_OK;
  return cudaFreeHost(ptr) == cudaSuccess ? NEMO_OK : NEMO_ERR_CUDA;
}

int nemo_record_wait(nemo_ctx* c) {
  if (!c) return NEMO_ERR_INVALID;
  if (!c->rec_copied) return NEMO_OK;
  int st = set_device(c); if (st) return st;
  CK(cudaEventSynchronize(c->rec_copied));
  return NEMO_OK;
}

int nemo_retrieve(nemo_ctx* c, int field, double* host, long ld) {
  if (!c || !host) return NEMO_ERR_INVALID;
  int i0, nx, j0, ny;
  if (!field_window(c, field, &i0, &nx, &j0, &ny)) return NEMO_ERR_INVALID;
  if (ld < nx) return NEMO_ERR_INVALID;
  if (field == NEMO_XT || field == NEMO_YT) {
    // grid, :224-233: xt(1,:) = 0 + 0.5*e1t, xt(ji) = xt(ji-1) + dx (same for yt)
    const double dx = c->p.dx, dy = c->p.dy;
    for (int jj = 0; jj < ny; ++jj) {
      double yv = 0.0 + 0.5 * dy;
      for (int k = 1; k <= jj; ++k) yv = yv + dy;
      double xv = 0.0 + 0.5 * dx;
      for (int ii = 0; ii < nx; ++ii) {
        if (ii > 0) xv = xv + dx;
        host[(long)jj * ld + ii] = (field == NEMO_XT) ? xv : yv;
      }
    }
    return NEMO_OK;
  }
  int st = set_device(c); if (st) return st;
  if ((field == NEMO_SSHN_U || field == NEMO_SSHN_V) && (st = prepare_routine(c, false))) return st;
  double* f = field_storage(c, field);
  const double* src = f + c->L.idx(i0, j0);
  CK(cudaMemcpy2DAsync(host, (size_t)ld * sizeof(double), src, (size_t)c->L.pitch * sizeof(double),
                       (size_t)nx * sizeof(double), (size_t)ny, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return NEMO_OK;
}

int nemo_set_state(nemo_ctx* c, const double* sshn, const double* un, const double* vn) {
  if (!c || !sshn || !un || !vn) return NEMO_ERR_INVALID;
  int st = set_device(c); if (st) return st;
  if ((st = prepare_routine(c, true))) return st;
  const Layout& L = c->L;
  const size_t P = (size_t)L.pitch * sizeof(double);
  CK(cudaMemcpy2DAsync(nset(c).ssh + L.idx(1, 1), P, sshn, (size_t)L.jpi * sizeof(double),
                       (size_t)L.jpi * sizeof(double), (size_t)L.jpj, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpy2DAsync(nset(c).u + L.idx(0, 1), P, un, (size_t)(L.jpi + 1) * sizeof(double),
                       (size_t)(L.jpi + 1) * sizeof(double), (size_t)L.jpj, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpy2DAsync(nset(c).v + L.idx(1, 0), P, vn, (size_t)L.jpi * sizeof(double),
                       (size_t)L.jpi * sizeof(double), (size_t)(L.jpj + 1), cudaMemcpyHostToDevice, c->stream));
  CK(launch_derive_sshn_uv(L, c->C, nset(c).ssh, c->sshn_u, c->sshn_v, c->stream, gridp(c)));
  CK(cudaStreamSynchronize(c->stream));
  c->uv_stale = false;
  // the state as after a complete step: `next` has made the a-fields equal
  // to these (they are materialised before a routine next writes them)
  c->a_mirrors_n = true;
  return NEMO_OK;
}

int nemo_set_grid(nemo_ctx* c, const nemo_grid* g) {
  if (!c || !g || !g->pt || !g->e1t || !g->e2t || !g->e1u || !g->e2u || !g->e1v || !g->e2v || !g->gphiu ||
      !g->gphiv)
    return NEMO_ERR_INVALID;
  const int jpi = c->L.jpi, jpj = c->L.jpj;
  const long ld = jpi + 2;
  const long nh = ld * (jpj + 2);
  for (long k = 0; k < nh; ++k)
    if (g->pt[k] < -1 || g->pt[k] > 1) return NEMO_ERR_INVALID;
  const double* in[] = {g->e1t, g->e2t, g->e1u, g->e2u, g->e1v, g->e2v, g->gphiu, g->gphiv, g->ht, g->hu, g->hv};
  for (const double* a : in)
    if (a)
      for (long k = 0; k < nh; ++k)
        if (!std::isfinite(a[k])) return NEMO_ERR_INVALID;
  int st = set_device(c); if (st) return st;
  CK(cudaStreamSynchronize(c->stream));  // queued steps may still read the depths
  const size_t fe = (size_t)c->L.elems();
  enum { E1T, E2T, E1U, E2U, E1V, E2V, E12T, E12U, E12V, FCU, FCV, NA };
  if (!c->gslab) {
    cudaError_t e = nemo::dev_alloc(&c->gslab, NA * fe * sizeof(double) + fe);
    if (e != cudaSuccess) { c->gslab = nullptr; cudaGetLastError(); return NEMO_ERR_ALLOC; }
  }
  double* base = static_cast<double*>(c->gslab);
  // one host image in the fields' layout at a time: (ji, jj) of the
  // reference's (0:jpi+1, 0:jpj+1) arrays at L.idx(ji, jj), the rest zero
  std::vector<double> img(fe);
  auto upload = [&](int k, auto value, int ji0, int ji1, int jj0, int jj1) -> int {
    std::fill(img.begin(), img.end(), 0.0);
    for (int jj = jj0; jj <= jj1; ++jj)
      for (int ji = ji0; ji <= ji1; ++ji) img[c->L.idx(ji, jj)] = value(jj * ld + ji);
    CK(cudaMemcpy(base + k * fe, img.data(), fe * sizeof(double), cudaMemcpyHostToDevice));
    return NEMO_OK;
  };
  for (int k = 0; k < 6 && !st; ++k)
    st = upload(k, [&](long q) { return in[k][q]; }, 0, jpi + 1, 0, jpj + 1);
  // cell areas over the ranges original/nemolite2d.f90:263-279 fills
  if (!st) st = upload(E12T, [&](long q) { return g->e1t[q] * g->e2t[q]; }, 1, jpi, 1, jpj);
  if (!st) st = upload(E12U, [&](long q) { return g->e1u[q] * g->e2u[q]; }, 0, jpi, 1, jpj);
  if (!st) st = upload(E12V, [&](long q) { return g->e1v[q] * g->e2v[q]; }, 1, jpi, 0, jpj);
  // Coriolis parameters, as the momentum loops form them (:503, :594)
  const double d2r = kPi / 180.0;
  if (!st) st = upload(FCU, [&](long q) { return 2.0 * kOmega * sin(g->gphiu[q] * d2r); }, 0, jpi + 1, 0, jpj + 1);
  if (!st) st = upload(FCV, [&](long q) { return 2.0 * kOmega * sin(g->gphiv[q] * d2r); }, 0, jpi + 1, 0, jpj + 1);
  if (st) return st;
  std::vector<signed char> hp(fe, 0);
  for (int jj = 0; jj <= jpj + 1; ++jj)
    for (int ji = 0; ji <= jpi + 1; ++ji) hp[c->L.idx(ji, jj)] = (signed char)g->pt[jj * ld + ji];
  signed char* pt = reinterpret_cast<signed char*>(base + NA * fe);
  CK(cudaMemcpy(pt, hp.data(), fe, cudaMemcpyHostToDevice));
  // Flather points of the mask, as chains in the sweeps' order
  std::vector<int4> chains;
  flather_chains(g->pt, jpi, jpj, chains);
  if (c->gchains) {
    cudaFree(c->gchains);
    c->gchains = nullptr;
    c->n_gchains = 0;
  }
  if (!chains.empty()) {
    cudaError_t e = nemo::dev_alloc(&c->gchains, chains.size() * sizeof(int4));
    if (e != cudaSuccess) { c->gchains = nullptr; cudaGetLastError(); return NEMO_ERR_ALLOC; }
    CK(cudaMemcpy(c->gchains, chains.data(), chains.size() * sizeof(int4), cudaMemcpyHostToDevice));
    c->n_gchains = (int)chains.size();
  }
  c->grid = GridDev{pt, base + E1T * fe, base + E2T * fe, base + E1U * fe, base + E2U * fe, base + E1V * fe,
                    base + E2V * fe, base + E12T * fe, base + E12U * fe, base + E12V * fe, base + FCU * fe,
                    base + FCV * fe};
  // depths, when given (the rest of each depth array is kept)
  double* hd[3] = {c->ht, c->hu, c->hv};
  for (int k = 0; k < 3; ++k) {
    if (!in[8 + k]) continue;
    CK(cudaMemcpy(img.data(), hd[k], fe * sizeof(double), cudaMemcpyDeviceToHost));
    for (int jj = 0; jj <= jpj + 1; ++jj)
      for (int ji = 0; ji <= jpi + 1; ++ji) img[c->L.idx(ji, jj)] = in[8 + k][jj * ld + ji];
    CK(cudaMemcpy(hd[k], img.data(), fe * sizeof(double), cudaMemcpyHostToDevice));
  }
  c->general = true;
  // the a-fields stay as they are; sshn_u/sshn_v restart from the current
  // sshn with the initialisation's averages (:337-353)
  if ((st = prepare_routine(c, true))) return st;
  CK(launch_init_sshn_uv(c->L, c->C, nset(c).ssh, c->sshn_u, c->sshn_v, c->stream, gridp(c)));
  CK(cudaStreamSynchronize(c->stream));
  c->uv_stale = false;
  return NEMO_OK;
}

int nemo_sync(nemo_ctx* c) {
  if (!c) return NEMO_ERR_STATE;
  int st = set_device(c); if (st) return st;
  CK(cudaStreamSynchronize(c->stream));
  return NEMO_OK;
}

int nemo_get_dims(nemo_ctx* c, int* jpi, int* jpj) {
  if (!c || !jpi || !jpj) return NEMO_ERR_INVALID;
  *jpi = c->L.jpi;
  *jpj = c->L.jpj;
  return NEMO_OK;
}

int nemo_device_field(nemo_ctx* c, int field, double** ptr, long* pitch) {
  if (!c || !ptr || !pitch) return NEMO_ERR_INVALID;
  double* f = field_storage(c, field);
  if (!f) return NEMO_ERR_INVALID;
  if (field == NEMO_SSHN_U || field == NEMO_SSHN_V) {
    int st = set_device(c); if (st) return st;
    if ((st = prepare_routine(c, false))) return st;
  }
  *ptr = f;
  *pitch = c->L.pitch;
  return NEMO_OK;
}

int nemo_set_schedule(nemo_ctx* c, const nemo_schedule* s) {
  if (!c) return NEMO_ERR_STATE;
  if (c->general) {
    if (!s || s->warps != 2 || (s->occupancy != 0 && s->occupancy != 3 && s->occupancy != 4) || s->rows < 1 ||
        s->rows > 65536)
      return NEMO_ERR_INVALID;
    c->gsched = *s;
    return NEMO_OK;
  }
  if (!s || !fused_variant_ok(s->warps, s->occupancy, c->recip_nr_ok) || s->rows < 0 || s->rows > 65536)
    return NEMO_ERR_INVALID;
  c->sched = *s;
  return NEMO_OK;
}

int nemo_get_schedule(nemo_ctx* c, nemo_schedule* s) {
  if (!c || !s) return NEMO_ERR_INVALID;
  *s = c->general ? c->gsched : c->sched;
  return NEMO_OK;
}

int nemo_autotune(nemo_ctx* c, int steps, nemo_schedule* best, double* best_ms) {
  if (!c || steps < 1) return NEMO_ERR_INVALID;
  if (c->general) return NEMO_ERR_STATE;  // no fused schedules on a general grid
  int st = set_device(c); if (st) return st;
  // both state sets and the bookkeeping are restored afterwards
  const size_t fe = (size_t)c->L.elems();
  double* backup = nullptr;
  CK(nemo::dev_alloc(&backup, 6 * fe * sizeof(double)));
  const int n_save = c->n_idx;
  const bool a_save = c->a_mirrors_n, uv_save = c->uv_stale;
  cudaError_t er = cudaSuccess;
  for (int s = 0; s < 2 && er == cudaSuccess; ++s) {
    double* f3[3] = {c->set[s].ssh, c->set[s].u, c->set[s].v};
    for (int k = 0; k < 3 && er == cudaSuccess; ++k)
      er = cudaMemcpyAsync(backup + (3 * s + k) * fe, f3[k], fe * sizeof(double), cudaMemcpyDeviceToDevice, c->stream);
  }
  const nemo_schedule keep = c->sched;
  nemo_schedule bsched = keep;
  double bms = 1e300;
  const int wo[][2] = {{2, 216}, {2, 220}, {4, 216}, {4, 220}, {2, 116}, {2, 120}, {4, 116}, {4, 120},
                       {2, -24}, {2, -20}, {2, -16}, {2, 0}, {2, 16}, {2, 20}, {2, 24}, {4, -20}, {4, 0},
                       {4, 16}, {4, 20}, {4, 24}, {8, 0}, {8, 16}, {8, 24}};
  const int rows_c[] = {8, 16, 32, 0};
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  if (er == cudaSuccess) er = cudaEventCreate(&t0);
  if (er == cudaSuccess) er = cudaEventCreate(&t1);
  for (const auto& w : wo) {
    if (!fused_variant_ok(w[0], w[1], c->recip_nr_ok)) continue;
    for (int rows : rows_c) {
      if (er != cudaSuccess || st) break;
      nemo_schedule cand{w[0], w[1], rows};
      c->sched = cand;
      if ((st = nemo_step_n(c, 1, 1))) break;  // warm
      er = cudaEventRecord(t0, c->stream);
      if (er == cudaSuccess && (st = nemo_step_n(c, 2, steps))) break;
      if (er == cudaSuccess) er = cudaEventRecord(t1, c->stream);
      if (er == cudaSuccess) er = cudaEventSynchronize(t1);
      float ms = 0.f;
      if (er == cudaSuccess) er = cudaEventElapsedTime(&ms, t0, t1);
      if (er == cudaSuccess && ms / steps < bms) {
        bms = ms / steps;
        bsched = cand;
      }
    }
  }
  if (t0) cudaEventDestroy(t0);
  if (t1) cudaEventDestroy(t1);
  for (int s = 0; s < 2; ++s) {
    double* f3[3] = {c->set[s].ssh, c->set[s].u, c->set[s].v};
    for (int k = 0; k < 3; ++k) {
      cudaError_t e2 = cudaMemcpyAsync(f3[k], backup + (3 * s + k) * fe, fe * sizeof(double),
                                       cudaMemcpyDeviceToDevice, c->stream);
      if (er == cudaSuccess) er = e2;
    }
  }
  cudaError_t e3 = cudaStreamSynchronize(c->stream);
  if (er == cudaSuccess) er = e3;
  cudaFree(backup);
  c->n_idx = n_save;
  c->a_mirrors_n = a_save;
  c->uv_stale = uv_save;
  c->sched = (bms < 1e300) ? bsched : keep;
  if (er != cudaSuccess) return status_from(er);
  if (st) return st;
  if (bms < 1e300) tune_store(c, c->sched, bms);
  if (best) *best = c->sched;
  if (best_ms) *best_ms = bms;
  return NEMO_OK;
}

int nemo_debug_fail_alloc(int n) {
  if (n < 0) return -1;
  return nemo::g_alloc_countdown.exchange(n, std::memory_order_relaxed);
}

const char* nemo_status_string(int s) {
  switch (s) {
    case NEMO_OK: return "ok";
    case NEMO_ERR_INVALID: return "invalid argument";
    case NEMO_ERR_CUDA: return "CUDA runtime error";
    case NEMO_ERR_ALLOC: return "allocation failed";
    case NEMO_ERR_STATE: return "invalid state";
    case NEMO_ERR_TIMEOUT: return "device wait timed out";
    case NEMO_ERR_UNSUPPORTED: return "unsupported";
    default: return "unknown status";
  }
}

int nemo_build_is_strict(void) {
#ifdef NEMO_STRICT_BUILD
  return 1;
#else
  return 0;
#endif
}

// ---- drop-in symbols: one default context, as the reference's globals -----
static nemo_params g_params;
static bool g_params_set = false;
static nemo_ctx* g_ctx = nullptr;
static int g_status = NEMO_OK;

static void compat_fail(const char* where, int st) {
  if (st == NEMO_OK) return;
  if (g_status == NEMO_OK) g_status = st;
  fprintf(stderr, "[nemo_b200] %s: %s\n", where, nemo_status_string(st));
}

int nemo_compat_last_status(void) { return g_status; }
nemo_ctx* nemo_compat_context(void) { return g_ctx; }

void cuda_setup_model_params_(int jpi, int jpj, double dx, double dy, double dep_const,
                              int nit000, int nitend, int irecord, double rdt, double cbfr,
                              double visc) {
  nemo_default_params(&g_params);
  g_params.jpi = jpi;
  g_params.jpj = jpj;
  g_params.dx = dx;
  g_params.dy = dy;
  g_params.dep_const = dep_const;
  g_params.nit000 = nit000;
  g_params.nitend = nitend;
  g_params.irecord = irecord;
  g_params.rdt = rdt;
  g_params.cbfr = cbfr;
  g_params.visc = visc;
  g_params_set = true;
  g_status = NEMO_OK;
}

void cuda_initialise_grid_(void) {
  if (!g_params_set) {
    // the reference only printed here (cuda/cuda_nemolite2d.cu:298-303)
    compat_fail("cuda_initialise_grid_ (have you set up model params?)", NEMO_ERR_STATE);
    return;
  }
  if (g_ctx) { nemo_destroy(g_ctx); g_ctx = nullptr; }
  compat_fail("cuda_initialise_grid_", nemo_create(&g_params, &g_ctx));
}

void cuda_continuity_(void) { compat_fail("cuda_continuity_", g_ctx ? nemo_continuity(g_ctx) : NEMO_ERR_STATE); }
void cuda_momentum_(void) { compat_fail("cuda_momentum_", g_ctx ? nemo_momentum(g_ctx) : NEMO_ERR_STATE); }
void cuda_boundary_conditions_(double rtime) {
  compat_fail("cuda_boundary_conditions_", g_ctx ? nemo_bc(g_ctx, rtime) : NEMO_ERR_STATE);
}
void cuda_next_(void) { compat_fail("cuda_next_", g_ctx ? nemo_next(g_ctx) : NEMO_ERR_STATE); }

void cuda_retrieve_grid_constants_(double* xt, double* yt, double* ht, int jpi, int jpj) {
  if (!g_ctx || jpi != g_ctx->L.jpi || jpj != g_ctx->L.jpj) {
    compat_fail("cuda_retrieve_grid_constants_", g_ctx ? NEMO_ERR_INVALID : NEMO_ERR_STATE);
    return;
  }
  compat_fail("cuda_retrieve_grid_constants_", nemo_retrieve(g_ctx, NEMO_XT, xt, jpi));
  compat_fail("cuda_retrieve_grid_constants_", nemo_retrieve(g_ctx, NEMO_YT, yt, jpi));
  compat_fail("cuda_retrieve_grid_constants_", nemo_retrieve(g_ctx, NEMO_HT, ht, jpi));
}

void cuda_retrieve_results_(double* sshn, double* un, double* vn, double* ua, double* va, int jpi,
                            int jpj) {
  if (!g_ctx || jpi != g_ctx->L.jpi || jpj != g_ctx->L.jpj) {
    compat_fail("cuda_retrieve_results_", g_ctx ? NEMO_ERR_INVALID : NEMO_ERR_STATE);
    return;
  }
  compat_fail("cuda_retrieve_results_", nemo_retrieve(g_ctx, NEMO_SSHN, sshn, jpi));
  compat_fail("cuda_retrieve_results_", nemo_retrieve(g_ctx, NEMO_UN, un, jpi + 1));
  compat_fail("cuda_retrieve_results_", nemo_retrieve(g_ctx, NEMO_VN, vn, jpi));
  compat_fail("cuda_retrieve_results_", nemo_retrieve(g_ctx, NEMO_UA, ua, jpi + 1));
  compat_fail("cuda_retrieve_results_", nemo_retrieve(g_ctx, NEMO_VA, va, jpi));
}

void cuda_finalise_(void) {
  if (g_ctx) nemo_destroy(g_ctx);
  g_ctx = nullptr;
  g_params_set = false;
}

}  // extern "C"
