// Batched ensemble: many independent NEMOLite2D instances of uneven size in
// one persistent launch per step (no reference counterpart).
//
// Every member has its own pitched storage (the single-grid layout) inside
// one slab and a row in a device table of member descriptors.  A work list
// of (member, column strip, row block) items, built on the host in the order
// the schedule asks for, is consumed by a persistent grid: each warp takes
// items w, w + W, w + 2W, ... and runs the same strip code as the single-grid
// kernel, so each member evolves bit-identically to a nemo_ctx with the same
// parameters.  Tides differ per member and step; the host evaluates them with
// the same libm call as the single-grid path and uploads one table per
// nemo_ens_step_n call.  The n launches of a call are captured once into a
// CUDA graph (per n and buffer parity) and replayed.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <new>
#include <utility>
#include <vector>

#include "nemo_step_dev.cuh"
#include "sur_internal.h"

using namespace nemo;

namespace {

struct MemberDev {
  Layout L;
  double* st[2][3];  // [set][sshn, un, vn]
  const double *ht, *hu, *hv, *sshv0;
  const double *rhu, *rhv;
};

// Next work item of a warp under the dynamic schedule: one atomic per item.
__device__ __forceinline__ int ens_fetch(int* counter, int lane) {
  int w = 0;
  if (lane == 0) w = atomicAdd(counter, 1);
  return __shfl_sync(0xffffffffu, w, 0);
}

// counter == nullptr: warp w takes items w, w + W, w + 2W, ... (W warps in
// the grid).  Otherwise the dynamic schedule: warps take the next item of the
// list from counter[parity] as they finish one (the list is ordered largest
// first), and the launch resets counter[parity ^ 1] for the next launch,
// whose buffer parity is the other one.
template <int NW, int MB, int PF>
__global__ void __launch_bounds__(32 * NW, MB)
k_ens_step(const MemberDev* __restrict__ mem, const int4* __restrict__ work, int nwork, Consts C,
           const double* __restrict__ tide, int parity, int* counter) {
  const int lane = threadIdx.x & 31;
  const int nw = (int)gridDim.x * NW;
  if (counter && blockIdx.x == 0 && threadIdx.x == 0) counter[parity ^ 1] = 0;
  for (int w = counter ? ens_fetch(counter + parity, lane) : (int)blockIdx.x * NW + (int)(threadIdx.x >> 5);
       w < nwork; w = counter ? ens_fetch(counter + parity, lane) : w + nw) {
    const int4 it = work[w];  // member, c0, J0, J1
    const MemberDev* M = mem + it.x;
    FusedArgs A;
    A.sshn = M->st[parity][0];
    A.un = M->st[parity][1];
    A.vn = M->st[parity][2];
    A.ssha = M->st[parity ^ 1][0];
    A.ua = M->st[parity ^ 1][1];
    A.va = M->st[parity ^ 1][2];
    A.ht = M->ht;
    A.hu = M->hu;
    A.hv = M->hv;
    A.rhu = M->rhu;
    A.rhv = M->rhv;
    A.sshv0 = M->sshv0;
    A.tide = tide[it.x];
    const Layout L = M->L;
    if constexpr (PF >= 2) {
      constexpr int RD = stepdev::ring_doubles<PF == 3>();
      __shared__ double ring[NW * RD];
      stepdev::run_strip_ring<PF == 3, 2>(L, C, A, it.y, it.z, it.w, lane, ring + (threadIdx.x >> 5) * RD);
    } else {
      stepdev::run_strip<PF>(L, C, A, it.y, it.z, it.w, lane);
    }
  }
}

// Checksums of every member in one pass: a block per (member row, field),
// then a block per (member, field) over that member's row sums -- the same
// fixed order as the single-grid checksum kernels.
constexpr int CT = 256;

__device__ __forceinline__ double block_sum(double acc, double* smem) {
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1) acc = acc + __shfl_xor_sync(0xffffffffu, acc, off);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) smem[warp] = acc;
  __syncthreads();
  double r = 0.0;
  if (warp == 0) {
    double x = (lane < CT / 32) ? smem[lane] : 0.0;
#pragma unroll
    for (int off = CT / 64; off >= 1; off >>= 1) x = x + __shfl_xor_sync(0xffffffffu, x, off);
    r = x;
  }
  return r;
}

__global__ void __launch_bounds__(CT) k_ens_rows(const MemberDev* __restrict__ mem,
                                                 const int2* __restrict__ rows, int nrows,
                                                 int parity, double* partial) {
  __shared__ double smem[CT / 32];
  const int2 r = rows[blockIdx.x];  // member, jj
  const MemberDev* M = mem + r.x;
  const Layout L = M->L;
  const double* a = M->st[parity][blockIdx.y] + L.idx(1, r.y);
  double acc = 0.0;
  for (int k = threadIdx.x; k < L.jpi; k += CT) acc = acc + fabs(a[k]);
  double s = block_sum(acc, smem);
  if (threadIdx.x == 0) partial[(long)blockIdx.y * nrows + blockIdx.x] = s;
}

__global__ void __launch_bounds__(CT) k_ens_cols(const int* __restrict__ row_off,
                                                 const int* __restrict__ row_cnt,
                                                 const double* __restrict__ partial, int nrows,
                                                 double* out) {
  __shared__ double smem[CT / 32];
  const int m = blockIdx.x, f = blockIdx.y;
  const double* a = partial + (long)f * nrows + row_off[m];
  const int n = row_cnt[m];
  double acc = 0.0;
  for (int k = threadIdx.x; k < n; k += CT) acc = acc + a[k];
  double s = block_sum(acc, smem);
  if (threadIdx.x == 0) out[3 * m + f] = s;
}

template <int NW, int MB, int PF>
cudaError_t launch_ens_variant(const MemberDev* mem, const int4* work, int nwork, const Consts& C,
                               const double* tide, int parity, int ctas, int* counter, cudaStream_t s) {
  if (ctas <= 0) {
    static int slots = 0;
    if (slots == 0) {
      int dev = 0, sms = 0, per_sm = 0;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_ens_step<NW, MB, PF>, 32 * NW, 0);
      slots = sms * (per_sm > 0 ? per_sm : 1);
    }
    ctas = slots;
  }
  const int need = (nwork + NW - 1) / NW;
  if (ctas > need) ctas = need;
  if (ctas < 1) ctas = 1;
  k_ens_step<NW, MB, PF><<<ctas, 32 * NW, 0, s>>>(mem, work, nwork, C, tide, parity, counter);
  return cudaGetLastError();
}

cudaError_t launch_ens(int warps, int occ, const MemberDev* mem, const int4* work, int nwork,
                       const Consts& C, const double* tide, int parity, int ctas, int* counter,
                       cudaStream_t s) {
#define ENS(NW, MB, PF) launch_ens_variant<NW, MB, PF>(mem, work, nwork, C, tide, parity, ctas, counter, s)
  if (warps == 2) {
    switch (occ) {
      case 212: return ENS(2, 6, 3);
      case 216: return ENS(2, 8, 3);
      case 220: return ENS(2, 10, 3);
      case 116: return ENS(2, 8, 2);
      case 120: return ENS(2, 10, 2);
      case -24: return ENS(2, 12, 0);
      case -20: return ENS(2, 10, 0);
      case 20: return ENS(2, 10, 1);
      case 24: return ENS(2, 12, 1);
    }
  } else if (warps == 4) {
    switch (occ) {
      case 212: return ENS(4, 3, 3);
      case 216: return ENS(4, 4, 3);
      case 116: return ENS(4, 4, 2);
      case -20: return ENS(4, 5, 0);
      case 20: return ENS(4, 5, 1);
      case 24: return ENS(4, 6, 1);
    }
  }
#undef ENS
  return cudaErrorInvalidValue;
}

bool ens_variant_ok(int warps, int occ, bool nr_ok) {
  if (warps == 2 && (occ == 212 || occ == 216 || occ == 220)) return nr_ok;
  if (warps == 4 && (occ == 212 || occ == 216)) return nr_ok;
  if (warps == 2) return occ == -24 || occ == -20 || occ == 20 || occ == 24 || occ == 116 || occ == 120;
  if (warps == 4) return occ == -20 || occ == 20 || occ == 24 || occ == 116;
  return false;
}

int status_of(cudaError_t e) {
  if (e == cudaSuccess) return NEMO_OK;
  if (e == cudaErrorMemoryAllocation) return NEMO_ERR_ALLOC;
  return NEMO_ERR_CUDA;
}

#define ECK(call)                                   \
  do {                                              \
    cudaError_t e_ = (call);                        \
    if (e_ != cudaSuccess) return status_of(e_);    \
  } while (0)

uint64_t smix(uint64_t* s) {
  uint64_t z = (*s += 0x9E3779B97F4A7C15ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
double unif(uint64_t* s) { return (double)(smix(s) >> 11) * 0x1.0p-53; }

}  // namespace

struct nemo_ens {
  nemo_params common;
  Consts C;
  int device = -1;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::vector<nemo_member> mem;
  std::vector<MemberDev> hmem;
  double* slab = nullptr;
  MemberDev* d_mem = nullptr;
  int4* d_work = nullptr;
  int nwork = 0, work_cap = 0;
  int2* d_rows = nullptr;
  int* d_row_off = nullptr;
  int* d_row_cnt = nullptr;
  int nrows = 0;
  double* d_partial = nullptr;
  double* d_ck = nullptr;
  double* h_ck = nullptr;
  double* d_tide = nullptr;
  double* h_tide = nullptr;
  int tide_cap = 0;  // steps
  cudaEvent_t tide_ev = nullptr;
  int parity = 0;
  nemo_ens_schedule sched{};
  bool use_graph = true;
  std::map<std::pair<int, int>, cudaGraphExec_t> graphs;
  long long cells = 0;
  int4* d_work_sub = nullptr;  // work list of a member subset (ens_step_subset)
  int* d_counter = nullptr;    // dynamic schedule: [main parity 0, 1, subset parity 0, 1]
  int sub_cap = 0;
  bool recip_nr_ok = false;    // every member's depths pass launch_recip's check
};

namespace {

int set_dev(nemo_ens* e) {
  if (e->device >= 0) ECK(cudaSetDevice(e->device));
  return NEMO_OK;
}

void drop_graphs(nemo_ens* e) {
  for (auto& kv : e->graphs) cudaGraphExecDestroy(kv.second);
  e->graphs.clear();
}

// Work items of every member (or of the members with sel[m] != 0) in the
// schedule's order: row blocks of `rows` rows, each split into 30-column
// strips, neighbouring strips of one row block consecutive so concurrently
// running warps share halo rows in L2.
// Order 2 (the dynamic schedule) lists the same items largest first: the
// members by size, then every item of R rows before the shorter last blocks.
std::vector<int4> work_items(const nemo_ens* e, const char* sel) {
  const int R = e->sched.rows;
  std::vector<int> order(e->mem.size());
  for (size_t m = 0; m < order.size(); ++m) order[m] = (int)m;
  if (e->sched.order >= 1)
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
      return (long)e->mem[a].jpi * e->mem[a].jpj > (long)e->mem[b].jpi * e->mem[b].jpj;
    });
  std::vector<int4> w;
  for (int m : order) {
    if (sel && !sel[m]) continue;
    const int jpi = e->mem[m].jpi, jpj = e->mem[m].jpj;
    for (int J0 = 1; J0 <= jpj; J0 += R)
      for (int c0 = 1; c0 <= jpi; c0 += 30) w.push_back(make_int4(m, c0, J0, std::min(J0 + R - 1, jpj)));
  }
  if (e->sched.order == 2)
    std::stable_sort(w.begin(), w.end(), [](const int4& a, const int4& b) { return a.w - a.z > b.w - b.z; });
  return w;
}

int* counter_of(nemo_ens* e, bool subset) {
  return e->sched.order == 2 ? e->d_counter + (subset ? 2 : 0) : nullptr;
}

int build_work(nemo_ens* e) {
  const std::vector<int4> w = work_items(e, nullptr);
  if ((int)w.size() > e->work_cap) {
    if (e->d_work) cudaFree(e->d_work);
    e->d_work = nullptr;
    ECK(nemo::dev_alloc(&e->d_work, w.size() * sizeof(int4)));
    e->work_cap = (int)w.size();
  }
  ECK(cudaMemcpyAsync(e->d_work, w.data(), w.size() * sizeof(int4), cudaMemcpyHostToDevice, e->stream));
  ECK(cudaStreamSynchronize(e->stream));
  e->nwork = (int)w.size();
  drop_graphs(e);
  return NEMO_OK;
}

int ensure_tide(nemo_ens* e, int n) {
  if (n <= e->tide_cap) return NEMO_OK;
  ECK(cudaStreamSynchronize(e->stream));
  if (e->d_tide) cudaFree(e->d_tide);
  if (e->h_tide) cudaFreeHost(e->h_tide);
  e->d_tide = nullptr;
  e->h_tide = nullptr;
  const size_t cnt = (size_t)n * e->mem.size();
  ECK(nemo::dev_alloc(&e->d_tide, cnt * sizeof(double)));
  ECK(nemo::host_alloc(&e->h_tide, cnt * sizeof(double)));
  e->tide_cap = n;
  drop_graphs(e);  // graphs hold the old table address
  return NEMO_OK;
}

// Tidal SSH of every member for steps istp0 .. istp0+n-1 into d_tide,
// amp*sin(omega_tide*rtime + phase) as original/nemolite2d.f90:629-635.
int upload_tides(nemo_ens* e, int istp0, int n) {
  int st = ensure_tide(e, n);
  if (st) return st;
  ECK(cudaEventSynchronize(e->tide_ev));  // previous upload has left the pinned buffer
  const size_t nm = e->mem.size();
  const double omega_tide = 2.0 * 3.14159 / (12.42 * 3600.0);
  for (int k = 0; k < n; ++k) {
    const double rtime = (double)(istp0 + k) * e->common.rdt;
    for (size_t m = 0; m < nm; ++m)
      e->h_tide[(size_t)k * nm + m] = e->mem[m].amp_tide * sin(omega_tide * rtime + e->mem[m].tide_phase);
  }
  ECK(cudaMemcpyAsync(e->d_tide, e->h_tide, (size_t)n * nm * sizeof(double), cudaMemcpyHostToDevice, e->stream));
  ECK(cudaEventRecord(e->tide_ev, e->stream));
  return NEMO_OK;
}

int launch_steps(nemo_ens* e, int n, int p0) {
  const size_t nm = e->mem.size();
  for (int k = 0; k < n; ++k)
    ECK(launch_ens(e->sched.warps, e->sched.occupancy, e->d_mem, e->d_work, e->nwork, e->C,
                   e->d_tide + (size_t)k * nm, (p0 + k) & 1, e->sched.ctas, counter_of(e, false),
                   e->stream));
  return NEMO_OK;
}

}  // namespace

extern "C" {

int nemo_ens_generate(uint64_t seed, int nmem, int side_min, int side_max, double amp_scale,
                      nemo_member* out) {
  if (!out || nmem < 1 || side_min < 2 || side_max < side_min) return NEMO_ERR_INVALID;
  uint64_t s = seed;
  const double l0 = log((double)side_min), l1 = log((double)side_max);
  const double a0 = log(0.5), a1 = log(2.0);
  for (int m = 0; m < nmem; ++m) {
    nemo_member& x = out[m];
    const double side = exp(l0 + (l1 - l0) * unif(&s));
    const double aspect = exp(a0 + (a1 - a0) * unif(&s));
    x.jpi = std::max(2, (int)lround(side));
    x.jpj = std::max(2, (int)lround(side * aspect));
    x.amp_tide = amp_scale * (0.5 + unif(&s));
    x.tide_phase = 2.0 * kPi * unif(&s);
    x.dep_const = 100.0;
    x.nbump = 8;
    x.seed = smix(&s);
    x.bump_amp = 50.0;
    const double lmin = 1000.0 * (double)std::min(x.jpi, x.jpj);
    x.bump_wmin = 0.05 * lmin;
    x.bump_wmax = 0.25 * lmin;
    x.hmin = 50.0;
    x.hmax = 150.0;
  }
  return NEMO_OK;
}

int nemo_ens_destroy(nemo_ens* e) {
  if (!e) return NEMO_ERR_INVALID;
  if (e->device >= 0) cudaSetDevice(e->device);
  if (e->stream) cudaStreamSynchronize(e->stream);
  drop_graphs(e);
  cudaFree(e->slab);
  cudaFree(e->d_mem);
  cudaFree(e->d_work);
  cudaFree(e->d_work_sub);
  cudaFree(e->d_rows);
  cudaFree(e->d_row_off);
  cudaFree(e->d_row_cnt);
  cudaFree(e->d_partial);
  cudaFree(e->d_ck);
  cudaFree(e->d_counter);
  cudaFree(e->d_tide);
  if (e->h_ck) cudaFreeHost(e->h_ck);
  if (e->h_tide) cudaFreeHost(e->h_tide);
  if (e->tide_ev) cudaEventDestroy(e->tide_ev);
  if (e->own_stream && e->stream) cudaStreamDestroy(e->stream);
  delete e;
  return NEMO_OK;
}

int nemo_ens_create(const nemo_params* common, const nemo_member* members, int nmem,
                    nemo_ens** out) {
  if (!out) return NEMO_ERR_INVALID;
  *out = nullptr;
  if (!common || !members || nmem < 1 || nmem > (1 << 20)) return NEMO_ERR_INVALID;
  if (!(common->dx > 0.0) || !(common->dy > 0.0) || !(common->rdt > 0.0)) return NEMO_ERR_INVALID;
  for (int m = 0; m < nmem; ++m) {
    const nemo_member& x = members[m];
    if (x.jpi < 2 || x.jpj < 2 || x.jpi > (1 << 15) || x.jpj > (1 << 15)) return NEMO_ERR_INVALID;
    if (x.nbump < 0 || x.nbump > 4096) return NEMO_ERR_INVALID;
    if (x.nbump > 0 && !(x.bump_wmin > 0.0 && x.bump_wmax >= x.bump_wmin)) return NEMO_ERR_INVALID;
  }
  nemo_ens* e = new (std::nothrow) nemo_ens();
  if (!e) return NEMO_ERR_ALLOC;
  e->common = *common;
  e->device = common->device;
  e->C = make_consts(*common);
  e->mem.assign(members, members + nmem);
  e->sched.warps = 2;
  e->sched.occupancy = 216;  // 116 when a member's depths fail the reciprocal check
  e->sched.rows = 16;
  e->sched.order = 1;
  e->sched.ctas = 0;
  int st = set_dev(e);
  if (st) { delete e; return st; }
  cudaError_t err;
  if (common->stream) {
    e->stream = (cudaStream_t)common->stream;
  } else {
    err = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking);
    if (err != cudaSuccess) { delete e; return status_of(err); }
    e->own_stream = true;
  }
  // storage: 13 fields per member in one slab
  std::vector<size_t> off(nmem);
  size_t total = 0;
  e->hmem.resize(nmem);
  for (int m = 0; m < nmem; ++m) {
    Layout L;
    L.jpi = members[m].jpi;
    L.jpj = members[m].jpj;
    L.pitch = layout_pitch(L.jpi);
    L.rows = (long)L.jpj + 3;
    e->hmem[m].L = L;
    off[m] = total;
    total += 13 * (size_t)L.elems();
    e->cells += (long long)L.jpi * L.jpj;
    e->nrows += L.jpj;
  }
  err = nemo::dev_alloc(&e->slab, total * sizeof(double));
  if (err != cudaSuccess) { e->slab = nullptr; cudaGetLastError(); nemo_ens_destroy(e); return NEMO_ERR_ALLOC; }
  err = cudaMemsetAsync(e->slab, 0, total * sizeof(double), e->stream);
  if (err != cudaSuccess) { nemo_ens_destroy(e); return status_of(err); }
  std::vector<int2> rows;
  std::vector<int> row_off(nmem), row_cnt(nmem);
  rows.reserve(e->nrows);
  double* tab = nullptr;
  size_t tab_cap = 0;
  int* d_bad = nullptr;  // depths whose in-kernel reciprocal differs from RN(1/h)
  err = nemo::dev_alloc(&d_bad, sizeof(int));
  if (err == cudaSuccess) err = cudaMemsetAsync(d_bad, 0, sizeof(int), e->stream);
  for (int m = 0; m < nmem && err == cudaSuccess; ++m) {
    MemberDev& d = e->hmem[m];
    const size_t fe = (size_t)d.L.elems();
    double* q = e->slab + off[m];
    for (int s = 0; s < 2; ++s)
      for (int f = 0; f < 3; ++f) { d.st[s][f] = q; q += fe; }
    double* sshn_u = q; q += fe;
    double* sshn_v = q; q += fe;
    double* ht = q; q += fe;
    double* hu = q; q += fe;
    double* hv = q; q += fe;
    double* rhu = q; q += fe;
    double* rhv = q; q += fe;
    d.ht = ht; d.hu = hu; d.hv = hv; d.sshv0 = sshn_v;
    d.rhu = rhu; d.rhv = rhv;
    // grid: seeded bathymetry of the member
    nemo_params p = *common;
    p.jpi = d.L.jpi; p.jpj = d.L.jpj;
    p.dep_const = members[m].dep_const;
    p.nbump = members[m].nbump; p.seed = members[m].seed;
    p.bump_amp = members[m].bump_amp; p.bump_wmin = members[m].bump_wmin;
    p.bump_wmax = members[m].bump_wmax; p.hmin = members[m].hmin; p.hmax = members[m].hmax;
    if (p.nbump > 0) {
      const size_t nax = (size_t)p.nbump * (2 * p.jpi + 2), ngy = (size_t)p.nbump * (2 * p.jpj + 2);
      std::vector<double> h(nax + ngy);
      depth_tables(p, h.data(), h.data() + nax);
      if (nax + ngy > tab_cap) {
        err = cudaStreamSynchronize(e->stream);
        if (tab) cudaFree(tab);
        tab = nullptr;
        if (err == cudaSuccess) err = nemo::dev_alloc(&tab, (nax + ngy) * sizeof(double));
        tab_cap = nax + ngy;
      }
      if (err == cudaSuccess)
        // stream-ordered: a pageable cudaMemcpy on the legacy stream may return
        // before its DMA lands and is not ordered with a non-blocking stream
        err = cudaMemcpyAsync(tab, h.data(), (nax + ngy) * sizeof(double), cudaMemcpyHostToDevice,
                              e->stream);
      if (err == cudaSuccess)
        err = launch_depth(d.L, p.dep_const, p.nbump, tab, tab + nax, p.hmin, p.hmax, ht, hu, hv, e->stream);
      if (err == cudaSuccess) err = cudaStreamSynchronize(e->stream);
    } else {
      err = launch_depth(d.L, p.dep_const, 0, nullptr, nullptr, p.hmin, p.hmax, ht, hu, hv, e->stream);
    }
    if (err == cudaSuccess) err = launch_recip(d.L, hu, hv, rhu, rhv, d_bad, e->stream);
    if (err == cudaSuccess) {
      Consts C = make_consts(p);
      err = launch_init_sshn_uv(d.L, C, d.st[0][0], sshn_u, sshn_v, e->stream);
    }
    row_off[m] = (int)rows.size();
    row_cnt[m] = d.L.jpj;
    for (int jj = 1; jj <= d.L.jpj; ++jj) rows.push_back(make_int2(m, jj));
  }
  if (tab) { cudaStreamSynchronize(e->stream); cudaFree(tab); }
  int h_bad = -1;
  if (err == cudaSuccess) err = cudaMemcpyAsync(&h_bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, e->stream);
  if (err == cudaSuccess) err = cudaStreamSynchronize(e->stream);
  if (d_bad) cudaFree(d_bad);
  e->recip_nr_ok = (err == cudaSuccess && h_bad == 0);
  if (!e->recip_nr_ok) e->sched.occupancy = 116;
  if (err != cudaSuccess) { nemo_ens_destroy(e); return status_of(err); }
  const size_t nm = (size_t)nmem;
  err = nemo::dev_alloc(&e->d_mem, nm * sizeof(MemberDev));
  if (err == cudaSuccess) err = nemo::dev_alloc(&e->d_rows, rows.size() * sizeof(int2));
  if (err == cudaSuccess) err = nemo::dev_alloc(&e->d_row_off, nm * sizeof(int));
  if (err == cudaSuccess) err = nemo::dev_alloc(&e->d_row_cnt, nm * sizeof(int));
  if (err == cudaSuccess) err = nemo::dev_alloc(&e->d_partial, 3 * rows.size() * sizeof(double));
  if (err == cudaSuccess) err = nemo::dev_alloc(&e->d_ck, 3 * nm * sizeof(double));
  if (err == cudaSuccess) err = nemo::dev_alloc(&e->d_counter, 4 * sizeof(int));
  if (err == cudaSuccess) err = cudaMemsetAsync(e->d_counter, 0, 4 * sizeof(int), e->stream);
  if (err == cudaSuccess) err = nemo::host_alloc(&e->h_ck, 3 * nm * sizeof(double));
  if (err == cudaSuccess) err = cudaEventCreateWithFlags(&e->tide_ev, cudaEventDisableTiming);
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(e->d_mem, e->hmem.data(), nm * sizeof(MemberDev), cudaMemcpyHostToDevice, e->stream);
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(e->d_rows, rows.data(), rows.size() * sizeof(int2), cudaMemcpyHostToDevice, e->stream);
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(e->d_row_off, row_off.data(), nm * sizeof(int), cudaMemcpyHostToDevice, e->stream);
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(e->d_row_cnt, row_cnt.data(), nm * sizeof(int), cudaMemcpyHostToDevice, e->stream);
  if (err == cudaSuccess) err = cudaStreamSynchronize(e->stream);
  if (err != cudaSuccess) { cudaGetLastError(); nemo_ens_destroy(e); return status_of(err); }
  st = build_work(e);
  if (st == NEMO_OK) st = ensure_tide(e, 128);
  if (st != NEMO_OK) { nemo_ens_destroy(e); return st; }
  *out = e;
  return NEMO_OK;
}

int nemo_ens_step_n(nemo_ens* e, int istp0, int n) {
  if (!e) return NEMO_ERR_STATE;
  if (n < 0) return NEMO_ERR_INVALID;
  if (n == 0) return NEMO_OK;
  int st = set_dev(e); if (st) return st;
  if ((st = upload_tides(e, istp0, n))) return st;
  const int p0 = e->parity;
  if (e->use_graph) {
    auto key = std::make_pair(n, p0);
    auto it = e->graphs.find(key);
    if (it == e->graphs.end()) {
      cudaGraph_t g;
      ECK(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
      st = launch_steps(e, n, p0);
      cudaError_t ce = cudaStreamEndCapture(e->stream, &g);
      if (st) { if (ce == cudaSuccess) cudaGraphDestroy(g); return st; }
      ECK(ce);
      cudaGraphExec_t ex;
      cudaError_t ie = cudaGraphInstantiate(&ex, g, 0);
      cudaGraphDestroy(g);
      ECK(ie);
      it = e->graphs.emplace(key, ex).first;
    }
    ECK(cudaGraphLaunch(it->second, e->stream));
  } else {
    if ((st = launch_steps(e, n, p0))) return st;
  }
  e->parity = (p0 + n) & 1;
  return NEMO_OK;
}

int nemo_ens_checksums(nemo_ens* e, double* out) {
  if (!e || !out) return NEMO_ERR_INVALID;
  int st = set_dev(e); if (st) return st;
  const int nm = (int)e->mem.size();
  k_ens_rows<<<dim3((unsigned)e->nrows, 3), CT, 0, e->stream>>>(e->d_mem, e->d_rows, e->nrows, e->parity, e->d_partial);
  ECK(cudaGetLastError());
  k_ens_cols<<<dim3((unsigned)nm, 3), CT, 0, e->stream>>>(e->d_row_off, e->d_row_cnt, e->d_partial, e->nrows, e->d_ck);
  ECK(cudaGetLastError());
  ECK(cudaMemcpyAsync(e->h_ck, e->d_ck, 3 * (size_t)nm * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
  ECK(cudaStreamSynchronize(e->stream));
  memcpy(out, e->h_ck, 3 * (size_t)nm * sizeof(double));
  return NEMO_OK;
}

int nemo_ens_retrieve(nemo_ens* e, int member, int field, double* host, long ld) {
  if (!e || !host || member < 0 || member >= (int)e->mem.size()) return NEMO_ERR_INVALID;
  const MemberDev& d = e->hmem[member];
  const double* src;
  int i0 = 1, j0 = 1, nx = d.L.jpi, ny = d.L.jpj;
  switch (field) {
    case NEMO_SSHN: src = d.st[e->parity][0]; break;
    case NEMO_UN: src = d.st[e->parity][1]; i0 = 0; nx = d.L.jpi + 1; break;
    case NEMO_VN: src = d.st[e->parity][2]; j0 = 0; ny = d.L.jpj + 1; break;
    case NEMO_HT: src = d.ht; break;
    case NEMO_HU: src = d.hu; i0 = 0; nx = d.L.jpi + 1; break;
    case NEMO_HV: src = d.hv; j0 = 0; ny = d.L.jpj + 1; break;
    default: return NEMO_ERR_INVALID;
  }
  if (ld < nx) return NEMO_ERR_INVALID;
  int st = set_dev(e); if (st) return st;
  ECK(cudaMemcpy2DAsync(host, (size_t)ld * sizeof(double), src + d.L.idx(i0, j0),
                        (size_t)d.L.pitch * sizeof(double), (size_t)nx * sizeof(double),
                        (size_t)ny, cudaMemcpyDeviceToHost, e->stream));
  ECK(cudaStreamSynchronize(e->stream));
  return NEMO_OK;
}

int nemo_ens_set_state(nemo_ens* e, int member, const double* sshn, const double* un,
                       const double* vn) {
  if (!e || !sshn || !un || !vn || member < 0 || member >= (int)e->mem.size()) return NEMO_ERR_INVALID;
  int st = set_dev(e); if (st) return st;
  const MemberDev& d = e->hmem[member];
  const Layout& L = d.L;
  const size_t P = (size_t)L.pitch * sizeof(double);
  ECK(cudaMemcpy2DAsync(d.st[e->parity][0] + L.idx(1, 1), P, sshn, (size_t)L.jpi * sizeof(double),
                        (size_t)L.jpi * sizeof(double), (size_t)L.jpj, cudaMemcpyHostToDevice, e->stream));
  ECK(cudaMemcpy2DAsync(d.st[e->parity][1] + L.idx(0, 1), P, un, (size_t)(L.jpi + 1) * sizeof(double),
                        (size_t)(L.jpi + 1) * sizeof(double), (size_t)L.jpj, cudaMemcpyHostToDevice, e->stream));
  ECK(cudaMemcpy2DAsync(d.st[e->parity][2] + L.idx(1, 0), P, vn, (size_t)L.jpi * sizeof(double),
                        (size_t)L.jpi * sizeof(double), (size_t)(L.jpj + 1), cudaMemcpyHostToDevice, e->stream));
  ECK(cudaStreamSynchronize(e->stream));
  return NEMO_OK;
}

int nemo_ens_set_schedule(nemo_ens* e, const nemo_ens_schedule* s) {
  if (!e) return NEMO_ERR_STATE;
  if (!s || !ens_variant_ok(s->warps, s->occupancy, e->recip_nr_ok) || s->rows < 1 || s->rows > 65536 ||
      s->order < 0 || s->order > 2 || s->ctas < 0)
    return NEMO_ERR_INVALID;
  int st = set_dev(e); if (st) return st;
  const bool rebuild = s->rows != e->sched.rows || s->order != e->sched.order;
  e->sched = *s;
  drop_graphs(e);
  // the dynamic schedule's counters start from zero whatever ran before
  ECK(cudaMemsetAsync(e->d_counter, 0, 4 * sizeof(int), e->stream));
  return rebuild ? build_work(e) : NEMO_OK;
}

int nemo_ens_get_schedule(nemo_ens* e, nemo_ens_schedule* s) {
  if (!e || !s) return NEMO_ERR_INVALID;
  *s = e->sched;
  return NEMO_OK;
}

int nemo_ens_use_graph(nemo_ens* e, int on) {
  if (!e) return NEMO_ERR_STATE;
  e->use_graph = on != 0;
  return NEMO_OK;
}

int nemo_ens_info(nemo_ens* e, int* nmem, long long* cells) {
  if (!e) return NEMO_ERR_STATE;
  if (nmem) *nmem = (int)e->mem.size();
  if (cells) *cells = e->cells;
  return NEMO_OK;
}

int nemo_ens_autotune(nemo_ens* e, int steps, nemo_ens_schedule* best, double* best_ms) {
  if (!e || steps < 1) return NEMO_ERR_INVALID;
  int st = set_dev(e); if (st) return st;
  // save every member's current state
  size_t tot = 0;
  for (auto& d : e->hmem) tot += 3 * (size_t)d.L.elems();
  double* backup = nullptr;
  ECK(nemo::dev_alloc(&backup, tot * sizeof(double)));
  const int p_save = e->parity;
  auto copy_state = [&](bool save) -> cudaError_t {
    size_t o = 0;
    for (auto& d : e->hmem) {
      const size_t b = (size_t)d.L.elems() * sizeof(double);
      for (int f = 0; f < 3; ++f) {
        double* dev = d.st[p_save][f];
        cudaError_t er = save ? cudaMemcpyAsync(backup + o, dev, b, cudaMemcpyDeviceToDevice, e->stream)
                              : cudaMemcpyAsync(dev, backup + o, b, cudaMemcpyDeviceToDevice, e->stream);
        if (er != cudaSuccess) return er;
        o += (size_t)d.L.elems();
      }
    }
    return cudaSuccess;
  };
  cudaError_t er = copy_state(true);
  const nemo_ens_schedule keep = e->sched;
  const bool keep_graph = e->use_graph;
  e->use_graph = false;
  nemo_ens_schedule bsched = keep;
  double bms = 1e300;
  const int warps_occ[][2] = {{2, 216}, {2, 220}, {4, 216}, {2, 212}, {4, 212}, {2, 116}, {2, 120}, {4, 116}, {2, -24},
                              {2, -20}, {2, 20}, {2, 24}, {4, -20}, {4, 20}, {4, 24}};
  const int rows_c[] = {8, 16, 32, 64, 128};
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  if (er == cudaSuccess) er = cudaEventCreate(&t0);
  if (er == cudaSuccess) er = cudaEventCreate(&t1);
  for (const auto& wo : warps_occ) {
    if (!ens_variant_ok(wo[0], wo[1], e->recip_nr_ok)) continue;
    for (int rows : rows_c) {
      for (int order = 0; order <= 2 && er == cudaSuccess; ++order) {
        if ((rows > 32) != (order == 2)) continue;  // tall blocks need the dynamic schedule
        nemo_ens_schedule c{wo[0], wo[1], rows, order, 0};
        if ((st = nemo_ens_set_schedule(e, &c))) break;
        nemo_ens_step_n(e, 1, 1);  // warm
        er = cudaEventRecord(t0, e->stream);
        if (er == cudaSuccess && (st = nemo_ens_step_n(e, 2, steps))) break;
        if (er == cudaSuccess) er = cudaEventRecord(t1, e->stream);
        if (er == cudaSuccess) er = cudaEventSynchronize(t1);
        float ms = 0.f;
        if (er == cudaSuccess) er = cudaEventElapsedTime(&ms, t0, t1);
        if (er == cudaSuccess && ms / steps < bms) {
          bms = ms / steps;
          bsched = c;
        }
      }
      if (st || er != cudaSuccess) break;
    }
    if (st || er != cudaSuccess) break;
  }
  if (t0) cudaEventDestroy(t0);
  if (t1) cudaEventDestroy(t1);
  e->parity = p_save;
  cudaError_t er2 = copy_state(false);
  if (er == cudaSuccess) er = er2;
  if (er == cudaSuccess) er = cudaStreamSynchronize(e->stream);
  cudaFree(backup);
  e->use_graph = keep_graph;
  if (st == NEMO_OK && er == cudaSuccess) st = nemo_ens_set_schedule(e, bms < 1e300 ? &bsched : &keep);
  if (er != cudaSuccess) return status_of(er);
  if (st) return st;
  if (best) *best = e->sched;
  if (best_ms) *best_ms = bms;
  return NEMO_OK;
}

}  // extern "C"

// ---- accessors for the surrogate and hybrid controller (same library) ----
namespace nemo {

int ens_member_state(nemo_ens* e, int m, MemberState* out) {
  if (!e || !out || m < 0 || m >= (int)e->mem.size()) return NEMO_ERR_INVALID;
  const MemberDev& d = e->hmem[m];
  out->sshn = d.st[e->parity][0];
  out->un = d.st[e->parity][1];
  out->vn = d.st[e->parity][2];
  out->ht = d.ht;
  out->hv = d.hv;
  out->sshv0 = d.sshv0;
  out->jpi = d.L.jpi;
  out->jpj = d.L.jpj;
  out->pitch = d.L.pitch;
  out->corr = nullptr;
  return NEMO_OK;
}

int ens_member_count(nemo_ens* e) { return e ? (int)e->mem.size() : 0; }

// Advances the members with sel[m] != 0 by n steps (direct launches over a
// work list of those members only); the others keep their state.  n must be
// even: every member then still holds its current state in the buffer set
// the ensemble's parity names.
int ens_step_subset(nemo_ens* e, int istp0, int n, const char* sel) {
  if (!e || !sel || n < 0 || (n & 1)) return NEMO_ERR_INVALID;
  if (n == 0) return NEMO_OK;
  int st = set_dev(e); if (st) return st;
  const std::vector<int4> w = work_items(e, sel);
  if (w.empty()) return NEMO_OK;
  if ((int)w.size() > e->sub_cap) {
    ECK(cudaStreamSynchronize(e->stream));
    if (e->d_work_sub) cudaFree(e->d_work_sub);
    e->d_work_sub = nullptr;
    e->sub_cap = 0;
    ECK(nemo::dev_alloc(&e->d_work_sub, w.size() * sizeof(int4)));
    e->sub_cap = (int)w.size();
  }
  // pageable source: the copy is staged before the call returns
  ECK(cudaMemcpyAsync(e->d_work_sub, w.data(), w.size() * sizeof(int4), cudaMemcpyHostToDevice, e->stream));
  if ((st = upload_tides(e, istp0, n))) return st;
  const size_t nm = e->mem.size();
  for (int k = 0; k < n; ++k)
    ECK(launch_ens(e->sched.warps, e->sched.occupancy, e->d_mem, e->d_work_sub, (int)w.size(), e->C,
                   e->d_tide + (size_t)k * nm, (e->parity + k) & 1, e->sched.ctas, counter_of(e, true),
                   e->stream));
  return NEMO_OK;
}
cudaStream_t ens_stream(nemo_ens* e) { return e->stream; }
int ens_device(nemo_ens* e) { return e->device; }

double ens_amp(nemo_ens* e, int m) { return fabs(e->mem[m].amp_tide); }

double ens_tide(nemo_ens* e, int m, int istp) {
  const double omega_tide = 2.0 * 3.14159 / (12.42 * 3600.0);
  const double rtime = (double)istp * e->common.rdt;
  return e->mem[m].amp_tide * sin(omega_tide * rtime + e->mem[m].tide_phase);
}

}  // namespace nemo
