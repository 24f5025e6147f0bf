// nemolite2d -- host driver for the B200 stepper.
//
// The program of original/nemolite2d.f90 (PROGRAM nemolite2d, :1-90) on top
// of the C ABI in include/nemo_b200.h:
//   setup           read &namctl from ./namelist (or argv[1]), echo it,
//                   jpi = jpiglo-2, jpj = jpjglo-2               (:96-141)
//   grid/init       nemo_create                                  (:145-371)
//   output(0)       go2d_00000.dat                                (:67-68)
//                   (records are staged on the device and copied back on a
//                   side stream, nemo_record; a writer thread formats the
//                   files while the stepper continues; x, y and depth are
//                   read back once)
//   DO istp        step: continuity, momentum, bc(rtime), next;  (:74-77,
//                   output and checksums every irecord steps       :375-386)
//   end            'ua checksum = ' / 'va checksum = ' (E16.8)    (:82-85)
//                   and a dl_timer-style report (shared/dl_timer
//                   dl_timer.f90:713-773) with the regions Time-stepping,
//                   Continuity, Momentum, BCs, Next.
//
// Extension keys accepted in &namctl (defaults reproduce the reference):
//   amp_tide, tide_phase, lat, nbump, seed, bump_amp, bump_wmin, bump_wmax,
//   hmin, hmax   -- physics/bathymetry (see nemo_params)
//   fused        -- .true.: one fused launch per step (nemo_step_n) between
//                   records instead of the four routine calls
//   write_dat    -- .false. skips the go2d_*.dat files
//   cta_warps, occupancy, rows -- fused kernel schedule (nemo_schedule);
//   checksum_csv -- file for the per-record checksums (default checksums.csv)
//
// Flags: --echo-namelist parses, echoes and exits (no GPU needed).
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <cctype>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "nemo_b200.h"

namespace {

// ---- Fortran-style formatting ---------------------------------------------
// Ew.d (exponent digits e): 0.ddddE+xx right-justified in w characters.
std::string fortran_E(double v, int w, int d, int e = 2) {
  std::string out;
  if (std::isnan(v)) {
    out = "NaN";
  } else if (std::isinf(v)) {
    out = v < 0 ? "-Infinity" : "Infinity";
  } else {
    bool neg = std::signbit(v) && v != 0.0;
    double a = fabs(v);
    int ex = 0;
    std::string digits(d, '0');
    if (a != 0.0) {
      char buf[64];
      snprintf(buf, sizeof buf, "%.*e", d - 1, a);  // correctly rounded d digits
      std::string s(buf);
      size_t epos = s.find('e');
      std::string mant = s.substr(0, epos);
      ex = atoi(s.c_str() + epos + 1) + 1;
      mant.erase(std::remove(mant.begin(), mant.end(), '.'), mant.end());
      digits = mant.substr(0, d);
    }
    char eb[16];
    int ae = abs(ex);
    if (e == 2 && ae > 99)
      snprintf(eb, sizeof eb, "%c%03d", ex < 0 ? '-' : '+', ae);  // Fortran drops the 'E'
    else
      snprintf(eb, sizeof eb, "E%c%0*d", ex < 0 ? '-' : '+', e, ae);
    out = std::string(neg ? "-" : "") + "0." + digits + eb;
  }
  if ((int)out.size() < w) out = std::string(w - out.size(), ' ') + out;
  return out;
}

// ---- namelist --------------------------------------------------------------
struct Namelist {
  std::map<std::string, std::string> kv;
  bool has(const std::string& k) const { return kv.count(k) != 0; }
  double real(const std::string& k, double def) const {
    auto it = kv.find(k);
    if (it == kv.end()) return def;
    std::string s = it->second;
    for (auto& ch : s)
      if (ch == 'd' || ch == 'D') ch = 'e';
    return strtod(s.c_str(), nullptr);
  }
  long integer(const std::string& k, long def) const {
    auto it = kv.find(k);
    return it == kv.end() ? def : strtol(it->second.c_str(), nullptr, 10);
  }
  bool logical(const std::string& k, bool def) const {
    auto it = kv.find(k);
    if (it == kv.end()) return def;
    std::string s = it->second;
    for (auto& ch : s) ch = (char)tolower(ch);
    if (!s.empty() && s[0] == '.') s = s.substr(1);
    return !s.empty() && s[0] == 't';
  }
};

// Parses the group &namctl ... / of a Fortran namelist file.  Returns false
// when the group is missing or malformed (the reference STOPs with
// "err found in reading namelist file", original/nemolite2d.f90:122-123).
bool read_namelist(const std::string& path, Namelist& nl, std::string& err) {
  std::ifstream f(path);
  if (!f) {
    err = "cannot open " + path;
    return false;
  }
  std::stringstream ss;
  std::string line;
  bool in = false, done = false;
  while (std::getline(f, line)) {
    size_t bang = line.find('!');
    if (bang != std::string::npos) line = line.substr(0, bang);
    std::string low = line;
    for (auto& ch : low) ch = (char)tolower(ch);
    if (!in) {
      size_t a = low.find("&namctl");
      if (a == std::string::npos) continue;
      in = true;
      line = line.substr(a + 7);
      low = low.substr(a + 7);
    }
    size_t slash = low.find('/');
    if (slash != std::string::npos) {
      ss << line.substr(0, slash) << '\n';
      done = true;
      break;
    }
    ss << line << '\n';
  }
  if (!in || !done) {
    err = "group &namctl not found or not terminated";
    return false;
  }
  std::string body = ss.str();
  for (auto& ch : body)
    if (ch == ',' || ch == '\n' || ch == '\t' || ch == '\r') ch = ' ';
  // tokens: key = value
  std::vector<std::string> tok;
  {
    std::string cur;
    for (char ch : body) {
      if (ch == '=') {
        if (!cur.empty()) tok.push_back(cur);
        tok.push_back("=");
        cur.clear();
      } else if (ch == ' ') {
        if (!cur.empty()) tok.push_back(cur);
        cur.clear();
      } else {
        cur += ch;
      }
    }
    if (!cur.empty()) tok.push_back(cur);
  }
  for (size_t k = 0; k < tok.size(); ++k) {
    if (k + 2 < tok.size() + 0 && tok[k + 1] == "=" && tok[k] != "=") {
      std::string key = tok[k];
      for (auto& ch : key) ch = (char)tolower(ch);
      if (k + 2 >= tok.size() || tok[k + 2] == "=") {
        err = "missing value for " + key;
        return false;
      }
      nl.kv[key] = tok[k + 2];
      k += 2;
    } else if (tok[k] == "=") {
      err = "malformed entry";
      return false;
    }
  }
  return true;
}

const char* KNOWN[] = {"jpiglo", "jpjglo", "jphgr_msh", "dx", "dy", "dep_const", "nit000",
                       "nitend", "irecord", "rdt", "cbfr", "visc", "amp_tide", "tide_phase",
                       "lat", "nbump", "seed", "bump_amp", "bump_wmin", "bump_wmax", "hmin",
                       "hmax", "fused", "write_dat", "cta_warps", "occupancy", "rows", "checksum_csv"};

struct Setup {
  long jpiglo, jpjglo, jphgr_msh, nit000, nitend, irecord;
  double dx, dy, dep_const, rdt, cbfr, visc;
  bool fused, write_dat;
  nemo_schedule sched;
  bool has_sched;
  std::string csv;
  nemo_params p;
};

std::string list_real(double v) {
  char b[64];
  snprintf(b, sizeof b, "%25.17g", v);
  return b;
}

void echo_namelist(const Setup& s) {
  // WRITE(*, NML=namctl), original/nemolite2d.f90:124
  printf("&NAMCTL\n");
  printf(" JPIGLO=%-11ld,\n", s.jpiglo);
  printf(" JPJGLO=%-11ld,\n", s.jpjglo);
  printf(" JPHGR_MSH=%-11ld,\n", s.jphgr_msh);
  printf(" DX=%s,\n", list_real(s.dx).c_str());
  printf(" DY=%s,\n", list_real(s.dy).c_str());
  printf(" DEP_CONST=%s,\n", list_real(s.dep_const).c_str());
  printf(" NIT000=%-11ld,\n", s.nit000);
  printf(" NITEND=%-11ld,\n", s.nitend);
  printf(" IRECORD=%-11ld,\n", s.irecord);
  printf(" RDT=%s,\n", list_real(s.rdt).c_str());
  printf(" CBFR=%s,\n", list_real(s.cbfr).c_str());
  printf(" VISC=%s,\n", list_real(s.visc).c_str());
  printf(" /\n");
}

bool setup(const std::string& path, Setup& s) {
  Namelist nl;
  std::string err;
  if (!read_namelist(path, nl, err)) {
    fprintf(stderr, "%s\n", err.c_str());
    printf("err found in reading namelist file\n");
    return false;
  }
  for (auto& kv : nl.kv) {
    bool ok = false;
    for (const char* k : KNOWN) ok = ok || kv.first == k;
    if (!ok) {
      fprintf(stderr, "unknown namelist key %s\n", kv.first.c_str());
      printf("err found in reading namelist file\n");
      return false;
    }
  }
  // defaults, original/nemolite2d.f90:107-118
  s.jpiglo = nl.integer("jpiglo", 258);
  s.jpjglo = nl.integer("jpjglo", 258);
  s.jphgr_msh = nl.integer("jphgr_msh", 1);
  s.dx = nl.real("dx", 1000.0);
  s.dy = nl.real("dy", 1000.0);
  s.dep_const = nl.real("dep_const", 100.0);
  s.nit000 = nl.integer("nit000", 1);
  s.nitend = nl.integer("nitend", 1000);
  s.irecord = nl.integer("irecord", 1);
  if (s.irecord < 1) {
    // the step loop takes MOD(istp, irecord) (original/nemolite2d.f90:384),
    // which has no value for irecord <= 0
    fprintf(stderr, "irecord = %ld: the output interval must be at least 1\n", s.irecord);
    printf("err found in reading namelist file\n");
    return false;
  }
  s.rdt = nl.real("rdt", 10.0);
  s.cbfr = nl.real("cbfr", 0.001);
  s.visc = nl.real("visc", 100.0);
  s.fused = nl.logical("fused", false);
  s.write_dat = nl.logical("write_dat", true);
  s.has_sched = nl.has("cta_warps") || nl.has("occupancy") || nl.has("rows");
  s.sched.warps = (int)nl.integer("cta_warps", 4);
  s.sched.occupancy = (int)nl.integer("occupancy", 0);
  s.sched.rows = (int)nl.integer("rows", 64);
  s.csv = nl.has("checksum_csv") ? nl.kv["checksum_csv"] : "checksums.csv";
  s.csv.erase(std::remove(s.csv.begin(), s.csv.end(), '\''), s.csv.end());
  s.csv.erase(std::remove(s.csv.begin(), s.csv.end(), '"'), s.csv.end());
  nemo_default_params(&s.p);
  s.p.jpi = (int)(s.jpiglo - 2);  // :133-137
  s.p.jpj = (int)(s.jpjglo - 2);
  s.p.dx = s.dx;
  s.p.dy = s.dy;
  s.p.dep_const = s.dep_const;
  s.p.nit000 = (int)s.nit000;
  s.p.nitend = (int)s.nitend;
  s.p.irecord = (int)s.irecord;
  s.p.rdt = s.rdt;
  s.p.cbfr = s.cbfr;
  s.p.visc = s.visc;
  s.p.amp_tide = nl.real("amp_tide", s.p.amp_tide);
  s.p.tide_phase = nl.real("tide_phase", s.p.tide_phase);
  s.p.lat = nl.real("lat", s.p.lat);
  s.p.nbump = (int)nl.integer("nbump", s.p.nbump);
  s.p.seed = (uint64_t)nl.integer("seed", (long)s.p.seed);
  s.p.bump_amp = nl.real("bump_amp", s.p.bump_amp);
  s.p.bump_wmin = nl.real("bump_wmin", s.p.bump_wmin);
  s.p.bump_wmax = nl.real("bump_wmax", s.p.bump_wmax);
  s.p.hmin = nl.real("hmin", s.p.hmin);
  s.p.hmax = nl.real("hmax", s.p.hmax);
  return true;
}

// ---- dl_timer-style region timers -----------------------------------------
struct Region {
  std::string label;
  long nrepeat = 1;
  std::vector<double> samples;
  double total() const {
    double t = 0.0;
    for (double x : samples) t += x;
    return t;
  }
};

struct Timers {
  std::vector<Region> r;
  int idx(const std::string& label, long nrep = 1) {
    for (size_t k = 0; k < r.size(); ++k)
      if (r[k].label == label) return (int)k;
    Region g;
    g.label = label;
    g.nrepeat = nrep;
    r.push_back(g);
    return (int)r.size() - 1;
  }
  void report() const {
    // timer_report_with_repeats layout (dl_timer.f90:713-773, :874-909)
    const int width = 88;
    printf("\n%s Timing report %s\n", std::string((width - 15) / 2, '=').c_str(),
           std::string((width - 15) / 2, '=').c_str());
    printf("Timed using std::chrono::steady_clock after a device synchronise. Units are seconds.\n");
    printf("%s\n", std::string(width, '-').c_str());
    printf("Region                          Counts      Total       Average*   Avg/repeat*  Std Err\n");
    printf("%s\n", std::string(width, '-').c_str());
    for (const Region& g : r) {
      long n = (long)g.samples.size();
      double tot = g.total();
      double mean = n ? tot / n : 0.0;
      double rep = mean / (double)g.nrepeat;
      double var = 0.0;
      for (double x : g.samples) var += (x - mean) * (x - mean);
      double err = n > 1 ? sqrt(var / (n - 1) / n) : 0.0;
      double terr = mean > 0 ? rep * err / mean : 0.0;
      std::string lab = g.label;
      lab.resize(32, ' ');
      printf("%s %6ld %s %s %s %s\n", lab.c_str(), n, fortran_E(tot, 12, 5).c_str(),
             fortran_E(mean, 12, 5).c_str(), fortran_E(rep, 12, 5).c_str(),
             fortran_E(terr, 9, 2).c_str());
    }
    printf("%s\n", std::string(width, '-').c_str());
    printf("* corrected for systematic error\n");
    printf("%s\n\n", std::string(width, '=').c_str());
  }
};

double now_s() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

int check(int st, const char* where) {
  if (st != NEMO_OK) {
    fprintf(stderr, "%s: %s\n", where, nemo_status_string(st));
    exit(2);
  }
  return st;
}

// output, original/nemolite2d.f90:773-799: go2d_%05d.dat, 6E20.7E4 per row,
// a blank line after each jj.  rec holds sshn and the cell-centred u, v as
// three [jpj][jpi] planes (nemo_record); xt, yt, ht are static.
void write_dat(int istp, int jpi, int jpj, const std::vector<double>& xt, const std::vector<double>& yt,
               const std::vector<double>& ht, const double* rec) {
  char name[32];
  snprintf(name, sizeof name, "go2d_%05d.dat", istp);
  FILE* f = fopen(name, "w");
  if (!f) {
    fprintf(stderr, "cannot write %s\n", name);
    return;
  }
  const size_t plane = (size_t)jpi * jpj;
  std::string line;
  for (int jj = 1; jj <= jpj; ++jj) {
    for (int ji = 1; ji <= jpi; ++ji) {
      const size_t t = (size_t)(jj - 1) * jpi + (ji - 1);
      line = fortran_E(xt[t], 20, 7, 4) + fortran_E(yt[t], 20, 7, 4) + fortran_E(ht[t], 20, 7, 4) +
             fortran_E(rec[t], 20, 7, 4) + fortran_E(rec[plane + t], 20, 7, 4) +
             fortran_E(rec[2 * plane + t], 20, 7, 4);
      fputs(line.c_str(), f);
      fputc('\n', f);
    }
    fputc('\n', f);
  }
  fclose(f);
}

// Records in flight: two page-locked buffers; the main thread starts a
// record into a free buffer and queues it, the writer thread waits for the
// copy and writes the file, then frees the buffer.
struct Writer {
  nemo_ctx* c;
  int jpi, jpj;
  std::vector<double> xt, yt, ht;
  double* buf[2] = {nullptr, nullptr};
  bool busy[2] = {false, false};
  int next = 0;
  std::deque<std::pair<int, int>> jobs;  // (istp, buffer)
  bool done = false;
  std::mutex mu;
  std::condition_variable cv;
  std::thread th;

  Writer(nemo_ctx* c_, int jpi_, int jpj_) : c(c_), jpi(jpi_), jpj(jpj_) {
    const size_t n = (size_t)jpi * jpj;
    xt.resize(n);
    yt.resize(n);
    ht.resize(n);
    check(nemo_retrieve(c, NEMO_XT, xt.data(), jpi), "retrieve xt");
    check(nemo_retrieve(c, NEMO_YT, yt.data(), jpi), "retrieve yt");
    check(nemo_retrieve(c, NEMO_HT, ht.data(), jpi), "retrieve ht");
    for (auto& b : buf) check(nemo_host_alloc(3 * n * sizeof(double), reinterpret_cast<void**>(&b)), "nemo_host_alloc");
    th = std::thread([this] { run(); });
  }
  ~Writer() {
    {
      std::lock_guard<std::mutex> lk(mu);
      done = true;
    }
    cv.notify_all();
    th.join();
    for (auto* b : buf) nemo_host_free(b);
  }
  void record(int istp) {
    int b;
    {
      std::unique_lock<std::mutex> lk(mu);
      cv.wait(lk, [&] { return !busy[next]; });
      b = next;
      busy[b] = true;
      next ^= 1;
    }
    check(nemo_record(c, buf[b]), "nemo_record");
    {
      std::lock_guard<std::mutex> lk(mu);
      jobs.emplace_back(istp, b);
    }
    cv.notify_all();
  }
  void run() {
    for (;;) {
      std::pair<int, int> job;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [&] { return done || !jobs.empty(); });
        if (jobs.empty()) return;
        job = jobs.front();
        jobs.pop_front();
      }
      check(nemo_record_wait(c), "nemo_record_wait");  // copies land in order
      write_dat(job.first, jpi, jpj, xt, yt, ht, buf[job.second]);
      {
        std::lock_guard<std::mutex> lk(mu);
        busy[job.second] = false;
      }
      cv.notify_all();
    }
  }
};

}  // namespace

int main(int argc, char** argv) {
  bool echo_only = false;
  std::string path = "namelist";
  for (int k = 1; k < argc; ++k) {
    std::string a = argv[k];
    if (a == "--echo-namelist")
      echo_only = true;
    else
      path = a;
  }
  Setup s;
  if (!setup(path, s)) return 1;
  echo_namelist(s);
  if (echo_only) return 0;
  if (s.jphgr_msh == 0) {
    printf("It is not ready to Read in grid from a file\n");  // :155-158
    return 1;
  }
  if (s.jphgr_msh != 1) {
    printf("Wrong grid defination type, check your setup !!!!\n");  // :256-259
    return 1;
  }
  const int jpi = s.p.jpi, jpj = s.p.jpj;
  nemo_ctx* c = nullptr;
  check(nemo_create(&s.p, &c), "nemo_create");
  if (s.has_sched) check(nemo_set_schedule(c, &s.sched), "nemo_set_schedule");
  Writer* writer = s.write_dat ? new Writer(c, jpi, jpj) : nullptr;
  if (writer) writer->record(0);
  FILE* csv = fopen(s.csv.c_str(), "w");
  if (csv) fprintf(csv, "istp,ssh_checksum,ua_checksum,va_checksum\n");

  Timers T;
  const long nsteps = s.nitend - s.nit000 + 1;
  int it_step = T.idx("Time-stepping", nsteps > 0 ? nsteps : 1);
  int it_c = -1, it_m = -1, it_b = -1, it_n = -1, it_f = -1;
  if (s.fused) {
    it_f = T.idx("Fused step");
  } else {
    it_c = T.idx("Continuity");
    it_m = T.idx("Momentum");
    it_b = T.idx("BCs");
    it_n = T.idx("Next");
  }
  auto record = [&](long istp) {
    double ck[3];
    check(nemo_checksums(c, ck), "nemo_checksums");
    printf(" istp=%8ld ssh checksum =%s ua checksum =%s va checksum =%s\n", istp,
           fortran_E(ck[0], 16, 8).c_str(), fortran_E(ck[1], 16, 8).c_str(),
           fortran_E(ck[2], 16, 8).c_str());
    if (csv) fprintf(csv, "%ld,%.17e,%.17e,%.17e\n", istp, ck[0], ck[1], ck[2]);
    if (!(std::isfinite(ck[0]) && std::isfinite(ck[1]) && std::isfinite(ck[2])))
      fprintf(stderr, "warning: non-finite checksum at istp=%ld (the state has diverged)\n", istp);
    if (writer) writer->record((int)istp);
  };

  check(nemo_sync(c), "nemo_sync");
  double t0 = now_s();
  if (s.fused) {
    long istp = s.nit000;
    while (istp <= s.nitend) {
      long next_rec = ((istp + s.irecord - 1) / s.irecord) * s.irecord;  // first multiple >= istp
      if (next_rec < istp) next_rec = istp;
      long last = std::min(next_rec, s.nitend);
      double a = now_s();
      check(nemo_step_n(c, (int)istp, (int)(last - istp + 1)), "nemo_step_n");
      check(nemo_sync(c), "nemo_sync");
      T.r[it_f].samples.push_back(now_s() - a);
      if (last % s.irecord == 0) record(last);
      istp = last + 1;
    }
  } else {
    for (long istp = s.nit000; istp <= s.nitend; ++istp) {
      double rtime = (double)istp * s.rdt;  // :378
      double a = now_s();
      check(nemo_continuity(c), "nemo_continuity");
      check(nemo_sync(c), "sync");
      double b = now_s();
      check(nemo_momentum(c), "nemo_momentum");
      check(nemo_sync(c), "sync");
      double d = now_s();
      check(nemo_bc(c, rtime), "nemo_bc");
      check(nemo_sync(c), "sync");
      double e = now_s();
      check(nemo_next(c), "nemo_next");
      check(nemo_sync(c), "sync");
      double f = now_s();
      T.r[it_c].samples.push_back(b - a);
      T.r[it_m].samples.push_back(d - b);
      T.r[it_b].samples.push_back(e - d);
      T.r[it_n].samples.push_back(f - e);
      if (istp % s.irecord == 0) record(istp);
    }
  }
  check(nemo_sync(c), "nemo_sync");
  T.r[it_step].samples.push_back(now_s() - t0);
  delete writer;  // the last files are written before the report
  if (csv) fclose(csv);

  // :82-85, field_checksum(ua(1:jpiglo,1:jpjglo)) -- ua == un after next
  double ua, va;
  check(nemo_checksum(c, NEMO_UA, &ua), "checksum ua");
  check(nemo_checksum(c, NEMO_VA, &va), "checksum va");
  printf("ua checksum = %s\n", fortran_E(ua, 16, 8).c_str());
  printf("va checksum = %s\n", fortran_E(va, 16, 8).c_str());
  nemo_destroy(c);
  T.report();
  printf(" Simulation finished!!\n");
  return 0;
}
