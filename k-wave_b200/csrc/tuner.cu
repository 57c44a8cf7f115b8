// Launch-schedule tuner and its wisdom cache.
//
// The time step can be launched several ways that give bit-identical
// results: the y-inverse / row kernel / y-forward chains whole or split into
// z slabs, the slabs one after another on one stream or alternating between
// two (one slab's latency-bound row kernel then runs beside the other's
// bandwidth-bound y passes), and, for lengths served by the runtime-plan FFT
// engine, the number of lines each row or column block transforms.  That
// engine's radix order can be chosen too; another order rounds differently
// (FP32 rounding, far inside the solver's tolerance), and once chosen it is
// kept for the key, so the runs of a process agree bit for bit.  Which is
// fastest depends on the grid and on the step's kernels, so the tuner times
// the candidates on a scratch copy of the simulation (same grid, medium,
// sources, sensor reductions; no recorded series) and keeps the fastest in a
// per-process table keyed by grid, step class and device, the way FFTW keeps
// plans as wisdom.  Sessions created later for the same key use it; the
// table can be written to and read from a text file (KWAVE_B200_WISDOM), so
// a binary started once per simulation reuses what an earlier run measured.
#include <cuda_runtime.h>
#include <unistd.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "kwave_b200.h"
#include "solver_internal.h"

namespace kwb {

bool ct_supported(int n);  // kernels.cu: a compile-time FFT kernel exists for length n

namespace {

std::mutex g_mu;
std::map<std::string, std::pair<Schedule, float>> g_wisdom;  // key -> (schedule, ms per step)
bool g_env_loaded = false;
thread_local bool g_tuning = false;  // set while a scratch session is timed

void cuda_ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw KwError(KW_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

int env_int(const char* name) {
  const char* v = std::getenv(name);
  return v ? std::atoi(v) : 0;
}

// Parse wisdom lines "<key> <slab> <streams> <row_lines> <col_lines> <radix>
// <ms>" into `into`; '#' lines are comments.  Returns the entries read.
int parse_wisdom(std::istream& is, std::map<std::string, std::pair<Schedule, float>>& into) {
  std::string line;
  int n = 0;
  while (std::getline(is, line)) {
    if (line.empty() || line[0] == '#') continue;
    std::istringstream ls(line);
    std::vector<std::string> tok;
    for (std::string t; ls >> t;) tok.push_back(t);
    if (tok.empty()) continue;
    Schedule s;
    float ms = 0.f;
    // whole-token integers and a number: "1.0" is not a schedule field
    auto to_int = [&](const std::string& t) {
      size_t used = 0;
      int v = 0;
      try {
        v = std::stoi(t, &used);
      } catch (const std::exception&) {
        used = 0;
      }
      if (used != t.size() || t.empty()) throw KwError(KW_ERR_IO, "malformed wisdom line: " + line);
      return v;
    };
    if (tok.size() != 7) throw KwError(KW_ERR_IO, "malformed wisdom line: " + line);
    const std::string key = tok[0];
    s.slab = to_int(tok[1]);
    s.streams = to_int(tok[2]);
    s.row_lines = to_int(tok[3]);
    s.col_lines = to_int(tok[4]);
    s.radix = to_int(tok[5]);
    try {
      size_t used = 0;
      ms = std::stof(tok[6], &used);
      if (used != tok[6].size()) throw std::invalid_argument("trailing");
    } catch (const std::exception&) {
      throw KwError(KW_ERR_IO, "malformed wisdom line: " + line);
    }
    if (s.slab < 1 || s.streams < 1 || s.streams > 2 || s.row_lines < 1 || s.col_lines < 1 || s.radix < 0 ||
        s.radix > 2)
      throw KwError(KW_ERR_IO, "wisdom entry out of range: " + line);
    into[key] = {s, ms};
    ++n;
  }
  return n;
}

int import_file(const std::string& path, bool missing_ok) {
  std::ifstream f(path);
  if (!f) {
    if (missing_ok) return 0;
    throw KwError(KW_ERR_IO, "cannot open wisdom file " + path);
  }
  std::map<std::string, std::pair<Schedule, float>> read;
  const int n = parse_wisdom(f, read);
  for (auto& kv : read) g_wisdom[kv.first] = kv.second;
  return n;
}

// Entries of the file (if any) overlaid with the table, written to a
// temporary file and renamed over the path.
void export_file(const std::string& path) {
  std::map<std::string, std::pair<Schedule, float>> all;
  {
    std::ifstream f(path);
    if (f) parse_wisdom(f, all);
  }
  for (auto& kv : g_wisdom) all[kv.first] = kv.second;
  const std::string tmp = path + ".tmp." + std::to_string((long)getpid());  // one per writing process
  {
    std::ofstream o(tmp);
    if (!o) throw KwError(KW_ERR_IO, "cannot write wisdom file " + tmp);
    o << "# kwave_b200 launch-schedule wisdom: key slab_planes streams row_lines col_lines radix_plan ms_per_step\n";
    for (auto& kv : all) {
      const Schedule& s = kv.second.first;
      o << kv.first << ' ' << s.slab << ' ' << s.streams << ' ' << s.row_lines << ' ' << s.col_lines << ' '
        << s.radix << ' ' << kv.second.second << '\n';
    }
    if (!o) throw KwError(KW_ERR_IO, "cannot write wisdom file " + tmp);
  }
  if (std::rename(tmp.c_str(), path.c_str()) != 0) throw KwError(KW_ERR_IO, "cannot replace wisdom file " + path);
}

void load_env_once() {
  // g_mu held
  if (g_env_loaded) return;
  g_env_loaded = true;
  const char* p = std::getenv("KWAVE_B200_WISDOM");
  if (p && *p) import_file(p, /*missing_ok=*/true);
}

bool lookup(const std::string& key, Schedule* s) {
  std::lock_guard<std::mutex> lk(g_mu);
  load_env_once();
  auto it = g_wisdom.find(key);
  if (it == g_wisdom.end()) return false;
  *s = it->second.first;
  return true;
}

void remember(const std::string& key, const Schedule& s, float ms) {
  std::lock_guard<std::mutex> lk(g_mu);
  load_env_once();
  g_wisdom[key] = {s, ms};
  const char* p = std::getenv("KWAVE_B200_WISDOM");
  if (p && *p) export_file(p);
}

Schedule normalise(Schedule s, const Dims& d, int row_max) {
  s.slab = std::max(1, std::min(s.slab, d.nz));
  const int nslab = (d.nz + s.slab - 1) / s.slab;
  s.slab = (d.nz + nslab - 1) / nslab;  // equal slabs
  s.streams = (nslab > 1 && s.streams >= 2) ? 2 : 1;
  s.row_lines = std::max(1, std::min(s.row_lines, row_max));
  s.col_lines = std::max(1, std::min(s.col_lines, 16));
  s.radix = std::max(0, std::min(s.radix, 2));
  return s;
}

int row_lines_max(const Dims& d) { return std::max(1, std::min(8, 2048 / d.nx)); }

}  // namespace

// Two slabs on two streams for large 3D grids, the whole volume otherwise.
// Measured on 256^3: two slabs one after another lose more to partial waves
// than the L2 reuse of a slab's half spectra gains (1.406 against 1.340 ms
// per step), two slabs on two streams win (1.299 ms), four slabs on two
// streams 1.347 ms.
Schedule Session::default_schedule() const {
  Schedule s;
  const bool big = d.dim == 3 && d.npts >= (1LL << 22) && d.nz >= 64;
  s.slab = big ? (d.nz + 1) / 2 : d.nz;
  s.streams = big ? 2 : 1;
  s.row_lines = row_lines_max(d);
  s.col_lines = 16;
  return normalise(s, d, row_lines_max(d));
}

bool Session::runtime_rows() const { return !ct_supported(d.nx); }

bool Session::runtime_cols() const {
  const int ns[3] = {d.nx, d.ny, d.nz};
  for (int a = 1; a < d.dim; ++a)
    if (!ct_supported(ns[a])) return true;
  return false;
}

void Session::set_schedule(const Schedule& s0) {
  const Schedule s = normalise(s0, d, row_lines_max(d));
  cuda_ck(cudaStreamSynchronize(st), "sync");
  if (st2) cuda_ck(cudaStreamSynchronize(st2), "sync");
  // the captured step holds the old launch shapes
  if (graph_exec) cuda_ck(cudaGraphExecDestroy(graph_exec), "cudaGraphExecDestroy");
  if (graph) cuda_ck(cudaGraphDestroy(graph), "cudaGraphDestroy");
  graph_exec = nullptr;
  graph = nullptr;
  if (s.streams == 2 && !st2) {
    int lo = 0, hi = 0;
    cuda_ck(cudaDeviceGetStreamPriorityRange(&lo, &hi), "stream priority range");
    cuda_ck(cudaStreamCreateWithPriority(&st2, cudaStreamNonBlocking, lo), "cudaStreamCreate");
    cuda_ck(cudaEventCreateWithFlags(&fork_ev, cudaEventDisableTiming), "cudaEventCreate");
    cuda_ck(cudaEventCreateWithFlags(&join_ev, cudaEventDisableTiming), "cudaEventCreate");
  } else if (s.streams == 1 && st2) {
    cuda_ck(cudaStreamDestroy(st2), "cudaStreamDestroy");
    cuda_ck(cudaEventDestroy(fork_ev), "cudaEventDestroy");
    cuda_ck(cudaEventDestroy(join_ev), "cudaEventDestroy");
    st2 = nullptr;
    fork_ev = join_ev = nullptr;
  }
  slab = s.slab;
  rowL = s.row_lines;
  for (int a = 1; a < d.dim; ++a) col_tl[a] = std::min(col_tl_max[a], s.col_lines);
  const int ns[3] = {d.nx, d.ny, d.nz};
  for (int a = 0; a < d.dim; ++a)
    if (!ct_supported(ns[a]) && !make_fft_plan(ns[a], &plan[a], s.radix))
      throw KwError(KW_ERR_INTERNAL, "no radix plan of this order for " + std::to_string(ns[a]));
  sched_ = s;
}

// Grid, step class (absorption, nonlinearity, axisymmetry, full-grid
// sensors) and device (compute capability, SM count).
std::string Session::schedule_key() const {
  int dev = 0, major = 0, minor = 0, sms = 0;
  cuda_ck(cudaGetDevice(&dev), "cudaGetDevice");
  cuda_ck(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev), "device attribute");
  cuda_ck(cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev), "device attribute");
  cuda_ck(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "device attribute");
  char b[192];
  std::snprintf(b, sizeof(b), "%dx%dx%d/eos%d/nl%d/as%d/dense%d/sm%d%d.%d", d.nx, d.ny, d.nz, eos, nonlinear ? 1 : 0,
                axisym ? 1 : 0, dense_sensor ? 1 : 0, major, minor, sms);
  return b;
}

// Phase 0: slab splits and streams (3D grids of 16 planes or more), the
// current schedule first.  Phase 1: halved runtime-engine tiles.  Phase 2:
// the runtime engine's other radix orders, where they give other plans.
std::vector<Schedule> Session::schedule_candidates(int phase) const {
  std::vector<Schedule> c{sched_};
  auto add = [&](Schedule s) {
    s = normalise(s, d, row_lines_max(d));
    if (std::find(c.begin(), c.end(), s) == c.end()) c.push_back(s);
  };
  if (phase == 0) {
    if (d.dim == 3 && d.nz >= 16) {
      const int split[5][2] = {{1, 1}, {2, 2}, {3, 2}, {4, 2}, {2, 1}};
      for (auto& sp : split) {
        Schedule s = sched_;
        s.slab = (d.nz + sp[0] - 1) / sp[0];
        s.streams = sp[1];
        add(s);
      }
    }
  } else if (phase == 1) {
    if (runtime_rows() && sched_.row_lines > 1) {
      Schedule s = sched_;
      s.row_lines = sched_.row_lines / 2;
      add(s);
    }
    if (runtime_cols()) {
      int cmax = 1;
      for (int a = 1; a < d.dim; ++a)
        if (!ct_supported(a == 1 ? d.ny : d.nz)) cmax = std::max(cmax, col_tl[a]);
      if (cmax > 1) {
        Schedule s = sched_;
        s.col_lines = cmax / 2;
        add(s);
      }
    }
  } else if (phase == 2) {
    const int ns[3] = {d.nx, d.ny, d.nz};
    for (int v = 0; v <= 2; ++v) {
      if (v == sched_.radix) continue;
      bool differs = false;
      for (int a = 0; a < d.dim; ++a) {
        if (ct_supported(ns[a])) continue;
        FFTPlan p0{}, p1{};
        if (!make_fft_plan(ns[a], &p0, sched_.radix) || !make_fft_plan(ns[a], &p1, v)) continue;
        differs = differs || p0.nst != p1.nst || !std::equal(p0.rad, p0.rad + p0.nst, p1.rad);
      }
      if (differs) {
        Schedule s = sched_;
        s.radix = v;
        add(s);
      }
    }
  }
  return c;
}

TuneOutcome tune_schedule(const kw_input* in, const kw_options* opt) {
  if (!in || !opt) throw KwError(KW_ERR_INVALID_ARGUMENT, "input and options must not be NULL");
  constexpr int kTimed = 6, kWarm = 2, kRounds = 2, kMaxCand = 12;
  kw_input in2 = *in;
  kw_options o2 = *opt;
  // recorded series are left out (their memory grows with Nt); reductions stay
  o2.p_raw = o2.u_raw = o2.u_non_staggered_raw = 0;
  o2.verbose = 0;
  const uint64_t need = 4 + (uint64_t)kRounds * kMaxCand * (kWarm + kTimed) + 2;
  in2.Nt = std::max<uint64_t>(in->Nt, need);
  TuneOutcome r;
  struct Guard {
    Guard() { g_tuning = true; }
    ~Guard() { g_tuning = false; }
  } guard;
  Session tmp;
  tmp.setup(&in2, &o2);
  r.key = tmp.schedule_key();
  const Schedule def = tmp.default_schedule();
  tmp.set_schedule(def);
  r.chosen = def;
  tmp.advance(4);  // the first steps (initial pressure, graph capture), clocks up
  tmp.sync();
  auto time_set = [&](const std::vector<Schedule>& cands) {
    std::vector<float> best(cands.size(), 1e30f);
    for (int round = 0; round < kRounds; ++round)
      for (size_t i = 0; i < cands.size(); ++i) {
        tmp.set_schedule(cands[i]);
        tmp.advance(kWarm);
        tmp.advance(kTimed);
        best[i] = std::min(best[i], tmp.elapsed_ms() / kTimed);
      }
    tmp.sync();
    return best;
  };
  for (int phase = 0; phase < 3; ++phase) {
    tmp.set_schedule(r.chosen);
    const std::vector<Schedule> cands = tmp.schedule_candidates(phase);
    if (cands.size() < 2) continue;
    const std::vector<float> ms = time_set(cands);
    r.candidates += (int)cands.size();
    if (phase == 0 || r.ms_default == 0.f) r.ms_default = ms[0];  // cands[0] is the current choice
    size_t b = 0;
    for (size_t i = 1; i < ms.size(); ++i)
      if (ms[i] < ms[b]) b = i;
    // a challenger must win by more than 1 %, so timing noise does not flip
    // the choice from one run to the next
    if (b != 0 && ms[b] > 0.99f * ms[0]) b = 0;
    r.chosen = cands[b];
    r.ms_chosen = ms[b];
  }
  if (r.candidates > 0) remember(r.key, r.chosen, r.ms_chosen);
  return r;
}

void Session::select_schedule() {
  Schedule s = default_schedule();
  const int env_slab = env_int("KWAVE_B200_SLAB"), env_streams = env_int("KWAVE_B200_SLAB_STREAMS");
  if (env_slab > 0 || env_streams > 0) {  // a fixed schedule asked for by hand
    if (env_slab > 0) s.slab = env_slab;
    if (env_streams > 0) s.streams = env_streams;
  } else if (!g_tuning) {
    Schedule w;
    if (lookup(schedule_key(), &w)) {
      s = w;
    } else if (env_int("KWAVE_B200_TUNE") == 1 && in_user) {
      // tune now if a scratch copy fits next to this session
      size_t free_b = 0, total_b = 0;
      cuda_ck(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
      const size_t need = device_bytes_estimate(in_user, &opt) * 5 / 4 + (256u << 20);
      if (free_b > need) {
        try {
          s = tune_schedule(in_user, &opt).chosen;
        } catch (const KwError& e) {
          if (e.code != KW_ERR_OUT_OF_MEMORY) throw;  // no room after all: the built-in schedule
        }
      }
    }
  }
  set_schedule(s);
}

}  // namespace kwb

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
namespace {

int status_of(kw_status* st, int code, const char* msg) {
  if (st) {
    st->code = code;
    std::snprintf(st->message, sizeof(st->message), "%s", msg);
  }
  return code;
}

template <class F>
int guarded_call(kw_status* st, F&& f) {
  try {
    f();
    return status_of(st, KW_OK, "");
  } catch (const kwb::KwError& e) {
    return status_of(st, e.code, e.what());
  } catch (const std::bad_alloc&) {
    return status_of(st, KW_ERR_OUT_OF_MEMORY, "host allocation failed");
  } catch (const std::exception& e) {
    return status_of(st, KW_ERR_INTERNAL, e.what());
  }
}

void fill(kw_schedule* out, const kwb::Schedule& s) {
  out->slab_planes = s.slab;
  out->streams = s.streams;
  out->row_lines = s.row_lines;
  out->col_lines = s.col_lines;
  out->radix_plan = s.radix;
}

}  // namespace

extern "C" {

int kw_tune(const kw_input* in, const kw_options* opt, kw_schedule* chosen, kw_status* status) {
  return guarded_call(status, [&] {
    if (!in || !opt || !chosen) throw kwb::KwError(KW_ERR_INVALID_ARGUMENT, "NULL argument");
    if (opt->device >= 0) {
      const cudaError_t e = cudaSetDevice(opt->device);
      if (e != cudaSuccess) throw kwb::KwError(KW_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    }
    const kwb::TuneOutcome r = kwb::tune_schedule(in, opt);
    std::memset(chosen, 0, sizeof(*chosen));
    fill(chosen, r.chosen);
    chosen->candidates = r.candidates;
    chosen->ms_per_step = r.ms_chosen;
    chosen->ms_default = r.ms_default;
  });
}

int kw_wisdom_import(const char* path, kw_status* status) {
  return guarded_call(status, [&] {
    if (!path) throw kwb::KwError(KW_ERR_INVALID_ARGUMENT, "NULL path");
    std::lock_guard<std::mutex> lk(kwb::g_mu);
    kwb::import_file(path, /*missing_ok=*/false);
  });
}

int kw_wisdom_export(const char* path, kw_status* status) {
  return guarded_call(status, [&] {
    if (!path) throw kwb::KwError(KW_ERR_INVALID_ARGUMENT, "NULL path");
    std::lock_guard<std::mutex> lk(kwb::g_mu);
    kwb::export_file(path);
  });
}

void kw_wisdom_forget(void) {
  std::lock_guard<std::mutex> lk(kwb::g_mu);
  kwb::g_wisdom.clear();
  kwb::g_env_loaded = true;  // and do not read KWAVE_B200_WISDOM again
}

}  // extern "C"
