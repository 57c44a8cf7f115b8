// Internal host-side types of the solver (not part of the C ABI).
#pragma once
#include <cuda_runtime.h>

#include <deque>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "kernels.cuh"
#include "kernels_tma.cuh"
#include "kwave_b200.h"

namespace kwb {

struct KwError : std::runtime_error {
  int code;
  KwError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

// Launch shape of the time step: the z slabs that the y-inverse / row
// kernel / y-forward chains are split into and the streams the slabs
// alternate on, and the lines per block of the runtime-plan engine's row and
// column kernels (compile-time lengths have fixed tiles) -- choices that give
// bit-identical results -- and the radix order of the runtime-plan engine
// (make_fft_plan variant), which rounds differently.
struct Schedule {
  int slab = 1;       // z planes per chain slab
  int streams = 1;    // 1, or 2: slabs alternate between two streams
  int row_lines = 8;  // runtime-engine row tiles (x)
  int col_lines = 16; // runtime-engine column tiles (y and z)
  int radix = 0;      // runtime-engine radix order
  bool operator==(const Schedule& o) const {
    return slab == o.slab && streams == o.streams && row_lines == o.row_lines && col_lines == o.col_lines &&
           radix == o.radix;
  }
};

// Owning device allocation.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf();
  void alloc(size_t nbytes, cudaStream_t st);
};

class Batch;

class Session {
  friend class Batch;  // advances member sessions' captured steps as one graph

 public:
  ~Session();
  // allow_ring: the caller drains raw series in blocks (drain_raw), so they
  // may be held on the device as a ring of steps when the full series would
  // not fit the recording budget
  void setup(const kw_input* in, const kw_options* opt, bool allow_ring = false);
  void drain_raw(kw_output* out);  // copy raw rows recorded since the last drain
  long long ring_rows = 0, drained = 0;
  bool allow_ring_ = false;
  void advance(uint64_t n);
  float elapsed_ms();
  void sync();
  uint64_t in_flight();  // advance() calls whose steps have not finished on the device
  // checkpoints: the state between two steps, written to / read from an HDF5 file
  void save_checkpoint(const std::string& path);
  void restore_checkpoint(const std::string& path);
  std::vector<std::pair<std::string, DevBuf*>> state_buffers();
  void set_priority(int priority);  // waits for queued work, then re-creates the stream
  void read(kw_output* out);
  uint64_t last_launches_per_step() const { return last_steps ? last_launches / last_steps : 0; }
  static size_t device_bytes_estimate(const kw_input* in, const kw_options* opt);
  // launch schedule: the built-in choice for this grid, the one in use,
  // the key it is tuned and cached under, and the candidates a tuner times
  Schedule default_schedule() const;
  Schedule schedule() const { return sched_; }
  void set_schedule(const Schedule& s);  // waits for queued work; the step graph is captured again
  std::string schedule_key() const;
  std::vector<Schedule> schedule_candidates(int phase) const;
  bool runtime_rows() const;
  bool runtime_cols() const;
  void select_schedule();  // end of setup(): wisdom, else tuning when enabled, else default_schedule()

  cudaStream_t st = nullptr;
  uint64_t Nt = 0;
  uint64_t t_done = 0;

 private:
  void check_field(const kw_field& f, const char* name, bool required);
  Map map_of(const kw_field& f, DevBuf& buf, float scalar_default);
  void setup_sources(const kw_input* in);
  void setup_sensors(const kw_input* in);
  void build_sensor_lists(const uint64_t* lin, size_t n, std::vector<int>& si, std::vector<int>& sl);
  void corrected_source(float* out, const int* idx, const int* slot, int n, const float* sig, int nrows_sig,
                        int t, const float* weight = nullptr);
  void corrected_source_into(float* out, const int* idx, const int* slot, int n, const float* sig,
                             int nrows_sig, int t, int work_i, const float* weight = nullptr);
  // axisymmetric inputs (Nx x Ny, y radial from the axis) become an ordinary
  // 2D problem on Nx x 4Ny: the fields mirrored even about the axis and odd
  // about the outer radius, as the reference's 'WSWA-FFT' symmetry mirrors
  // them each step (kspaceFirstOrderAS.m:488-519, 709-722, 911-931)
  const kw_input* expand_axisymmetric(const kw_input* in);
  void run_spectral(std::vector<int> ins, std::vector<int> outs, std::vector<SpecOp> ops, int fanout);
  void col_pass(bool inv, const std::vector<int>& bufs, int z0, int nzs, int dual_field = -1, int dual_src = -1,
                const float2* dual_tab = nullptr);
  void fused_pass(const std::vector<int>& ins, const std::vector<int>& outs, const std::vector<SpecOp>& ops,
                  int fanout, const std::vector<int>& dual = {}, const float2* dual_tab = nullptr);
  void grad_pass();
  bool grad_dual_in_y() const;
  void grad_col_inverse(int z0, int nzs);
  Dims slab_dims(int z0, int nzs) const;
  void enqueue_init();
  void enqueue_step();
  void enqueue_step_body(uint64_t t);
  bool graphable(uint64_t t) const;
  UArgs u_args(float2* const* S);

  kw_options opt{};
  Dims d{};
  FFTPlan plan[3]{};
  const float2* twd[3]{};
  int col_tl[3]{16, 16, 16};
  int col_tl_max[3]{16, 16, 16};
  int rowL = 8;
  int slab = 1;  // z planes per chain slab
  Schedule sched_{};
  const kw_input* in_user = nullptr;  // the caller's input (before any axisymmetric expansion)
  uint64_t input_fp = 0;              // fingerprint of that input, kept with checkpoints
  // slabs of a chain alternate between st and st2, forked and joined by
  // events, so one slab's row kernel can run beside another's y passes
  cudaStream_t st2 = nullptr;
  cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
  template <class F>
  void for_slabs(F&& body);
  // captured steady-state step
  bool use_graph = true;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  uint64_t graph_launches = 0;
  uint64_t graph_gen = 0;  // captures so far (a batch rebuilds its parent graph when this changes)
  SpecTables T{};
  float dtf = 0.f;
  bool nonlinear = false;
  int eos = 0;
  bool p0 = false;

  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::deque<cudaEvent_t> pending_ev;  // one per advance() still running, oldest first
  std::vector<cudaEvent_t> spare_ev;
  uint64_t launches_ = 0, last_launches = 0, last_steps = 0;

  // operator tables
  DevBuf tw_buf[3], k2_buf[3], pos_buf[3], neg_buf[3], sh_buf[3], pml_buf[3], pmls_buf[3];
  const float* pml_d[3]{};
  RhoBox rho_box{};  // merged-density points (RhoBox)
  const float* pml_sg_d[3]{};
  // medium
  DevBuf c0sq_buf, rho0_buf, rinv_buf[3], bona_buf, c2tau_buf, c2eta_buf;
  Map c0sq_m{}, rho0_m{}, rinv_m[3]{}, bona_m{}, c2tau_m{}, c2eta_m{}, tau_m{};
  // fields
  DevBuf u_buf[3], rho_buf[3], S_buf[5], ploc_buf, p_buf, p0_buf, clock_buf, err_buf;
  // axisymmetric state: the original radial size, the expanded inputs, the
  // mirrored pressure-source entries (original entry, sign) and 1 / r
  bool axisym = false;
  int ny0 = 0;
  struct AxisymmetricInput {
    kw_input in;
    std::vector<float> c0, rho0, sgx, sgy, bona, alpha, p0;
    std::vector<uint64_t> p_idx, u_idx;
    std::vector<int> p_orig, u_orig;
    std::vector<float> p_w, u_w;
  } asx;
  uint64_t p_rows0 = 0, u_rows0 = 0;  // source points before mirroring
  DevBuf psrc_w, usrc_w, inv_r_buf, ur_buf;
  // TMA tensor maps over the half-spectrum buffers (y pass / z pass)
  bool use_tma[3]{false, false, false};
  CUtensorMap map_y[5], map_z[5];  // [4]: the axisymmetric u_r / r spectrum
  CUtensorMap map_zr[5];           // last-axis remainder tiles (box {2, rem_y, nz})
  bool use_rem = false;
  int rem_y = 0;
  TmaWaitArgs tma_wait{2000000000ull, -1};  // wait limit (2 s) and the test hook of the TMA kernels
  WaitCtl row_wait() const { return WaitCtl{(int*)err_buf.p, tma_wait.limit_ns}; }  // the row kernels' waits
  Clock clk{};
  // sources
  SparseSource psrc{}, usrc{};
  DenseSource pdense{}, udense[3]{};
  DevBuf psrc_idx, psrc_slot, psrc_sig, psrc_field;
  DevBuf usrc_idx, usrc_slot, usig_buf[3], ufield_buf[3], ones_buf;
  DevBuf tsrc_delay, tsrc_apod;
  const float* usig_d[3]{};
  int u_len[3]{};
  int p_mode = 0, p_len = 0, p_nsrc = 0, p_nsig = 1;
  int u_mode = 0, u_nsrc = 0, u_nsig = 1;
  bool p_many_additive = false, u_many_additive = false, ones_ready = false;
  int ones_field = 0;
  // sensors
  long long ns = 0, nrec = 0;
  bool dense_sensor = false;
  DevBuf sidx_buf, sslot_buf;
  const int* sidx_d = nullptr;
  const int* sslot_d = nullptr;
  Sensor sens_p{}, sens_u[3]{};
  Sensor sens_uns[3]{};                 // u on the regular grid (u_non_staggered_raw)
  // Cartesian points by linear interpolation: the step kernels record the
  // simplex vertices (vsens_*, this step only), k_interp_sensor forms the
  // points (sens_*, mode 3) from them
  bool interp = false;
  int interp_k = 0;
  long long nvert = 0;
  Sensor vsens_p{}, vsens_u[3]{}, vsens_uns[3]{};
  DevBuf vslot_buf, vweight_buf, vval_p_buf, vval_u_buf[3], vval_uns_buf[3];
  const Sensor& row_sens_p() const { return interp ? vsens_p : sens_p; }
  const Sensor& row_sens_u(int a) const { return interp ? vsens_u[a] : sens_u[a]; }
  const Sensor& row_sens_uns(int a) const { return interp ? vsens_uns[a] : sens_uns[a]; }
  void interp_points(int which);  // 0: p, 1: u, 2: u on the regular grid
  DevBuf uns_raw_buf[3], uns_field_buf;  // its series; the shifted field of one component
  void record_non_staggered();
  DevBuf p_raw_buf, p_max_buf, p_min_buf, p_rms_buf, p_rmsb_buf, p_rmsf_buf, p_maxall_buf, p_minall_buf;
  DevBuf u_raw_buf[3], u_max_buf[3], u_min_buf[3], u_rms_buf[3], u_rmsb_buf[3], u_rmsf_buf[3], u_maxall_buf[3],
      u_minall_buf[3];
};

// What tune_schedule() measured: the schedule chosen for the key, its device
// time per step and the built-in default's, and how many schedules it timed
// (0: the grid offers no choice).  The choice is remembered for the key.
struct TuneOutcome {
  std::string key;
  Schedule chosen{};
  float ms_chosen = 0.f, ms_default = 0.f;
  int candidates = 0;
};
TuneOutcome tune_schedule(const kw_input* in, const kw_options* opt);

}  // namespace kwb

// The C ABI's session handle.
struct kw_session {
  std::unique_ptr<kwb::Session> s;
};
