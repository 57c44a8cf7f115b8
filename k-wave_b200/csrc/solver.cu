// Host orchestrator and C ABI of the B200 k-space solver.
//
// A session owns one simulation resident in HBM: medium maps, the split
// density and velocity fields, four half-spectrum work buffers, operator
// tables and sensor accumulators.  kw_session_advance() enqueues time steps
// on the session's stream; kw_solve() is create + advance(Nt) + read.
//
// The operators that the v1.2 input file omits are rebuilt here from the
// scalars it carries (dx, dt, c_ref, pml_*), in FP64, then stored as FP32
// 1D tables (k-Wave/kspaceFirstOrder3D.m:617-659, private/getPML.m:49-85,
// kWaveGrid.m:779-797, kspaceFirstOrder_createAbsorptionVariables.m:27-99).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "kernels.cuh"
#include "kwave_b200.h"
#include "hdf5_lite.h"
#include "solver_internal.h"

namespace kwb {

// launch helpers (kernels.cu)
cudaError_t launch_col_fft(bool inv, const ColArgs& a, int nfields, long long nouter, const FFTPlan& plan,
                           const float2* tw, cudaStream_t st);
cudaError_t launch_fused_last(const FusedArgs& a, int ninputs, long long nouter, const FFTPlan& plan,
                              const float2* tw, const SpecTables& T, int dim, cudaStream_t st);
cudaError_t launch_x_u(const UArgs& a, const Dims& d, const FFTPlan& plan, const float2* tw, int L,
                       cudaStream_t st);
cudaError_t launch_x_rho(const RhoArgs& a, const Dims& d, const FFTPlan& plan, const float2* tw, int L,
                         cudaStream_t st);
cudaError_t launch_x_eos(const EosArgs& a, const Dims& d, const FFTPlan& plan, const float2* tw, int L,
                         cudaStream_t st);
cudaError_t launch_x_r2c(const float* f, float2* S, const Dims& d, const FFTPlan& plan, const float2* tw,
                         int L, cudaStream_t st);
cudaError_t launch_x_c2r(const float2* S, float* out, int accumulate, const Dims& d, const FFTPlan& plan,
                         const float2* tw, int L, cudaStream_t st);
cudaError_t launch_scatter(float* f, const int* idx, const int* slot, int n, const float* sig,
                           int nrows_sig, int t, const float* weight, cudaStream_t st);
cudaError_t launch_rho_init(float* r0, float* r1, float* r2, const float* p0, Map c0sq, int dim, const RhoBox& box,
                            int nx, int ny, long long n, cudaStream_t st);
cudaError_t launch_scale_rows(float* out, const float* in, const float* r, int nx, int ny, long long n,
                              cudaStream_t st);
cudaError_t launch_interp_sensor(const Sensor& s, const float* vals, const int* vslot, const float* w, int K,
                                 const Clock& clk, cudaStream_t st);
cudaError_t launch_record_field(const float* f, const Sensor& s, const Clock& clk, long long n,
                                cudaStream_t st);
cudaError_t launch_advance(int* t, cudaStream_t st);
cudaError_t launch_rms_final(const float2* acc, const float* blk, int partial, float* out, long long n, float inv_n,
                             cudaStream_t st);
cudaError_t launch_medium_maps(float* c0_to_c0sq, float c0_scalar, float* ctau, float* ceta, const float* alpha,
                               float alpha_scalar, double np_per_db, double y, double tan_py, int eos, long long n,
                               cudaStream_t st);
cudaError_t launch_reciprocal(float* v, long long n, cudaStream_t st);
bool tma_col_supported(int n);    // TMA-fed y pass
bool tma_fused_supported(int n);  // TMA-fed fused last-axis operator
int tma_lines(int n);
bool make_spec_map(CUtensorMap* m, void* base, const Dims& d, int yaxis, int n);
bool make_spec_map_rem(CUtensorMap* m, void* base, const Dims& d, int n, int rows);
cudaError_t launch_col_tma(bool inv, int n, const ColTmaArgs& a, const float2* tw, cudaStream_t st);
cudaError_t launch_fused_tma(int n, const FusedTmaArgs& a, const float2* tw, const SpecTables& T, cudaStream_t st);

static void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    if (e == cudaErrorMemoryAllocation) throw KwError(KW_ERR_OUT_OF_MEMORY, std::string(what) + ": " + cudaGetErrorString(e));
    throw KwError(KW_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  }
}

// ---------------------------------------------------------------------------
// device buffer
// ---------------------------------------------------------------------------
// Stream-ordered allocations from the device's default memory pool, which
// keeps freed memory for the next session (set up once per device), so
// creating and destroying sessions neither synchronises the device nor goes
// back to the driver.  Buffers are freed on the legacy stream after the
// session's own stream has been synchronised.
static void retain_pool_memory() {
  static std::once_flag once[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return;
  std::call_once(once[dev], [dev] {
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) != cudaSuccess) return;
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  });
}

DevBuf::~DevBuf() {
  if (p) cudaFreeAsync(p, nullptr);
}
void DevBuf::alloc(size_t nbytes, cudaStream_t st) {
  if (p) cudaFreeAsync(p, st);
  p = nullptr;
  bytes = nbytes;
  if (nbytes == 0) return;
  ck(cudaMallocAsync(&p, nbytes, st), "cudaMallocAsync");
}

// ---------------------------------------------------------------------------
// FP64 operator construction
// ---------------------------------------------------------------------------
// centred wavenumbers (kWaveGrid.m:779-797) reordered with ifftshift
static std::vector<double> kvec_fft_order(int n, double d) {
  std::vector<double> c(n);
  const int h = n / 2;
  for (int j = 0; j < n; ++j) {
    double nx = (n % 2 == 0) ? (double)(j - h) / n : (double)(j - (n - 1) / 2) / n;
    c[j] = nx;
  }
  c[h] = 0.0;
  std::vector<double> k(n);
  for (int b = 0; b < n; ++b) k[b] = (2.0 * M_PI / d) * c[(b + h) % n];
  return k;
}

// getPML.m:49-85 (non-axisymmetric)
static std::vector<double> pml_profile(int n, double d, double dt, double c, int size, double alpha, bool stag) {
  std::vector<double> pml(n, 1.0);
  for (int i = 1; i <= size && size > 0; ++i) {
    double x = i;
    double left, right;
    if (stag) {
      left = alpha * (c / d) * std::pow(((x + 0.5) - size - 1) / (0.0 - size), 4);
      right = alpha * (c / d) * std::pow((x + 0.5) / size, 4);
    } else {
      left = alpha * (c / d) * std::pow((x - size - 1) / (0.0 - size), 4);
      right = alpha * (c / d) * std::pow(x / size, 4);
    }
    pml[i - 1] = std::exp(-left * dt / 2);
    pml[n - size + i - 1] = std::exp(-right * dt / 2);
  }
  return pml;
}

// db2neper.m:50
static double db2neper(double a, double y) {
  return 100.0 * a * std::pow(1e-6 / (2 * M_PI), y) / (20.0 * std::log10(std::exp(1.0)));
}

static bool factors_2357(uint64_t n) {
  if (n == 0) return false;
  for (uint64_t p : {2ull, 3ull, 5ull, 7ull})
    while (n % p == 0) n /= p;
  return n == 1;
}

// ---------------------------------------------------------------------------
// Session
// ---------------------------------------------------------------------------
template <class T>
static T* up(DevBuf& b, const T* h, size_t n, cudaStream_t st) {
  b.alloc(n * sizeof(T), st);
  if (n) ck(cudaMemcpyAsync(b.p, h, n * sizeof(T), cudaMemcpyHostToDevice, st), "upload");
  return (T*)b.p;
}

void Session::check_field(const kw_field& f, const char* name, bool required) {
  if (!f.data || f.numel == 0) {
    if (required) throw KwError(KW_ERR_INVALID_ARGUMENT, std::string(name) + " is missing");
    return;
  }
  if (f.numel != 1 && f.numel != (uint64_t)d.npts)
    throw KwError(KW_ERR_INVALID_ARGUMENT, std::string(name) + " must be a scalar or hold Nx*Ny*Nz values");
}

Map Session::map_of(const kw_field& f, DevBuf& buf, float scalar_default) {
  Map m{nullptr, scalar_default};
  if (!f.data || f.numel == 0) return m;
  if (f.numel == 1) {
    m.s = f.data[0];
    return m;
  }
  m.p = up(buf, f.data, f.numel, st);
  return m;
}

// Sort 1-based indices, keep the last duplicate (MATLAB assignment order),
// and return (sorted 0-based index, original position).
static void sort_indices(const uint64_t* idx1, uint64_t n, uint64_t npts, std::vector<int>& sidx,
                         std::vector<int>& slot, const char* name) {
  std::vector<std::pair<long long, int>> v(n);
  for (uint64_t j = 0; j < n; ++j) {
    if (idx1[j] < 1 || idx1[j] > npts)
      throw KwError(KW_ERR_INVALID_ARGUMENT, std::string(name) + " holds an index outside the grid");
    v[j] = {(long long)idx1[j] - 1, (int)j};
  }
  std::stable_sort(v.begin(), v.end(), [](auto& a, auto& b) { return a.first < b.first; });
  sidx.clear();
  slot.clear();
  for (size_t j = 0; j < v.size(); ++j) {
    if (j + 1 < v.size() && v[j + 1].first == v[j].first) continue;  // a later entry wins
    sidx.push_back((int)v[j].first);
    slot.push_back(v[j].second);
  }
}

// Set-up phase timings on stderr at --verbose 2 (host wall time, the
// device work of each phase included).
struct PhaseTimer {
  bool on;
  cudaStream_t st = nullptr;
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  void mark(const char* what) {
    if (!on) return;
    if (st) cudaStreamSynchronize(st);
    const auto t = std::chrono::steady_clock::now();
    std::fprintf(stderr, "kwave_b200 set-up: %-28s %8.1f ms\n", what,
                 std::chrono::duration<double, std::milli>(t - t0).count());
    t0 = t;
  }
};

const kw_input* Session::expand_axisymmetric(const kw_input* in) {
  if (in->Nz != 1) throw KwError(KW_ERR_INVALID_ARGUMENT, "axisymmetric grids are 2D (Nz must be 1)");
  if (in->absorbing_flag == 1)
    throw KwError(KW_ERR_UNSUPPORTED, "axisymmetric simulations take Stokes absorption only (absorbing_flag 2)");
  if (in->uy_source_flag || in->uz_source_flag || in->transducer_source_flag)
    throw KwError(KW_ERR_UNSUPPORTED, "radial velocity and transducer sources are not supported on axisymmetric grids");
  if (opt.u_non_staggered_raw)
    throw KwError(KW_ERR_UNSUPPORTED, "u_non_staggered_raw is not supported on axisymmetric grids");
  if (in->Ny < 2 || in->Nx < 1) throw KwError(KW_ERR_INVALID_ARGUMENT, "Nx and Ny must be positive");
  const uint64_t nx = in->Nx, ny = in->Ny, ny4 = 4 * ny;
  // column maps: expanded radial index j -> original column and sign, for the
  // pressure points (even about the axis, odd about the outer radius, zero on
  // the outer-radius columns) and the radially staggered points
  std::vector<uint64_t> pc(ny4), sc(ny4);
  std::vector<float> ps(ny4), ss(ny4);
  for (uint64_t j = 0; j < ny4; ++j) {
    const uint64_t q = j / ny, m = j % ny;
    if (q == 0 || q == 2) {
      pc[j] = m;
      ps[j] = (q == 0) ? 1.f : -1.f;
    } else {
      pc[j] = (m == 0) ? ny - 1 : ny - m;  // m == 0: the odd point, zero field; medium from the edge
      ps[j] = (m == 0) ? 0.f : (q == 1 ? -1.f : 1.f);
    }
    sc[j] = (q == 0 || q == 2) ? m : ny - 1 - m;
    ss[j] = (q < 2) ? 1.f : -1.f;
  }
  auto expand = [&](const kw_field& f, bool staggered, std::vector<float>& store) {
    kw_field o = f;
    if (f.numel <= 1) return o;
    if (f.numel != nx * ny) throw KwError(KW_ERR_INVALID_ARGUMENT, "axisymmetric medium arrays must be Nx x Ny");
    store.resize(nx * ny4);
    const std::vector<uint64_t>& col = staggered ? sc : pc;
    for (uint64_t j = 0; j < ny4; ++j)
      for (uint64_t x = 0; x < nx; ++x) store[x + nx * j] = f.data[x + nx * col[j]];
    o.data = store.data();
    o.numel = store.size();
    return o;
  };
  asx.in = *in;
  asx.in.Ny = ny4;
  asx.in.c0 = expand(in->c0, false, asx.c0);
  asx.in.rho0 = expand(in->rho0, false, asx.rho0);
  asx.in.rho0_sgx = expand(in->rho0_sgx, false, asx.sgx);
  asx.in.rho0_sgy = expand(in->rho0_sgy, true, asx.sgy);
  if (in->nonlinear_flag) asx.in.BonA = expand(in->BonA, false, asx.bona);
  if (in->absorbing_flag) asx.in.alpha_coeff = expand(in->alpha_coeff, false, asx.alpha);
  if (in->p0_source_flag && in->p0_source_input) {
    asx.p0.resize(nx * ny4);
    for (uint64_t j = 0; j < ny4; ++j)
      for (uint64_t x = 0; x < nx; ++x) asx.p0[x + nx * j] = ps[j] * in->p0_source_input[x + nx * pc[j]];
    asx.in.p0_source_input = asx.p0.data();
  }
  // source points and their mirror images, with the sign of the field there:
  // pressure and the axial velocity follow the pressure-point pattern
  // (kspaceFirstOrderAS.m:795-798, 1041-1044)
  auto mirror_points = [&](const uint64_t* idx, uint64_t n, std::vector<uint64_t>& out, std::vector<int>& orig,
                           std::vector<float>& w, const char* name) {
    for (uint64_t e = 0; e < n; ++e) {
      const uint64_t lin = idx[e];
      if (lin < 1 || lin > nx * ny) throw KwError(KW_ERR_INVALID_ARGUMENT, std::string(name) + " holds an index outside the grid");
      const uint64_t x = (lin - 1) % nx, y = (lin - 1) / nx;
      const uint64_t cols[4] = {y, 2 * ny - y, 2 * ny + y, 4 * ny - y};
      const float sg[4] = {1.f, -1.f, -1.f, 1.f};
      for (int k = 0; k < 4; ++k) {
        if ((k == 1 || k == 3) && y == 0) continue;
        out.push_back(x + nx * cols[k] + 1);
        orig.push_back((int)e);
        w.push_back(sg[k]);
      }
    }
  };
  p_rows0 = in->p_source_index_numel;
  if (in->p_source_flag && in->p_source_index) {
    mirror_points(in->p_source_index, in->p_source_index_numel, asx.p_idx, asx.p_orig, asx.p_w, "p_source_index");
    asx.in.p_source_index = asx.p_idx.data();
    asx.in.p_source_index_numel = asx.p_idx.size();
  }
  u_rows0 = in->u_source_index_numel;
  if (in->ux_source_flag && in->u_source_index) {
    mirror_points(in->u_source_index, in->u_source_index_numel, asx.u_idx, asx.u_orig, asx.u_w, "u_source_index");
    asx.in.u_source_index = asx.u_idx.data();
    asx.in.u_source_index_numel = asx.u_idx.size();
  }
  if (in->sensor_mask_type == 0) {
    for (uint64_t j = 0; j < in->sensor_mask_index_numel; ++j)
      if (in->sensor_mask_index[j] < 1 || in->sensor_mask_index[j] > nx * ny)
        throw KwError(KW_ERR_INVALID_ARGUMENT, "sensor_mask_index holds an index outside the grid");
  } else if (in->sensor_mask_corners) {
    for (uint64_t k = 0; k + 5 < in->sensor_mask_corners_numel; k += 6)
      if (in->sensor_mask_corners[k + 4] > ny)
        throw KwError(KW_ERR_INVALID_ARGUMENT, "sensor_mask_corners reach past the grid");
  }
  axisym = true;
  ny0 = (int)ny;
  return &asx.in;
}

// A fingerprint of a simulation's input, stored with its checkpoints: every
// scalar and flag, the length of every array, and up to 65536 evenly spaced
// elements of each array (64-bit FNV-1a over their bytes).  It tells apart
// checkpoints of different media, sources, sensors, grids or time steps
// without reading whole arrays at session creation.
namespace {
struct Fnv {
  uint64_t h = 1469598103934665603ull;
  void bytes(const void* p, size_t n) {
    const unsigned char* b = static_cast<const unsigned char*>(p);
    for (size_t i = 0; i < n; ++i) h = (h ^ b[i]) * 1099511628211ull;
  }
  template <class T>
  void val(T v) { bytes(&v, sizeof(v)); }
  template <class T>
  void sampled(const T* a, uint64_t n) {
    val(n);
    if (!a || n == 0) {
      val<uint64_t>(0);
      return;
    }
    const uint64_t m = std::min<uint64_t>(n, 65536);
    for (uint64_t i = 0; i < m; ++i) val(a[m == 1 ? 0 : (i * (n - 1)) / (m - 1)]);
  }
};
}  // namespace

static uint64_t input_fingerprint(const kw_input* in) {
  Fnv f;
  for (uint64_t v : {in->Nx, in->Ny, in->Nz, in->Nt, in->pml_x_size, in->pml_y_size, in->pml_z_size,
                     in->nonlinear_flag, in->absorbing_flag, in->p0_source_flag, in->p_source_flag,
                     in->p_source_mode, in->p_source_many, in->ux_source_flag, in->uy_source_flag,
                     in->uz_source_flag, in->u_source_mode, in->u_source_many, in->sensor_mask_type,
                     in->transducer_source_flag, in->axisymmetric_flag})
    f.val(v);
  for (float v : {in->dx, in->dy, in->dz, in->dt, in->c_ref, in->pml_x_alpha, in->pml_y_alpha, in->pml_z_alpha,
                  in->alpha_power})
    f.val(v);
  for (const kw_field* k : {&in->c0, &in->rho0, &in->rho0_sgx, &in->rho0_sgy, &in->rho0_sgz, &in->BonA,
                            &in->alpha_coeff})
    f.sampled(k->data, k->data ? k->numel : 0);
  const uint64_t npts = in->Nx * in->Ny * in->Nz;
  f.sampled(in->p0_source_flag ? in->p0_source_input : nullptr, in->p0_source_flag ? npts : 0);
  f.sampled(in->p_source_index, in->p_source_index_numel);
  const uint64_t p_rows = in->p_source_many ? in->p_source_index_numel : 1;
  f.sampled(in->p_source_input, in->p_source_input ? in->p_source_flag * p_rows : 0);
  f.sampled(in->u_source_index, in->u_source_index_numel);
  const uint64_t u_rows = in->u_source_many ? in->u_source_index_numel : 1;
  f.sampled(in->ux_source_input, in->ux_source_input ? in->ux_source_flag * u_rows : 0);
  f.sampled(in->uy_source_input, in->uy_source_input ? in->uy_source_flag * u_rows : 0);
  f.sampled(in->uz_source_input, in->uz_source_input ? in->uz_source_flag * u_rows : 0);
  f.sampled(in->sensor_mask_index, in->sensor_mask_index_numel);
  f.sampled(in->sensor_mask_corners, in->sensor_mask_corners_numel);
  f.sampled(in->transducer_source_input, in->transducer_source_input_numel);
  f.sampled(in->delay_mask, in->delay_mask ? in->u_source_index_numel : 0);
  f.sampled(in->transducer_source_apodization,
            in->transducer_source_apodization ? in->u_source_index_numel : 0);
  f.sampled(in->sensor_interp_index, in->sensor_interp_numel);
  f.sampled(in->sensor_interp_weight, in->sensor_interp_numel);
  return f.h;
}

void Session::setup(const kw_input* in, const kw_options* o, bool allow_ring) {
  allow_ring_ = allow_ring;
  if (!in || !o) throw KwError(KW_ERR_INVALID_ARGUMENT, "input and options must not be NULL");
  opt = *o;
  PhaseTimer timer{opt.verbose >= 2};
  if (opt.start_index == 0) opt.start_index = 1;
  if (in->Nx < 1 || in->Ny < 1 || in->Nz < 1 || in->Nt < 1)
    throw KwError(KW_ERR_INVALID_ARGUMENT, "Nx, Ny, Nz and Nt must be positive");
  p_rows0 = in->p_source_index_numel;
  u_rows0 = in->u_source_index_numel;
  in_user = in;
  input_fp = input_fingerprint(in);
  if (in->axisymmetric_flag) in = expand_axisymmetric(in);
  if (in->Ny == 1) throw KwError(KW_ERR_UNSUPPORTED, "1D simulations are not supported (Ny must be > 1)");
  for (uint64_t n : {in->Nx, in->Ny, in->Nz}) {
    if (n > 1 && !factors_2357(n))
      throw KwError(KW_ERR_UNSUPPORTED, "grid sizes must factor into 2, 3, 5 and 7");
    if (n > 4096) throw KwError(KW_ERR_UNSUPPORTED, "grid sizes above 4096 are not supported");
  }
  if (in->Nx < 2) throw KwError(KW_ERR_UNSUPPORTED, "Nx must be at least 2");
  d.nx = (int)in->Nx;
  d.ny = (int)in->Ny;
  d.nz = (int)in->Nz;
  d.dim = (in->Nz == 1) ? 2 : 3;
  d.nxh = d.nx / 2 + 1;
  // row pitch in bins: even, so rows start on 16-byte boundaries (TMA strides,
  // paired-bin vector accesses); TMA column tiles that run past bin nxh - 1
  // are cut by the tensor maps' extent (zero fill on loads, clipped stores), so
  // no padding bin is read from or written to memory
  d.nxp = (d.nxh + 1) / 2 * 2;
  d.nrows = (long long)d.ny * d.nz;
  d.npts = (long long)d.nx * d.nrows;
  d.row0 = 0;
  d.row1 = d.nrows;
  if (d.npts >= (1LL << 31)) throw KwError(KW_ERR_UNSUPPORTED, "grids above 2^31 points are not supported");
  Nt = in->Nt;
  if (!(in->dx > 0) || !(in->dy > 0) || (d.dim == 3 && !(in->dz > 0)) || !(in->dt > 0))
    throw KwError(KW_ERR_INVALID_ARGUMENT, "dx, dy, (dz) and dt must be positive");
  if (!(in->c_ref > 0)) throw KwError(KW_ERR_INVALID_ARGUMENT, "c_ref must be positive");
  check_field(in->c0, "c0", true);
  check_field(in->rho0, "rho0", true);
  check_field(in->rho0_sgx, "rho0_sgx", true);
  check_field(in->rho0_sgy, "rho0_sgy", true);
  if (d.dim == 3) check_field(in->rho0_sgz, "rho0_sgz", true);
  nonlinear = in->nonlinear_flag != 0;
  if (nonlinear) check_field(in->BonA, "BonA", true);
  eos = (int)in->absorbing_flag;
  if (eos < 0 || eos > 2) throw KwError(KW_ERR_INVALID_ARGUMENT, "absorbing_flag must be 0, 1 or 2");
  if (eos) check_field(in->alpha_coeff, "alpha_coeff", true);
  if (in->p0_source_flag && !in->p0_source_input)
    throw KwError(KW_ERR_INVALID_ARGUMENT, "p0_source_input is missing");
  if (in->p0_source_flag && in->p_source_flag)
    throw KwError(KW_ERR_INVALID_ARGUMENT, "p0 and p sources cannot be used together");

  retain_pool_memory();
  ck(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "cudaStreamCreate");
  ck(cudaEventCreate(&ev0), "cudaEventCreate");
  ck(cudaEventCreate(&ev1), "cudaEventCreate");

  timer.st = st;
  timer.mark("validation, stream");
  // ----- FFT plans and twiddles (FP64 -> FP32) -----
  const int ns[3] = {d.nx, d.ny, d.nz};
  for (int a = 0; a < d.dim; ++a) {
    if (!make_fft_plan(ns[a], &plan[a])) throw KwError(KW_ERR_UNSUPPORTED, "unsupported FFT size");
    std::vector<float2> tw(ns[a]);
    for (int k = 0; k < ns[a]; ++k) {
      const double ang = -2.0 * M_PI * (double)k / ns[a];
      tw[k] = make_float2((float)std::cos(ang), (float)std::sin(ang));
    }
    twd[a] = up(tw_buf[a], tw.data(), tw.size(), st);
  }
  // runtime-engine tiles: the most lines (up to 16) whose shared-memory
  // buffers stay under 160 KB; the schedule may lower them
  col_tl[0] = 16;
  for (int a = 1; a < d.dim; ++a) {
    int tl = 16;
    while (tl > 1 && (size_t)tl * ns[a] * 3 * 8 + ns[a] * 8 > 160 * 1024) tl /= 2;
    col_tl[a] = col_tl_max[a] = tl;
  }
  rowL = std::max(1, std::min(8, 2048 / d.nx));

  // ----- operator tables -----
  const double dd[3] = {in->dx, in->dy, in->dz};
  const double dt = in->dt, c_ref = in->c_ref;
  for (int a = 0; a < d.dim; ++a) {
    std::vector<double> k = kvec_fft_order(ns[a], dd[a]);
    const int cnt = (a == 0) ? d.nxh : ns[a];
    std::vector<float> k2(cnt);
    std::vector<float2> pos(cnt), neg(cnt), sh(cnt);
    for (int b = 0; b < cnt; ++b) {
      k2[b] = (float)(k[b] * k[b]);
      std::complex<double> ik(0.0, k[b]);
      const std::complex<double> e = std::exp(std::complex<double>(0.0, -k[b] * dd[a] / 2));
      std::complex<double> p = ik * std::exp(std::complex<double>(0.0, k[b] * dd[a] / 2));
      std::complex<double> q = ik * e;
      pos[b] = make_float2((float)p.real(), (float)p.imag());
      neg[b] = make_float2((float)q.real(), (float)q.imag());
      // kspaceFirstOrder_createStorageVariables.m:91-97.  At the Nyquist bin of an
      // even axis the factor is i; real(ifft(.)) keeps only its Hermitian part,
      // the real part, which is what a half-spectrum pipeline must apply.
      const bool nyq = (ns[a] % 2 == 0) && (b == ns[a] / 2);
      sh[b] = make_float2((float)e.real(), nyq ? 0.f : (float)e.imag());
    }
    T.k2[a] = up(k2_buf[a], k2.data(), cnt, st);
    T.ddk_pos[a] = up(pos_buf[a], pos.data(), cnt, st);
    T.ddk_neg[a] = up(neg_buf[a], neg.data(), cnt, st);
    T.shift_neg[a] = up(sh_buf[a], sh.data(), cnt, st);
    const uint64_t psz[3] = {in->pml_x_size, in->pml_y_size, in->pml_z_size};
    const double pal[3] = {in->pml_x_alpha, in->pml_y_alpha, in->pml_z_alpha};
    std::vector<double> pm, pms;
    if (axisym && a == 1) {
      // getPML.m with `axisymmetric`: the profile at the outer radius only,
      // then mirrored like the fields it damps
      if (psz[a] > (uint64_t)ny0) throw KwError(KW_ERR_INVALID_ARGUMENT, "PML is larger than the grid");
      std::vector<double> p1 = pml_profile(ny0, dd[a], dt, c_ref, (int)psz[a], pal[a], false);
      std::vector<double> s1 = pml_profile(ny0, dd[a], dt, c_ref, (int)psz[a], pal[a], true);
      for (uint64_t j = 0; j < psz[a]; ++j) p1[j] = s1[j] = 1.0;
      pm.resize(ns[a]);
      pms.resize(ns[a]);
      for (int j = 0; j < ns[a]; ++j) {
        const int q = j / ny0, m = j % ny0;
        pm[j] = (q == 0 || q == 2) ? p1[m] : p1[m == 0 ? ny0 - 1 : ny0 - m];
        pms[j] = (q == 0 || q == 2) ? s1[m] : s1[ny0 - 1 - m];
      }
    } else {
      if (psz[a] * 2 > (uint64_t)ns[a]) throw KwError(KW_ERR_INVALID_ARGUMENT, "PML is larger than the grid");
      pm = pml_profile(ns[a], dd[a], dt, c_ref, (int)psz[a], pal[a], false);
      pms = pml_profile(ns[a], dd[a], dt, c_ref, (int)psz[a], pal[a], true);
    }
    std::vector<float> f1(pm.begin(), pm.end()), f2(pms.begin(), pms.end());
    {  // the merged-density box along this axis: the first run of PML factors equal to 1
      int lo = 0;
      while (lo < (int)f1.size() && f1[lo] != 1.f) ++lo;
      int hi = lo;
      while (hi < (int)f1.size() && f1[hi] == 1.f) ++hi;
      if (a == 0) {  // whole aligned groups of 4 x points
        lo = (lo + 3) & ~3;
        hi &= ~3;
      }
      rho_box.lo[a] = lo;
      rho_box.hi[a] = std::max(lo, hi);
    }
    pml_d[a] = up(pml_buf[a], f1.data(), f1.size(), st);
    pml_sg_d[a] = up(pmls_buf[a], f2.data(), f2.size(), st);
  }
  if (d.dim == 2) {
    T.k2[2] = T.k2[1];
    T.ddk_pos[2] = T.ddk_pos[1];
    T.ddk_neg[2] = T.ddk_neg[1];
    T.shift_neg[2] = T.shift_neg[1];
  }
  T.cdt2 = (float)(c_ref * dt / 2.0);
  T.scale = (float)(1.0 / (double)d.npts);
  T.ym2 = (float)(in->alpha_power - 2.0);
  T.ym1 = (float)(in->alpha_power - 1.0);
  dtf = in->dt;

  timer.mark("plans, operator tables");
  // ----- medium -----
  // Maps are uploaded as given and derived on the device (c0^2, 1/rho0_sg,
  // and the FP64 absorption maps), scalars stay scalars.
  {
    const bool c0_map = in->c0.numel > 1;
    if (c0_map) {
      c0sq_m.p = up(c0sq_buf, in->c0.data, (size_t)in->c0.numel, st);  // squared below
      c0sq_m.s = 0.f;
    } else {
      c0sq_m = Map{nullptr, in->c0.data[0] * in->c0.data[0]};
    }
    rho0_m = map_of(in->rho0, rho0_buf, 0.f);
    const kw_field* sg[3] = {&in->rho0_sgx, &in->rho0_sgy, &in->rho0_sgz};
    for (int a = 0; a < d.dim; ++a) {
      if (sg[a]->numel > 1) {
        float* v = up(rinv_buf[a], sg[a]->data, (size_t)sg[a]->numel, st);
        ck(launch_reciprocal(v, (long long)sg[a]->numel, st), "1/rho0_sg");
        rinv_m[a] = Map{v, 0.f};
      } else {
        rinv_m[a] = Map{nullptr, 1.0f / sg[a]->data[0]};
      }
    }
    if (nonlinear) bona_m = map_of(in->BonA, bona_buf, 0.f);
    float* ctau = nullptr;
    float* ceta = nullptr;
    const double y = in->alpha_power;
    const double np_per_db = db2neper(1.0, eos == 1 ? y : 2.0);  // linear in the coefficient
    const double tan_py = std::tan(M_PI * y / 2.0);
    const bool absorb = eos == 1 || eos == 2;
    const bool het = absorb && (c0_map || in->alpha_coeff.numel > 1);
    DevBuf alpha_tmp;
    const float* alpha_d = nullptr;
    if (het) {
      ctau = (float*)(c2tau_buf.alloc(sizeof(float) * d.npts, st), c2tau_buf.p);
      if (eos == 1) ceta = (float*)(c2eta_buf.alloc(sizeof(float) * d.npts, st), c2eta_buf.p);
      if (in->alpha_coeff.numel > 1) alpha_d = up(alpha_tmp, in->alpha_coeff.data, (size_t)in->alpha_coeff.numel, st);
    }
    if (c0_map || het)
      ck(launch_medium_maps(c0_map ? (float*)c0sq_buf.p : nullptr, in->c0.data[0], ctau, ceta, alpha_d,
                            in->alpha_coeff.numel ? in->alpha_coeff.data[0] : 0.f, np_per_db, y, tan_py, eos,
                            d.npts, st),
         "medium maps");
    if (absorb && !het) {  // scalar medium: the same formulas on the host
      const double c = in->c0.data[0];
      const double al = in->alpha_coeff.data[0] * np_per_db;
      const double csq = (double)((float)c * (float)c);
      if (eos == 1) {
        const double cy1 = std::pow(c, y - 1.0);
        c2tau_m = Map{nullptr, (float)(csq * (double)(float)(-2.0 * al * cy1))};
        c2eta_m = Map{nullptr, (float)(csq * (double)(float)(2.0 * al * cy1 * c * tan_py))};
      } else {
        tau_m = Map{nullptr, (float)(-2.0 * al * c)};
      }
    } else if (het) {
      if (eos == 1) {
        c2tau_m = Map{ctau, 0.f};
        c2eta_m = Map{ceta, 0.f};
      } else {
        tau_m = Map{ctau, 0.f};
      }
    }
    if (alpha_tmp.p) ck(cudaStreamSynchronize(st), "medium maps");  // alpha_tmp is freed on leaving
  }
  timer.mark("medium maps");
  // ----- fields and spectral work buffers -----
  const size_t fb = sizeof(float) * d.npts;
  const size_t sb = sizeof(float2) * (size_t)d.nxp * d.nrows;
  for (int a = 0; a < d.dim; ++a) {
    u_buf[a].alloc(fb, st);
    rho_buf[a].alloc(fb, st);
    ck(cudaMemsetAsync(u_buf[a].p, 0, fb, st), "memset");
    ck(cudaMemsetAsync(rho_buf[a].p, 0, fb, st), "memset");
  }
  const int nspec = axisym ? 5 : 4;
  for (int s = 0; s < nspec; ++s) {
    S_buf[s].alloc(sb, st);
    ck(cudaMemsetAsync(S_buf[s].p, 0, sb, st), "memset");
  }
  if (axisym) {
    // 1 / r on the radially staggered points, signed as u_r / r is mirrored
    // (kspaceFirstOrderAS.m:570-571, 920-923): [1/r, -flip(1/r), 1/r, -flip(1/r)]
    std::vector<float> ir(d.ny);
    for (int j = 0; j < d.ny; ++j) {
      const int q = j / ny0, m = j % ny0;
      const int src = (q == 0 || q == 2) ? m : ny0 - 1 - m;
      const double r = (src + 0.5) * in->dy;
      ir[j] = (float)(((q == 0 || q == 2) ? 1.0 : -1.0) / r);
    }
    up(inv_r_buf, ir.data(), ir.size(), st);
    ur_buf.alloc(fb, st);
  }
  err_buf.alloc(sizeof(int), st);
  ck(cudaMemsetAsync(err_buf.p, 0, sizeof(int), st), "memset");
  const char* no_graph = std::getenv("KWAVE_B200_NO_GRAPH");
  use_graph = !(no_graph && no_graph[0] == '1');
  // TMA-fed column passes for the compile-time lengths they support
  const char* no_tma = std::getenv("KWAVE_B200_NO_TMA");
  const bool tma_ok = !(no_tma && no_tma[0] == '1');
  // the TMA kernels' wait limit (microseconds; default 2 s) and the failure-
  // detection test's hook (a tile whose load is never issued)
  if (const char* w = std::getenv("KWAVE_B200_TMA_WAIT_US")) {
    const double us = std::atof(w);
    if (us > 0) tma_wait.limit_ns = (unsigned long long)(us * 1e3);
  }
  if (const char* k = std::getenv("KWAVE_B200_TEST_SKIP_TMA_TILE")) tma_wait.skip_tile = std::atoi(k);
  // use_tma[1]: the y pass in 3D, the fused last-axis operator in 2D
  use_tma[1] = tma_ok && (d.dim == 3 ? tma_col_supported(d.ny) : tma_fused_supported(d.ny));
  use_tma[2] = tma_ok && d.dim == 3 && tma_fused_supported(d.nz);
  for (int s = 0; s < nspec; ++s) {
    if (use_tma[1] && !make_spec_map(&map_y[s], S_buf[s].p, d, 1, d.ny)) use_tma[1] = false;
    if (use_tma[2] && !make_spec_map(&map_z[s], S_buf[s].p, d, 2, d.nz)) use_tma[2] = false;
  }
  // last-axis remainder tiles: when kx = nx / 2 would be alone in its column
  // tile, it is gathered for TL / 2 consecutive y into one tile instead
  {
    const int tl = use_tma[2] ? tma_lines(d.nz) : 0;
    rem_y = tl / 2;
    use_rem = use_tma[2] && tl % 2 == 0 && (d.nxh - 1) % tl == 0 && (d.nxh - 1) % 2 == 0 && d.ny % rem_y == 0;
    for (int s = 0; s < nspec && use_rem; ++s)
      if (!make_spec_map_rem(&map_zr[s], S_buf[s].p, d, d.nz, rem_y)) use_rem = false;
  }
  if (eos == 1) ploc_buf.alloc(fb, st);
  if (opt.p_final) {
    p_buf.alloc(fb, st);
    ck(cudaMemsetAsync(p_buf.p, 0, fb, st), "memset");
  }
  int one = 1;
  clock_buf.alloc(sizeof(int), st);
  ck(cudaMemcpyAsync(clock_buf.p, &one, sizeof(int), cudaMemcpyHostToDevice, st), "clock");
  clk.t = (const int*)clock_buf.p;
  clk.start = (int)opt.start_index;

  timer.mark("fields, TMA maps, clock");
  // ----- sources -----
  p0 = in->p0_source_flag != 0;
  if (p0) up(p0_buf, in->p0_source_input, (size_t)d.npts, st);
  setup_sources(in);

  timer.mark("sources");
  // ----- sensors -----
  setup_sensors(in);
  timer.mark("sensors");
  // ----- launch schedule: wisdom, tuning or the built-in choice -----
  select_schedule();
  in_user = nullptr;
  timer.mark("schedule");
  ck(cudaStreamSynchronize(st), "setup");
}

void Session::setup_sources(const kw_input* in) {
  psrc = SparseSource{};
  pdense = DenseSource{};
  if (in->p_source_flag) {
    if (!in->p_source_index || !in->p_source_input || in->p_source_index_numel == 0)
      throw KwError(KW_ERR_INVALID_ARGUMENT, "p_source_index / p_source_input missing");
    std::vector<int> si, sl;
    sort_indices(in->p_source_index, in->p_source_index_numel, d.npts, si, sl, "p_source_index");
    const int nsig = in->p_source_many ? (int)p_rows0 : 1;
    p_mode = (int)in->p_source_mode;
    if (p_mode < 0 || p_mode > 2) throw KwError(KW_ERR_INVALID_ARGUMENT, "p_source_mode must be 0, 1 or 2");
    p_len = (int)in->p_source_flag;
    const float* dw = nullptr;
    if (axisym) {
      // mirrored entries read their original point's signal, with its sign
      std::vector<float> w(sl.size());
      for (size_t j = 0; j < sl.size(); ++j) {
        w[j] = asx.p_w[sl[j]];
        sl[j] = asx.p_orig[sl[j]];
      }
      dw = up(psrc_w, w.data(), w.size(), st);
    }
    const int* didx = up(psrc_idx, si.data(), si.size(), st);
    const int* dslot = up(psrc_slot, sl.data(), sl.size(), st);
    const float* dsig = up(psrc_sig, in->p_source_input, (size_t)nsig * p_len, st);
    p_nsrc = (int)si.size();
    p_nsig = nsig;
    if (p_mode == 2) {
      pdense.len = p_len;
      if (nsig == 1) {
        // single signal: the corrected field is sig(t) * F^-1{cos(.) F{mask}}
        psrc_field.alloc(sizeof(float) * d.npts, st);
        std::vector<float> ones(1, 1.0f);
        DevBuf onebuf;
        const float* d1 = up(onebuf, ones.data(), 1, st);
        corrected_source((float*)psrc_field.p, didx, dslot, p_nsrc, d1, 1, 1, dw);
        ck(cudaStreamSynchronize(st), "source setup");
        pdense.field = (const float*)psrc_field.p;
        pdense.sig = dsig;
      } else {
        psrc_field.alloc(sizeof(float) * d.npts, st);
        pdense.field = (const float*)psrc_field.p;
        pdense.sig = nullptr;
        p_many_additive = true;
      }
    } else {
      psrc.n = p_nsrc;
      psrc.idx = didx;
      psrc.slot = dslot;
      psrc.sig = dsig;
      psrc.nrows_sig = nsig;
      psrc.len = p_len;
      psrc.mode = p_mode;  // 0 dirichlet, 1 add
      psrc.weight = dw;
    }
  }
  usrc = SparseSource{};
  for (int a = 0; a < 3; ++a) {
    udense[a] = DenseSource{};
    usig_d[a] = nullptr;
    u_len[a] = 0;
  }
  const uint64_t uf[3] = {in->ux_source_flag, in->uy_source_flag, in->uz_source_flag};
  const float* uin[3] = {in->ux_source_input, in->uy_source_input, in->uz_source_input};
  if (uf[0] || uf[1] || (d.dim == 3 && uf[2])) {
    if (!in->u_source_index || in->u_source_index_numel == 0)
      throw KwError(KW_ERR_INVALID_ARGUMENT, "u_source_index missing");
    std::vector<int> si, sl;
    sort_indices(in->u_source_index, in->u_source_index_numel, d.npts, si, sl, "u_source_index");
    const int nsig = in->u_source_many ? (int)u_rows0 : 1;
    u_mode = (int)in->u_source_mode;
    if (u_mode < 0 || u_mode > 2) throw KwError(KW_ERR_INVALID_ARGUMENT, "u_source_mode must be 0, 1 or 2");
    const float* duw = nullptr;
    if (axisym) {
      std::vector<float> w(sl.size());
      for (size_t j = 0; j < sl.size(); ++j) {
        w[j] = asx.u_w[sl[j]];
        sl[j] = asx.u_orig[sl[j]];
      }
      duw = up(usrc_w, w.data(), w.size(), st);
    }
    const int* didx = up(usrc_idx, si.data(), si.size(), st);
    const int* dslot = up(usrc_slot, sl.data(), sl.size(), st);
    u_nsrc = (int)si.size();
    u_nsig = nsig;
    for (int a = 0; a < d.dim; ++a) {
      if (!uf[a]) continue;
      if (!uin[a]) throw KwError(KW_ERR_INVALID_ARGUMENT, "velocity source input missing");
      u_len[a] = (int)uf[a];
      usig_d[a] = up(usig_buf[a], uin[a], (size_t)nsig * u_len[a], st);
    }
    if (u_mode == 2) {
      for (int a = 0; a < d.dim; ++a) {
        if (!uf[a]) continue;
        udense[a].len = u_len[a];
        ufield_buf[a].alloc(sizeof(float) * d.npts, st);
        udense[a].field = (const float*)ufield_buf[a].p;
        if (nsig == 1) {
          if (!ones_ready) {
            std::vector<float> ones(1, 1.0f);
            const float* d1 = up(ones_buf, ones.data(), 1, st);
            corrected_source((float*)ufield_buf[a].p, didx, dslot, u_nsrc, d1, 1, 1, duw);
            ones_ready = true;
            ones_field = a;
          } else {
            ck(cudaMemcpyAsync(ufield_buf[a].p, ufield_buf[ones_field].p, sizeof(float) * d.npts,
                               cudaMemcpyDeviceToDevice, st), "copy");
          }
          udense[a].sig = usig_d[a];
        } else {
          udense[a].sig = nullptr;
          u_many_additive = true;
        }
      }
    } else {
      usrc.n = u_nsrc;
      usrc.idx = didx;
      usrc.slot = dslot;
      usrc.nrows_sig = nsig;
      usrc.mode = u_mode;
      usrc.len = 0;
      usrc.weight = duw;
    }
  }
  // transducer source (kspaceFirstOrder_inputChecking.m:1155-1213 builds
  // what the file holds; kspaceFirstOrder3D.m:886-902 applies it)
  if (in->transducer_source_flag) {
    if (d.dim != 3) throw KwError(KW_ERR_INVALID_ARGUMENT, "transducer sources are 3D only");
    if (uf[0] || uf[1] || uf[2])
      throw KwError(KW_ERR_INVALID_ARGUMENT, "a transducer source excludes the velocity sources");
    if (!in->u_source_index || in->u_source_index_numel == 0)
      throw KwError(KW_ERR_INVALID_ARGUMENT, "u_source_index missing");
    if (!in->delay_mask || !in->transducer_source_input)
      throw KwError(KW_ERR_INVALID_ARGUMENT, "transducer source needs delay_mask and transducer_source_input");
    if (in->transducer_source_flag > (uint64_t)INT32_MAX ||
        in->transducer_source_input_numel > (uint64_t)INT32_MAX)
      throw KwError(KW_ERR_INVALID_ARGUMENT, "transducer signal too long");
    const uint64_t len = in->transducer_source_flag, nsig = in->transducer_source_input_numel;
    std::vector<int> si, sl;
    sort_indices(in->u_source_index, in->u_source_index_numel, d.npts, si, sl, "u_source_index");
    std::vector<int> dl(si.size());
    std::vector<float> ap;
    if (in->transducer_source_apodization) ap.resize(si.size());
    for (size_t j = 0; j < si.size(); ++j) {
      const uint64_t dm = in->delay_mask[sl[j]];
      // every sample read, delay_mask + t - 2 for t <= len, lies in the signal
      if (dm < 1 || dm - 1 + len > nsig)
        throw KwError(KW_ERR_INVALID_ARGUMENT, "delay_mask reads past the end of transducer_source_input");
      dl[j] = (int)(dm - 1);
      if (!ap.empty()) ap[j] = in->transducer_source_apodization[sl[j]];
    }
    // an additive x-velocity source whose entries read one signal at their
    // own offsets (SparseSource::delay, ::weight)
    u_nsrc = (int)si.size();
    u_nsig = 1;
    u_mode = 1;
    usrc.n = u_nsrc;
    usrc.idx = up(usrc_idx, si.data(), si.size(), st);
    usrc.slot = nullptr;
    usrc.nrows_sig = 1;
    usrc.mode = 1;
    usrc.len = 0;
    usrc.delay = up(tsrc_delay, dl.data(), dl.size(), st);
    usrc.weight = ap.empty() ? nullptr : up(tsrc_apod, ap.data(), ap.size(), st);
    usig_d[0] = up(usig_buf[0], in->transducer_source_input, nsig, st);
    u_len[0] = (int)len;
  }
}

// out = real(ifftn(source_kappa .* fftn(scatter(sig(:, t)))))
// (kspaceFirstOrder3D.m:813-821, 938-945)
void Session::corrected_source(float* out, const int* idx, const int* slot, int n, const float* sig,
                               int nrows_sig, int t, const float* weight) {
  ck(cudaMemsetAsync(out, 0, sizeof(float) * d.npts, st), "memset");
  ck(launch_scatter(out, idx, slot, n, sig, nrows_sig, t, weight, st), "scatter");
  float2* S = (float2*)S_buf[3].p;
  ck(launch_x_r2c(out, S, d, plan[0], twd[0], rowL, st), "x_r2c");
  run_spectral({3}, {3}, {SpecOp{OP_SRC_KAPPA, 0}}, 1);
  ck(launch_x_c2r(S, out, 0, d, plan[0], twd[0], rowL, st), "x_c2r");
}

// The y pass (3D) over z planes [z0, z0 + nzs) of the listed half-spectrum
// buffers, forward or inverse.
// dual_field >= 0 (TMA-fed pass only): bufs[dual_field] is derived from
// bufs[dual_src] times dual_tab along y as the pass runs (ColTmaArgs).
void Session::col_pass(bool inv, const std::vector<int>& bufs, int z0, int nzs, int dual_field, int dual_src,
                       const float2* dual_tab) {
  if (d.dim != 3 || bufs.empty()) return;
  const int n = (int)bufs.size();
  if (dual_field >= 0 && !use_tma[1]) throw KwError(KW_ERR_INTERNAL, "derived field in a y pass without TMA");
  if (use_tma[1]) {
    ColTmaArgs ca;
    std::memset(&ca, 0, sizeof(ca));
    for (int i = 0; i < n; ++i) ca.map[i] = map_y[bufs[i]];
    ca.dual_field = dual_field;
    ca.dual_src = dual_src;
    ca.dual_tab = dual_tab;
    ca.nfields = n;
    ca.ncx = (d.nxh + tma_lines(d.ny) - 1) / tma_lines(d.ny);
    ca.nouter = nzs;
    ca.outer0 = z0;
    ca.yaxis = 1;
    ca.err = (int*)err_buf.p;
    ca.wait = tma_wait;
    ck(launch_col_tma(inv, d.ny, ca, twd[1], st), "col_tma");
  } else {
    ColArgs ca{};
    for (int i = 0; i < n; ++i) ca.buf[i] = (float2*)S_buf[bufs[i]].p;
    ca.outer0 = z0;
    ca.ncols = d.nxh;
    ca.lstride = d.nxp;
    ca.ostride = (long long)d.nxp * d.ny;
    ca.tl = col_tl[1];
    ck(launch_col_fft(inv, ca, n, nzs, plan[1], twd[1], st), "col_fft");
  }
  ++launches_;
}

// The last-axis operator (z in 3D, y in 2D) over the whole volume: forward
// transform, multiply by `fanout` operators per input, inverse transforms.
void Session::fused_pass(const std::vector<int>& ins, const std::vector<int>& outs, const std::vector<SpecOp>& ops,
                         int fanout, const std::vector<int>& dual, const float2* dual_tab) {
  const int nin = (int)ins.size();
  const int nout = (int)outs.size();
  const int last = d.dim - 1;
  const int ns[3] = {d.nx, d.ny, d.nz};
  auto Sp = [&](int i) { return (float2*)S_buf[i].p; };
  if (use_tma[last]) {
    FusedTmaArgs fa;
    std::memset(&fa, 0, sizeof(fa));
    const CUtensorMap* maps = (d.dim == 3) ? map_z : map_y;
    for (int i = 0; i < nin; ++i) fa.in[i] = maps[ins[i]];
    for (int i = 0; i < nout; ++i) {
      fa.out[i] = maps[outs[i]];
      fa.outp[i] = Sp(outs[i]);
      fa.op[i] = ops[i];
      if (i < (int)dual.size() && dual[i] >= 0) {
        fa.dual_outp[i] = Sp(dual[i]);
        fa.dual_tab[i] = dual_tab;
      }
    }
    fa.lstride = (long long)d.nxp * (d.dim == 3 ? d.ny : 1);
    fa.ostride = d.nxp;
    fa.nin = nin;
    fa.fanout = fanout;
    fa.ncx = (d.nxh + tma_lines(ns[last]) - 1) / tma_lines(ns[last]);
    fa.nouter = (d.dim == 3) ? d.ny : 1;
    if (d.dim == 3 && use_rem) {
      fa.ncx = (d.nxh - 1) / tma_lines(ns[last]);
      fa.nrem = d.ny / rem_y;
      fa.rem_y = rem_y;
      for (int i = 0; i < nin; ++i) fa.in_rem[i] = map_zr[ins[i]];
    }
    fa.yaxis = (d.dim == 3) ? 2 : 1;
    fa.dim = d.dim;
    fa.ncols = d.nxh;
    fa.err = (int*)err_buf.p;
    fa.wait = tma_wait;
    ck(launch_fused_tma(ns[last], fa, twd[last], T, st), "fused_tma");
  } else {
    FusedArgs fa{};
    for (int i = 0; i < nin; ++i) fa.in[i] = Sp(ins[i]);
    for (int i = 0; i < nout; ++i) {
      fa.out[i] = Sp(outs[i]);
      fa.op[i] = ops[i];
      if (i < (int)dual.size() && dual[i] >= 0) {
        fa.dual_out[i] = Sp(dual[i]);
        fa.dual_tab[i] = dual_tab;
      }
    }
    fa.fanout = fanout;
    fa.ncols = d.nxh;
    fa.lstride = (long long)d.nxp * (d.dim == 3 ? d.ny : 1);
    fa.ostride = d.nxp;
    fa.tl = col_tl[last];
    ck(launch_fused_last(fa, nin, d.dim == 3 ? d.ny : 1, plan[last], twd[last], T, d.dim, st), "fused_last");
  }
  ++launches_;
}

// A whole-volume spectral operation on x-transformed buffers: y forward,
// last-axis operator, y inverse (setup work and "many"-signal sources).
void Session::run_spectral(std::vector<int> ins, std::vector<int> outs, std::vector<SpecOp> ops, int fanout) {
  col_pass(false, ins, 0, d.nz);
  fused_pass(ins, outs, ops, fanout);
  col_pass(true, outs, 0, d.nz);
}

// Gradient of p along each axis (kspaceFirstOrder3D.m:790-801) from S0
// (transformed along x and y) into S1..S3, still transformed along x and y.
// The x and y derivative factors do not vary along the last axis, so one
// inverse transform of kappa * F{p} serves both: S1 = F_z^-1{kappa F_z S0}
// (the x factor is applied when the row kernel reads S1), S2 = ddy(ky) S1,
// S3 = F_z^-1{ddz kappa F_z S0}.  In 2D the last axis is y: S1 as above,
// S2 = F_y^-1{ddy kappa F_y S0}.
// The y derivative of p (3D) is kappa P times the y derivative factor along
// ky.  With the TMA-fed y pass that product is formed in the y-inverse pass
// as kappa P's tiles are loaded (grad_col_inverse): the last-axis pass then
// writes two fields instead of three and the y pass reads kappa P's tiles
// twice, the second time from L2.  Otherwise the last-axis pass writes it as
// a second output of kappa P.
bool Session::grad_dual_in_y() const { return d.dim == 3 && use_tma[1]; }

void Session::grad_pass() {
  if (d.dim == 3) {
    if (grad_dual_in_y())
      fused_pass({0}, {1, 3}, {SpecOp{OP_KAPPA, 0}, SpecOp{OP_GRAD_POS, 2}}, 2);
    else
      fused_pass({0}, {1, 3}, {SpecOp{OP_KAPPA, 0}, SpecOp{OP_GRAD_POS, 2}}, 2, {2, -1}, T.ddk_pos[1]);
  } else {
    fused_pass({0}, {1, 2}, {SpecOp{OP_KAPPA, 0}, SpecOp{OP_GRAD_POS, 1}}, 2);
  }
}

// The y-inverse pass of the gradient spectra S1..S3 over z planes [z0, z0 + nzs).
void Session::grad_col_inverse(int z0, int nzs) {
  if (grad_dual_in_y()) {
    col_pass(true, {1, 3, 2}, z0, nzs, 2, 0, T.ddk_pos[1]);
  } else {
    std::vector<int> f;
    for (int a = 0; a < d.dim; ++a) f.push_back(a + 1);
    col_pass(true, f, z0, nzs);
  }
}

// The y-inverse / row kernel / y-forward chain over z slabs; with two
// streams the slabs alternate between them and all start together.
// (Starting each slab after the previous slab's y-inverse pass, so that a
// y pass runs beside the other slab's row kernel, measured slower: 1.316
// against 1.260 ms per 256^3 step with two slabs, 1.308 against 1.282 with
// four.)
template <class F>
void Session::for_slabs(F&& body) {
  if (!st2) {
    for (int z0 = 0; z0 < d.nz; z0 += slab) body(z0, std::min(slab, d.nz - z0));
    return;
  }
  cudaStream_t main = st;
  ck(cudaEventRecord(fork_ev, main), "fork");
  ck(cudaStreamWaitEvent(st2, fork_ev, 0), "fork");
  int k = 0;
  for (int z0 = 0; z0 < d.nz; z0 += slab, ++k) {
    st = (k % 2) ? st2 : main;
    body(z0, std::min(slab, d.nz - z0));
  }
  st = main;
  ck(cudaEventRecord(join_ev, st2), "join");
  ck(cudaStreamWaitEvent(main, join_ev, 0), "join");
}

Dims Session::slab_dims(int z0, int nzs) const {
  Dims s = d;
  s.row0 = (long long)z0 * d.ny;
  s.row1 = (long long)(z0 + nzs) * d.ny;
  return s;
}

void Session::setup_sensors(const kw_input* in) {
  std::vector<int> si, sl;
  std::vector<int> vslot;
  if (in->sensor_interp_index) {
    // Cartesian points by linear interpolation: record the distinct
    // vertices, form the points on the device
    interp_k = d.dim + 1;
    if (!in->sensor_interp_weight || in->sensor_interp_numel == 0 || in->sensor_interp_numel % interp_k)
      throw KwError(KW_ERR_INVALID_ARGUMENT, "sensor_interp_index / _weight must hold Nd + 1 entries per point");
    if (in->sensor_mask_type != 0) throw KwError(KW_ERR_INVALID_ARGUMENT, "sensor interpolation needs sensor_mask_type 0");
    std::vector<uint64_t> verts(in->sensor_interp_index, in->sensor_interp_index + in->sensor_interp_numel);
    for (uint64_t v : verts)
      if (v < 1 || v > (uint64_t)d.npts) throw KwError(KW_ERR_INVALID_ARGUMENT, "sensor_interp_index holds an index outside the grid");
    std::sort(verts.begin(), verts.end());
    verts.erase(std::unique(verts.begin(), verts.end()), verts.end());
    vslot.resize(in->sensor_interp_numel);
    for (uint64_t e = 0; e < in->sensor_interp_numel; ++e)
      vslot[e] = (int)(std::lower_bound(verts.begin(), verts.end(), in->sensor_interp_index[e]) - verts.begin());
    nvert = (long long)verts.size();
    build_sensor_lists(verts.data(), verts.size(), si, sl);
    interp = true;
    ns = (long long)(in->sensor_interp_numel / interp_k);
  } else if (in->sensor_mask_type == 0) {
    if (!in->sensor_mask_index || in->sensor_mask_index_numel == 0)
      throw KwError(KW_ERR_INVALID_ARGUMENT, "sensor_mask_index missing");
    ns = (long long)in->sensor_mask_index_numel;
    build_sensor_lists(in->sensor_mask_index, (size_t)ns, si, sl);
  } else if (in->sensor_mask_type == 1) {
    if (!in->sensor_mask_corners || in->sensor_mask_corners_numel == 0 || in->sensor_mask_corners_numel % 6)
      throw KwError(KW_ERR_INVALID_ARGUMENT, "sensor_mask_corners must hold 6 values per cuboid");
    std::vector<uint64_t> lin;
    const uint64_t K = in->sensor_mask_corners_numel / 6;
    for (uint64_t k = 0; k < K; ++k) {
      const uint64_t* c = in->sensor_mask_corners + 6 * k;
      const uint64_t lim[3] = {(uint64_t)d.nx, (uint64_t)d.ny, (uint64_t)d.nz};
      for (int a = 0; a < 3; ++a)
        if (c[a] < 1 || c[a + 3] < c[a] || c[a + 3] > lim[a])
          throw KwError(KW_ERR_INVALID_ARGUMENT, "sensor_mask_corners outside the grid or not ordered");
      // concatenated find() per cuboid (kspaceFirstOrder_inputChecking.m:1615-1636)
      for (uint64_t z = c[2]; z <= c[5]; ++z)
        for (uint64_t y = c[1]; y <= c[4]; ++y)
          for (uint64_t x = c[0]; x <= c[3]; ++x)
            lin.push_back((x - 1) + (uint64_t)d.nx * ((y - 1) + (uint64_t)d.ny * (z - 1)) + 1);
    }
    ns = (long long)lin.size();
    build_sensor_lists(lin.data(), lin.size(), si, sl);
  } else {
    throw KwError(KW_ERR_INVALID_ARGUMENT, "sensor_mask_type must be 0 or 1");
  }
  if (opt.start_index > Nt) nrec = 0;
  else nrec = (long long)(Nt - opt.start_index + 1);
  // Raw series (p, u, u on the regular grid) recorded every step can exceed
  // the device: when streaming is allowed and they would take more than the
  // recording budget (KWAVE_B200_RECORD_BUDGET bytes, default a quarter of the
  // device memory), only a ring of steps is kept on the device and the caller
  // drains it in blocks.
  {
    const long long streams = (opt.p_raw ? 1 : 0) + d.dim * ((opt.u_raw ? 1 : 0) + (opt.u_non_staggered_raw ? 1 : 0));
    const double per_step = 4.0 * (double)ns * (double)streams;
    double budget = 0.0;
    if (const char* e = std::getenv("KWAVE_B200_RECORD_BUDGET")) budget = std::atof(e);
    if (!(budget > 0)) {
      size_t fr = 0, tot = 0;
      budget = cudaMemGetInfo(&fr, &tot) == cudaSuccess ? 0.25 * (double)tot : 16e9;
    }
    ring_rows = 0;
    if (allow_ring_ && streams && nrec > 0 && per_step * (double)nrec > budget)
      ring_rows = std::max<long long>(1, std::min<long long>(nrec, (long long)(budget / per_step)));
    drained = 0;
  }
  // sensor state for p and u
  auto mk = [&](Sensor& s) {
    s = Sensor{};
    s.mode = interp ? 3 : (dense_sensor ? 1 : 2);
    s.ns = (int)ns;
    s.ring = (int)ring_rows;
    s.idx = (dense_sensor || interp) ? nullptr : sidx_d;
    s.slot = (dense_sensor || interp) ? nullptr : sslot_d;
  };
  // the vertices' values of this step (one row, always overwritten)
  auto mkv = [&](Sensor& s, DevBuf& vals) {
    s = Sensor{};
    s.mode = dense_sensor ? 1 : 2;
    s.ns = (int)nvert;
    s.ring = 1;
    s.idx = dense_sensor ? nullptr : sidx_d;
    s.slot = dense_sensor ? nullptr : sslot_d;
    vals.alloc(sizeof(float) * (size_t)nvert, st);
    ck(cudaMemsetAsync(vals.p, 0, sizeof(float) * (size_t)nvert, st), "memset");
    s.raw = (float*)vals.p;
  };
  if (interp) {
    up(vslot_buf, vslot.data(), vslot.size(), st);
    std::vector<float> w(in->sensor_interp_weight, in->sensor_interp_weight + in->sensor_interp_numel);
    up(vweight_buf, w.data(), w.size(), st);
  }
  mk(sens_p);
  const size_t ser = sizeof(float) * (size_t)ns * (size_t)(ring_rows ? ring_rows : nrec);
  if (ring_rows && sens_p.ring != ring_rows)
    throw KwError(KW_ERR_INTERNAL, "streamed series: sensor ring not set");
  const size_t per = sizeof(float) * (size_t)ns;
  const size_t all = sizeof(float) * (size_t)d.npts;
  auto zalloc = [&](DevBuf& b, size_t n) -> void* {
    b.alloc(n, st);
    if (n) ck(cudaMemsetAsync(b.p, 0, n, st), "memset");
    return b.p;
  };
  if (opt.p_raw && nrec) sens_p.raw = (float*)zalloc(p_raw_buf, ser);
  if (opt.p_max) sens_p.vmax = (float*)zalloc(p_max_buf, per);
  if (opt.p_min) sens_p.vmin = (float*)zalloc(p_min_buf, per);
  if (opt.p_rms) {
    sens_p.rms = (float2*)zalloc(p_rms_buf, 2 * per);
    sens_p.rms_blk = (float*)zalloc(p_rmsb_buf, per);
    zalloc(p_rmsf_buf, per);
  }
  if (opt.p_max_all) sens_p.max_all = (float*)zalloc(p_maxall_buf, all);
  if (opt.p_min_all) sens_p.min_all = (float*)zalloc(p_minall_buf, all);
  for (int a = 0; a < d.dim; ++a) {
    mk(sens_u[a]);
    if (opt.u_raw && nrec) sens_u[a].raw = (float*)zalloc(u_raw_buf[a], ser);
    if (opt.u_max) sens_u[a].vmax = (float*)zalloc(u_max_buf[a], per);
    if (opt.u_min) sens_u[a].vmin = (float*)zalloc(u_min_buf[a], per);
    if (opt.u_rms) {
      sens_u[a].rms = (float2*)zalloc(u_rms_buf[a], 2 * per);
      sens_u[a].rms_blk = (float*)zalloc(u_rmsb_buf[a], per);
      zalloc(u_rmsf_buf[a], per);
    }
    if (opt.u_max_all) sens_u[a].max_all = (float*)zalloc(u_maxall_buf[a], all);
    if (opt.u_min_all) sens_u[a].min_all = (float*)zalloc(u_minall_buf[a], all);
    const bool any = sens_u[a].raw || sens_u[a].vmax || sens_u[a].vmin || sens_u[a].rms ||
                     sens_u[a].max_all || sens_u[a].min_all;
    if (!any) sens_u[a].mode = 0;
  }
  {
    const bool any = sens_p.raw || sens_p.vmax || sens_p.vmin || sens_p.rms || sens_p.max_all || sens_p.min_all;
    if (!any) sens_p.mode = 0;
  }
  if (opt.u_non_staggered_raw && nrec) {
    for (int a = 0; a < d.dim; ++a) {
      mk(sens_uns[a]);
      sens_uns[a].raw = (float*)zalloc(uns_raw_buf[a], ser);
    }
    uns_field_buf.alloc(all, st);
  }
  if (interp) {
    // the step kernels see the vertex sensors; the full-grid reductions,
    // which do not depend on the mask, move there with them
    auto split = [&](Sensor& pt, Sensor& vs, DevBuf& vals) {
      const bool per_point = pt.raw || pt.vmax || pt.vmin || pt.rms;
      if (!per_point && !pt.max_all && !pt.min_all) {
        vs = Sensor{};
        return;
      }
      mkv(vs, vals);
      if (!per_point) vs.raw = nullptr;
      vs.max_all = pt.max_all;
      vs.min_all = pt.min_all;
      pt.max_all = pt.min_all = nullptr;
      if (!per_point) pt.mode = 0;
    };
    split(sens_p, vsens_p, vval_p_buf);
    for (int a = 0; a < d.dim; ++a) {
      split(sens_u[a], vsens_u[a], vval_u_buf[a]);
      if (sens_uns[a].mode) split(sens_uns[a], vsens_uns[a], vval_uns_buf[a]);
    }
  }
}

void Session::interp_points(int which) {
  if (!interp) return;
  const int* vs = (const int*)vslot_buf.p;
  const float* w = (const float*)vweight_buf.p;
  if (which == 0 && vsens_p.raw) {
    ck(launch_interp_sensor(sens_p, vsens_p.raw, vs, w, interp_k, clk, st), "interp p");
    ++launches_;
  }
  for (int a = 0; a < d.dim; ++a) {
    const Sensor& pt = (which == 1) ? sens_u[a] : sens_uns[a];
    const Sensor& vx = (which == 1) ? vsens_u[a] : vsens_uns[a];
    if (which != 0 && vx.raw) {
      ck(launch_interp_sensor(pt, vx.raw, vs, w, interp_k, clk, st), "interp u");
      ++launches_;
    }
  }
}

// u on the regular grid at the sensors (kspaceFirstOrder_extractSensorData.m:109-120):
// u_a shifted by half a cell back along its own axis,
// real(ifft(exp(-i k_a d_a / 2) fft(u_a))), one component at a time through S0
// (free between the gradient and the rho update) and a scratch field.
void Session::record_non_staggered() {
  if (!uns_field_buf.p) return;
  float2* work = (float2*)S_buf[0].p;
  float* f = (float*)uns_field_buf.p;
  for (int a = 0; a < d.dim; ++a) {
    ck(launch_x_r2c((const float*)u_buf[a].p, work, d, plan[0], twd[0], rowL, st), "x_r2c");
    run_spectral({0}, {0}, {SpecOp{OP_SHIFT_NEG, a}}, 1);
    ck(launch_x_c2r(work, f, 0, d, plan[0], twd[0], rowL, st), "x_c2r");
    ck(launch_record_field(f, row_sens_uns(a), clk, d.npts, st), "record");
    launches_ += 3;  // r2c, c2r, record (the spectral passes count themselves)
  }
  interp_points(2);
}

void Session::build_sensor_lists(const uint64_t* lin, size_t n, std::vector<int>& si, std::vector<int>& sl) {
  // dense identity: every grid point in linear order
  dense_sensor = ((long long)n == d.npts);
  if (dense_sensor)
    for (long long j = 0; j < d.npts; ++j)
      if (lin[j] != (uint64_t)j + 1) {
        dense_sensor = false;
        break;
      }
  if (dense_sensor) return;
  std::vector<std::pair<long long, int>> v(n);
  for (size_t j = 0; j < n; ++j) {
    if (lin[j] < 1 || lin[j] > (uint64_t)d.npts)
      throw KwError(KW_ERR_INVALID_ARGUMENT, "sensor_mask_index holds an index outside the grid");
    v[j] = {(long long)lin[j] - 1, (int)j};
  }
  std::stable_sort(v.begin(), v.end(), [](auto& a, auto& b) { return a.first < b.first; });
  si.resize(v.size());
  sl.resize(v.size());
  for (size_t j = 0; j < v.size(); ++j) {
    si[j] = (int)v[j].first;
    sl[j] = v[j].second;
  }
  sidx_d = up(sidx_buf, si.data(), si.size(), st);
  sslot_d = up(sslot_buf, sl.data(), sl.size(), st);
}

// t = 1 with an initial pressure (kspaceFirstOrder3D.m:1021-1035):
// p = p0, rho_i = p0 / (dim c0^2), u_i = dt rho0_sg_inv grad_i(p0) / 2.
void Session::enqueue_init() {
  const float* p0d = (const float*)p0_buf.p;
  ck(launch_record_field(p0d, row_sens_p(), clk, d.npts, st), "record p0");
  interp_points(0);
  ++launches_;
  ck(launch_rho_init((float*)rho_buf[0].p, (float*)rho_buf[1].p, d.dim == 3 ? (float*)rho_buf[2].p : nullptr,
                     p0d, c0sq_m, d.dim, rho_box, d.nx, d.ny, d.npts, st), "rho init");
  ++launches_;
  float2* S[4] = {(float2*)S_buf[0].p, (float2*)S_buf[1].p, (float2*)S_buf[2].p, (float2*)S_buf[3].p};
  ck(launch_x_r2c(p0d, S[0], d, plan[0], twd[0], rowL, st), "x_r2c");
  ++launches_;
  col_pass(false, {0}, 0, d.nz);
  grad_pass();
  grad_col_inverse(0, d.nz);
  UArgs ua = u_args(S);
  ua.init = 1;
  ua.do_r2c = 0;
  ck(launch_x_u(ua, d, plan[0], twd[0], rowL, st), "x_u init");
  interp_points(1);
  ++launches_;
  record_non_staggered();
  // the x and y transforms of p for the next step's gradient
  ck(launch_x_r2c(p0d, S[0], d, plan[0], twd[0], rowL, st), "x_r2c");
  ++launches_;
  col_pass(false, {0}, 0, d.nz);
  if (p_buf.p)
    ck(cudaMemcpyAsync(p_buf.p, p0d, sizeof(float) * d.npts, cudaMemcpyDeviceToDevice, st), "p0 copy");
}

UArgs Session::u_args(float2* const* S) {
  UArgs ua{};
  ua.kmul[0] = T.ddk_pos[0];  // the x derivative factor, applied as S1 is read
  for (int a = 0; a < d.dim; ++a) {
    ua.S[a] = S[a + 1];
    ua.Sout[a] = S[a + 1];
    ua.u[a] = (float*)u_buf[a].p;
    ua.rinv[a] = rinv_m[a];
    ua.pml_sg[a] = pml_sg_d[a];
    ua.src_sig[a] = usig_d[a];
    ua.src_len[a] = u_len[a];
    ua.dsrc[a] = udense[a];
    ua.sens[a] = row_sens_u(a);
  }
  ua.dt = dtf;
  ua.init = 0;
  ua.do_r2c = 1;
  ua.src = usrc;
  ua.clk = clk;
  ua.wait = row_wait();
  return ua;
}

// One time step (kspaceFirstOrder3D.m:767-1206) as three chains, each a
// whole-volume last-axis operator followed, per z slab, by the y inverse,
// the fused row kernel and the y forward transform of its outputs.  A slab's
// half spectra stay in L2 from one kernel of the chain to the next.
// On entry S0 holds p transformed along x and y; on exit too.
// Steps whose launch sequence is the same every time (no initial-pressure
// start, not the last step, no per-step "many"-signal corrected source) are
// captured once as a CUDA graph and replayed: every time-dependent value
// (record index, source sample) is read on the device from the clock.
bool Session::graphable(uint64_t t) const {
  if (!use_graph) return false;
  if (t == 1 && p0) return false;
  if (t == Nt) return false;
  for (int a = 0; a < d.dim; ++a)
    if (u_many_additive && udense[a].field && (int)t <= u_len[a]) return false;
  if (p_many_additive && (int)t <= p_len) return false;
  return true;
}

void Session::enqueue_step() {
  const uint64_t t = t_done + 1;
  if (graphable(t)) {
    if (!graph_exec) {
      cudaGraph_t g = nullptr;
      ck(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "begin capture");
      const uint64_t l0 = launches_;
      enqueue_step_body(t);
      graph_launches = launches_ - l0;
      launches_ = l0;
      ck(cudaStreamEndCapture(st, &g), "end capture");
      graph = g;
      ++graph_gen;
      ck(cudaGraphInstantiate(&graph_exec, graph, 0), "graph instantiate");
    }
    ck(cudaGraphLaunch(graph_exec, st), "graph launch");
    launches_ += graph_launches;
  } else {
    enqueue_step_body(t);
  }
  ++t_done;
}

void Session::enqueue_step_body(uint64_t t) {
  if (t == 1 && p0) {
    enqueue_init();
  } else {
    float2* S[4] = {(float2*)S_buf[0].p, (float2*)S_buf[1].p, (float2*)S_buf[2].p, (float2*)S_buf[3].p};
    std::vector<int> f123, f12;
    for (int a = 0; a < d.dim; ++a) f123.push_back(a + 1);
    f12 = {1, 2};
    const bool last = (t == Nt);
    // (1) momentum: grad p -> u (kspaceFirstOrder3D.m:790-884)
    grad_pass();
    if (u_many_additive) {
      for (int a = 0; a < d.dim; ++a)
        if (udense[a].field && (int)t <= u_len[a]) {
          // S0 is free here: the gradient has been taken
          corrected_source_into((float*)ufield_buf[a].p, (const int*)usrc_idx.p, (const int*)usrc_slot.p, u_nsrc,
                                usig_d[a], u_nsig, (int)t, 0, (const float*)usrc_w.p);
        }
    }
    UArgs ua = u_args(S);
    for_slabs([&](int z0, int nzs) {
      grad_col_inverse(z0, nzs);
      ck(launch_x_u(ua, slab_dims(z0, nzs), plan[0], twd[0], rowL, st), "x_u");
      ++launches_;
      col_pass(false, f123, z0, nzs);
    });
    if (axisym) {
      // the radial term of the divergence: u_r / r, transformed along x
      // (kspaceFirstOrderAS.m:920-934)
      ck(launch_scale_rows((float*)ur_buf.p, (const float*)u_buf[1].p, (const float*)inv_r_buf.p, d.nx, d.ny,
                           d.npts, st), "u_r / r");
      ck(launch_x_r2c((const float*)ur_buf.p, (float2*)S_buf[4].p, d, plan[0], twd[0], rowL, st), "x_r2c");
      launches_ += 2;
    }
    interp_points(1);
    record_non_staggered();
    // (2) mass conservation: div u -> rho, EOS (:905-1017)
    {
      std::vector<SpecOp> ops;
      for (int a = 0; a < d.dim; ++a) ops.push_back(SpecOp{OP_GRAD_NEG, a});
      if (axisym) {
        // the radial divergence gains kappa * shift_neg * F{u_r / r}
        // (kspaceFirstOrderAS.m:930-931), summed into du_r/dr as x_rho reads it
        ops.push_back(SpecOp{OP_KAPPA_SHIFT_NEG, 1});
        fused_pass({1, 2, 4}, {1, 2, 4}, ops, 1);
      } else {
        fused_pass(f123, f123, ops, 1);
      }
    }
    if (p_many_additive && (int)t <= p_len)
      corrected_source_into((float*)psrc_field.p, (const int*)psrc_idx.p, (const int*)psrc_slot.p, p_nsrc,
                            (const float*)psrc_sig.p, p_nsig, (int)t, 0, (const float*)psrc_w.p);
    RhoArgs ra{};
    for (int a = 0; a < d.dim; ++a) {
      ra.S[a] = S[a + 1];
      ra.rho[a] = (float*)rho_buf[a].p;
      ra.pml[a] = pml_d[a];
    }
    ra.rho0 = rho0_m;
    ra.box = rho_box;
    ra.dt = dtf;
    ra.nonlinear = nonlinear;
    ra.bona = bona_m;
    ra.c0sq = c0sq_m;
    ra.eos = eos;
    ra.tau = tau_m;
    ra.src = psrc;
    ra.dsrc = pdense;
    ra.sens = row_sens_p();
    ra.clk = clk;
    ra.wait = row_wait();
    ra.S_rr = axisym ? (const float2*)S_buf[4].p : nullptr;
    if (eos == 1) {
      ra.p_loc = (float*)ploc_buf.p;
      ra.S_q = S[1];
      ra.S_r = S[2];
    } else {
      ra.p_out = last ? (float*)p_buf.p : nullptr;
      ra.S_p = S[0];
    }
    for_slabs([&](int z0, int nzs) {
      col_pass(true, f123, z0, nzs);
      ck(launch_x_rho(ra, slab_dims(z0, nzs), plan[0], twd[0], rowL, st), "x_rho");
      ++launches_;
      if (eos == 1)
        col_pass(false, f12, z0, nzs);
      else
        col_pass(false, {0}, z0, nzs);
    });
    if (eos != 1) interp_points(0);
    if (eos == 1) {
      // (3) power-law absorption and dispersion (:970-977)
      fused_pass(f12, f12, {SpecOp{OP_NABLA1, 0}, SpecOp{OP_NABLA2, 0}}, 1);
      EosArgs ea{};
      ea.S_a = S[1];
      ea.S_b = S[2];
      ea.p_loc = (const float*)ploc_buf.p;
      ea.c2tau = c2tau_m;
      ea.c2eta = c2eta_m;
      ea.p_out = last ? (float*)p_buf.p : nullptr;
      ea.S_p = S[0];
      ea.sens = row_sens_p();
      ea.clk = clk;
      ea.wait = row_wait();
      for_slabs([&](int z0, int nzs) {
        col_pass(true, f12, z0, nzs);
        ck(launch_x_eos(ea, slab_dims(z0, nzs), plan[0], twd[0], rowL, st), "x_eos");
        ++launches_;
        col_pass(false, {0}, z0, nzs);
      });
      interp_points(0);
    }
  }
  ck(launch_advance((int*)clock_buf.p, st), "advance");
  ++launches_;
}

// corrected source field for "many" signals, using `work` as spectral scratch
void Session::corrected_source_into(float* out, const int* idx, const int* slot, int n, const float* sig,
                                    int nrows_sig, int t, int work_i, const float* weight) {
  float2* work = (float2*)S_buf[work_i].p;
  ck(cudaMemsetAsync(out, 0, sizeof(float) * d.npts, st), "memset");
  ck(launch_scatter(out, idx, slot, n, sig, nrows_sig, t, weight, st), "scatter");
  ck(launch_x_r2c(out, work, d, plan[0], twd[0], rowL, st), "x_r2c");
  run_spectral({work_i}, {work_i}, {SpecOp{OP_SRC_KAPPA, 0}}, 1);
  ck(launch_x_c2r(work, out, 0, d, plan[0], twd[0], rowL, st), "x_c2r");
  launches_ += 4;
}

void Session::advance(uint64_t n) {
  if (t_done + n > Nt) throw KwError(KW_ERR_INVALID_ARGUMENT, "advance beyond Nt");
  if (ring_rows) {  // rows recorded but not yet drained must still fit the ring
    const long long after = std::min<long long>(nrec, std::max<long long>(0, (long long)(t_done + n) - (long long)opt.start_index + 1));
    if (after - drained > ring_rows) throw KwError(KW_ERR_INVALID_ARGUMENT, "drain the streamed series before advancing further");
  }
  ck(cudaEventRecord(ev0, st), "event");
  const uint64_t l0 = launches_;
  for (uint64_t i = 0; i < n; ++i) enqueue_step();
  last_launches = launches_ - l0;
  last_steps = n;
  ck(cudaEventRecord(ev1, st), "event");
  cudaEvent_t e = nullptr;
  if (!spare_ev.empty()) {
    e = spare_ev.back();
    spare_ev.pop_back();
  } else {
    ck(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
  }
  pending_ev.push_back(e);
  ck(cudaEventRecord(e, st), "event");
}

void Session::set_priority(int priority) {
  int least = 0, greatest = 0;
  ck(cudaDeviceGetStreamPriorityRange(&least, &greatest), "stream priority range");
  priority = std::max(greatest, std::min(least, priority));
  ck(cudaStreamSynchronize(st), "sync");
  in_flight();
  cudaStream_t ns = nullptr;
  ck(cudaStreamCreateWithPriority(&ns, cudaStreamNonBlocking, priority), "cudaStreamCreateWithPriority");
  ck(cudaStreamDestroy(st), "cudaStreamDestroy");
  st = ns;  // the step graph is launched on whatever stream the session holds
}

// Everything a step reads from the previous one: the split densities, the
// staggered velocities, the pressure spectrum S0 (p transformed along x and
// y, raw), and every sensor accumulator.  Source fields, medium maps and
// operator tables are rebuilt from the input by setup().
std::vector<std::pair<std::string, DevBuf*>> Session::state_buffers() {
  std::vector<std::pair<std::string, DevBuf*>> v;
  const char* c = "xyz";
  for (int a = 0; a < d.dim; ++a) {
    v.push_back({std::string("rho_") + c[a], &rho_buf[a]});
    v.push_back({std::string("u_") + c[a] + "_sg", &u_buf[a]});
  }
  v.push_back({"p_spectrum", &S_buf[0]});
  v.push_back({"p", &p_raw_buf});
  v.push_back({"p_max", &p_max_buf});
  v.push_back({"p_min", &p_min_buf});
  v.push_back({"p_rms_acc", &p_rms_buf});
  v.push_back({"p_rms_block", &p_rmsb_buf});
  v.push_back({"p_max_all", &p_maxall_buf});
  v.push_back({"p_min_all", &p_minall_buf});
  for (int a = 0; a < d.dim; ++a) {
    const std::string u = std::string("u") + c[a];
    v.push_back({u, &u_raw_buf[a]});
    v.push_back({u + "_max", &u_max_buf[a]});
    v.push_back({u + "_min", &u_min_buf[a]});
    v.push_back({u + "_rms_acc", &u_rms_buf[a]});
    v.push_back({u + "_rms_block", &u_rmsb_buf[a]});
    v.push_back({u + "_max_all", &u_maxall_buf[a]});
    v.push_back({u + "_min_all", &u_minall_buf[a]});
    v.push_back({u + "_non_staggered", &uns_raw_buf[a]});
  }
  return v;
}

void Session::save_checkpoint(const std::string& path) {
  sync();
  h5::Writer w;
  std::vector<std::vector<float>> host;
  host.reserve(64);
  for (auto& nb : state_buffers()) {
    DevBuf* b = nb.second;
    if (!b->p || !b->bytes) continue;
    host.emplace_back(b->bytes / sizeof(float));
    ck(cudaMemcpy(host.back().data(), b->p, b->bytes, cudaMemcpyDeviceToHost), "checkpoint d2h");
    w.dataset("/" + nb.first, h5::DType::F32, {(uint64_t)host.back().size()}, host.back().data());
  }
  const uint64_t meta[6] = {t_done, (uint64_t)d.nx, (uint64_t)d.ny, (uint64_t)d.nz, Nt, input_fp};
  const char* names[6] = {"t_index", "Nx", "Ny", "Nz", "Nt", "input_fingerprint"};
  for (int i = 0; i < 6; ++i) w.dataset(std::string("/") + names[i], h5::DType::U64, {1}, &meta[i]);
  w.root_attribute("created_by", kw_version());
  w.root_attribute("file_type", "checkpoint");
  w.root_attribute("major_version", "1");
  w.root_attribute("minor_version", "2");
  try {
    w.write(path);
  } catch (const h5::Error& e) {
    throw KwError(KW_ERR_IO, e.what());
  }
}

void Session::restore_checkpoint(const std::string& path) {
  if (t_done != 0) throw KwError(KW_ERR_INVALID_ARGUMENT, "a checkpoint is restored into a fresh session only");
  try {
    h5::Reader r(path);
    if (r.attribute_string("/", "file_type") != "checkpoint")
      throw KwError(KW_ERR_IO, path + " is not a checkpoint file");
    auto one = [&](const char* n) -> uint64_t {
      auto v = r.read_u64(std::string("/") + n);
      if (v.size() != 1) throw KwError(KW_ERR_IO, std::string("checkpoint lacks ") + n);
      return v[0];
    };
    if (one("Nx") != (uint64_t)d.nx || one("Ny") != (uint64_t)d.ny || one("Nz") != (uint64_t)d.nz ||
        one("Nt") != Nt)
      throw KwError(KW_ERR_INVALID_ARGUMENT, "the checkpoint belongs to a different simulation");
    if (!r.exists("/input_fingerprint") || one("input_fingerprint") != input_fp)
      throw KwError(KW_ERR_INVALID_ARGUMENT,
                    "the checkpoint belongs to a different simulation (its input fingerprint differs: medium, "
                    "sources, sensor or time step)");
    const uint64_t t = one("t_index");
    if (t > Nt) throw KwError(KW_ERR_IO, "checkpoint time index beyond Nt");
    for (auto& nb : state_buffers()) {
      DevBuf* b = nb.second;
      if (!b->p || !b->bytes) continue;
      const std::string name = "/" + nb.first;
      if (!r.exists(name))
        throw KwError(KW_ERR_INVALID_ARGUMENT, "checkpoint lacks " + nb.first + " (recorded outputs differ)");
      std::vector<float> v = r.read_float(name);
      if (v.size() * sizeof(float) != b->bytes) throw KwError(KW_ERR_IO, "checkpoint dataset size of " + nb.first);
      ck(cudaMemcpy(b->p, v.data(), b->bytes, cudaMemcpyHostToDevice), "checkpoint h2d");
    }
    t_done = t;
    const int clock = (int)t + 1;  // the device clock holds the index of the next step
    ck(cudaMemcpy(clock_buf.p, &clock, sizeof(int), cudaMemcpyHostToDevice), "clock");
  } catch (const h5::Error& e) {
    throw KwError(KW_ERR_IO, path + ": " + e.what());
  }
}

uint64_t Session::in_flight() {
  while (!pending_ev.empty()) {
    const cudaError_t q = cudaEventQuery(pending_ev.front());
    if (q == cudaErrorNotReady) break;
    ck(q, "cudaEventQuery");
    spare_ev.push_back(pending_ev.front());
    pending_ev.pop_front();
  }
  return pending_ev.size();
}

float Session::elapsed_ms() {
  ck(cudaEventSynchronize(ev1), "event sync");
  float ms = 0;
  ck(cudaEventElapsedTime(&ms, ev0, ev1), "elapsed");
  return ms;
}

void Session::sync() {
  ck(cudaStreamSynchronize(st), "sync");
  int e = 0;
  ck(cudaMemcpy(&e, err_buf.p, sizeof(int), cudaMemcpyDeviceToHost), "error word");
  if (e) throw KwError(KW_ERR_CUDA, "a device-side wait timed out (error " + std::to_string(e) + ")");
}

static void d2h(float* dst, const void* src, size_t n, cudaStream_t st) {
  if (dst && src && n) ck(cudaMemcpyAsync(dst, src, n * sizeof(float), cudaMemcpyDeviceToHost, st), "d2h");
}

void Session::drain_raw(kw_output* out) {
  if (!ring_rows) return;
  const long long nr = std::min<long long>(nrec, std::max<long long>(0, (long long)t_done - (long long)opt.start_index + 1));
  float* dst[10] = {out->p, out->ux, out->uy, out->uz, out->ux_non_staggered, out->uy_non_staggered,
                    out->uz_non_staggered, nullptr, nullptr, nullptr};
  const void* src[10] = {p_raw_buf.p, u_raw_buf[0].p, u_raw_buf[1].p, u_raw_buf[2].p, uns_raw_buf[0].p,
                         uns_raw_buf[1].p, uns_raw_buf[2].p, nullptr, nullptr, nullptr};
  for (long long r = drained; r < nr;) {
    const long long slot = r % ring_rows;
    const long long cnt = std::min(nr - r, ring_rows - slot);  // contiguous up to the ring's end
    for (int k = 0; k < 7; ++k)
      if (dst[k] && src[k])
        ck(cudaMemcpyAsync(dst[k] + (size_t)r * ns, (const float*)src[k] + (size_t)slot * ns,
                           sizeof(float) * (size_t)cnt * (size_t)ns, cudaMemcpyDeviceToHost, st),
           "drain");
    r += cnt;
  }
  ck(cudaStreamSynchronize(st), "drain");
  drained = nr;
}

void Session::read(kw_output* out) {
  if (!out) throw KwError(KW_ERR_INVALID_ARGUMENT, "output must not be NULL");
  drain_raw(out);
  const long long nr = std::min<long long>(nrec, std::max<long long>(0, (long long)t_done - (long long)opt.start_index + 1));
  const float inv = nr > 0 ? 1.0f / (float)nr : 0.f;
  const int partial = (nr % kRmsBlock) != 0;  // a block of the blocked rms sum is still open
  if (p_rms_buf.p)
    ck(launch_rms_final((const float2*)p_rms_buf.p, (const float*)p_rmsb_buf.p, partial, (float*)p_rmsf_buf.p, ns,
                        inv, st),
       "rms");
  for (int a = 0; a < d.dim; ++a)
    if (u_rms_buf[a].p)
      ck(launch_rms_final((const float2*)u_rms_buf[a].p, (const float*)u_rmsb_buf[a].p, partial,
                          (float*)u_rmsf_buf[a].p, ns, inv, st),
         "rms");
  const size_t ser = ring_rows ? 0 : (size_t)ns * (size_t)nrec, per = (size_t)ns;
  const size_t all = axisym ? (size_t)d.nx * ny0 : (size_t)d.npts;  // axisymmetric: the unmirrored quarter
  d2h(out->p, p_raw_buf.p, ser, st);
  d2h(out->p_max, p_max_buf.p, per, st);
  d2h(out->p_min, p_min_buf.p, per, st);
  d2h(out->p_rms, p_rmsf_buf.p, per, st);
  d2h(out->p_max_all, p_maxall_buf.p, all, st);
  d2h(out->p_min_all, p_minall_buf.p, all, st);
  d2h(out->p_final, p_buf.p, all, st);
  float* ur[3] = {out->ux, out->uy, out->uz};
  float* umx[3] = {out->ux_max, out->uy_max, out->uz_max};
  float* umn[3] = {out->ux_min, out->uy_min, out->uz_min};
  float* urm[3] = {out->ux_rms, out->uy_rms, out->uz_rms};
  float* uma[3] = {out->ux_max_all, out->uy_max_all, out->uz_max_all};
  float* umi[3] = {out->ux_min_all, out->uy_min_all, out->uz_min_all};
  float* ufi[3] = {out->ux_final, out->uy_final, out->uz_final};
  float* uns[3] = {out->ux_non_staggered, out->uy_non_staggered, out->uz_non_staggered};
  for (int a = 0; a < d.dim; ++a) {
    d2h(ur[a], u_raw_buf[a].p, ser, st);
    d2h(umx[a], u_max_buf[a].p, per, st);
    d2h(umn[a], u_min_buf[a].p, per, st);
    d2h(urm[a], u_rmsf_buf[a].p, per, st);
    d2h(uma[a], u_maxall_buf[a].p, all, st);
    d2h(umi[a], u_minall_buf[a].p, all, st);
    if (opt.u_final) d2h(ufi[a], u_buf[a].p, all, st);
    d2h(uns[a], uns_raw_buf[a].p, ser, st);
  }
  sync();
}

Session::~Session() {
  if (st) cudaStreamSynchronize(st);
  if (graph_exec) cudaGraphExecDestroy(graph_exec);
  if (graph) cudaGraphDestroy(graph);
  if (ev0) cudaEventDestroy(ev0);
  if (ev1) cudaEventDestroy(ev1);
  if (st2) {
    cudaStreamSynchronize(st2);
    cudaStreamDestroy(st2);
  }
  if (fork_ev) cudaEventDestroy(fork_ev);
  if (join_ev) cudaEventDestroy(join_ev);
  for (cudaEvent_t e : pending_ev) cudaEventDestroy(e);
  for (cudaEvent_t e : spare_ev) cudaEventDestroy(e);
  if (st) cudaStreamDestroy(st);
}

size_t Session::device_bytes_estimate(const kw_input* in, const kw_options* o) {
  const size_t n = (size_t)(in->Nx * in->Ny * in->Nz) * (in->axisymmetric_flag ? 4 : 1);
  const size_t dim = in->Nz == 1 ? 2 : 3;
  const size_t nxp = ((in->Nx / 2 + 1) + 1) / 2 * 2;
  const size_t nspec = in->axisymmetric_flag ? 5 : 4;
  size_t b = nspec * 8 * nxp * (n / in->Nx) + 2 * dim * 4 * n;  // spectra, u, rho
  b += 4 * n * (2 + dim);                                       // medium maps
  return b;
}

}  // namespace kwb

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
using kwb::KwError;
using kwb::Session;

static int set_status(kw_status* st, int code, const std::string& msg) {
  if (st) {
    st->code = code;
    std::snprintf(st->message, sizeof(st->message), "%s", msg.c_str());
  }
  return code;
}

template <class F>
static int guarded(kw_status* st, F&& f) {
  try {
    f();
    return set_status(st, KW_OK, "");
  } catch (const KwError& e) {
    return set_status(st, e.code, e.what());
  } catch (const std::bad_alloc&) {
    return set_status(st, KW_ERR_OUT_OF_MEMORY, "host allocation failed");
  } catch (const std::exception& e) {
    return set_status(st, KW_ERR_INTERNAL, e.what());
  }
}

static void select_device(const kw_options* opt) {
  if (opt && opt->device >= 0) {
    cudaError_t e = cudaSetDevice(opt->device);
    if (e != cudaSuccess) throw KwError(KW_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
  }
}

extern "C" {

const char* kw_version(void) { return "kwave_b200 0.1.0 (sm_100a)"; }

int kw_output_sizes_query(const kw_input* in, const kw_options* opt, kw_output_sizes* sizes, kw_status* status) {
  return guarded(status, [&] {
    if (!in || !opt || !sizes) throw KwError(KW_ERR_INVALID_ARGUMENT, "NULL argument");
    if (in->Nx < 1 || in->Ny < 1 || in->Nz < 1 || in->Nt < 1)
      throw KwError(KW_ERR_INVALID_ARGUMENT, "Nx, Ny, Nz and Nt must be positive");
    uint64_t nsens = 0;
    if (in->sensor_interp_index) {
      const uint64_t k = (in->Nz == 1 ? 3 : 4);
      if (in->sensor_interp_numel % k) throw KwError(KW_ERR_INVALID_ARGUMENT, "sensor_interp_numel must be a multiple of Nd + 1");
      nsens = in->sensor_interp_numel / k;
    } else if (in->sensor_mask_type == 0) {
      nsens = in->sensor_mask_index_numel;
    } else if (in->sensor_mask_type == 1) {
      if (!in->sensor_mask_corners || in->sensor_mask_corners_numel % 6)
        throw KwError(KW_ERR_INVALID_ARGUMENT, "sensor_mask_corners must hold 6 values per cuboid");
      for (uint64_t k = 0; k < in->sensor_mask_corners_numel / 6; ++k) {
        const uint64_t* c = in->sensor_mask_corners + 6 * k;
        uint64_t m = 1;
        for (int a = 0; a < 3; ++a) {
          if (c[a + 3] < c[a]) throw KwError(KW_ERR_INVALID_ARGUMENT, "sensor_mask_corners not ordered");
          m *= c[a + 3] - c[a] + 1;
        }
        nsens += m;
      }
    } else {
      throw KwError(KW_ERR_INVALID_ARGUMENT, "sensor_mask_type must be 0 or 1");
    }
    const uint64_t s = opt->start_index ? opt->start_index : 1;
    sizes->num_sensor_points = nsens;
    sizes->num_recorded_steps = (s > in->Nt) ? 0 : in->Nt - s + 1;
    sizes->grid_points = in->Nx * in->Ny * in->Nz;
    sizes->device_bytes = Session::device_bytes_estimate(in, opt);
  });
}

int kw_session_create(const kw_input* in, const kw_options* opt, kw_session** session, kw_status* status) {
  return guarded(status, [&] {
    if (!session) throw KwError(KW_ERR_INVALID_ARGUMENT, "session must not be NULL");
    *session = nullptr;
    select_device(opt);
    auto h = std::make_unique<kw_session>();
    h->s = std::make_unique<Session>();
    h->s->setup(in, opt);
    *session = h.release();
  });
}

int kw_session_advance(kw_session* s, uint64_t nsteps, kw_status* status) {
  return guarded(status, [&] {
    if (!s) throw KwError(KW_ERR_INVALID_ARGUMENT, "NULL session");
    s->s->advance(nsteps);
  });
}

int kw_session_elapsed_ms(kw_session* s, float* ms, kw_status* status) {
  return guarded(status, [&] {
    if (!s || !ms) throw KwError(KW_ERR_INVALID_ARGUMENT, "NULL argument");
    *ms = s->s->elapsed_ms();
  });
}

int kw_session_sync(kw_session* s, kw_status* status) {
  return guarded(status, [&] {
    if (!s) throw KwError(KW_ERR_INVALID_ARGUMENT, "NULL session");
    s->s->sync();
  });
}

uint64_t kw_session_steps_done(const kw_session* s) { return s ? s->s->t_done : 0; }

int kw_stream_priority_range(int* least, int* greatest) {
  int l = 0, g = 0;
  const cudaError_t e = cudaDeviceGetStreamPriorityRange(&l, &g);
  if (least) *least = l;
  if (greatest) *greatest = g;
  return e == cudaSuccess ? KW_OK : KW_ERR_CUDA;
}

int kw_session_save(kw_session* s, const char* path, kw_status* status) {
  return guarded(status, [&] {
    if (!s || !path) throw KwError(KW_ERR_INVALID_ARGUMENT, "NULL argument");
    s->s->save_checkpoint(path);
  });
}

int kw_session_restore(kw_session* s, const char* path, kw_status* status) {
  return guarded(status, [&] {
    if (!s || !path) throw KwError(KW_ERR_INVALID_ARGUMENT, "NULL argument");
    s->s->restore_checkpoint(path);
  });
}

int kw_session_set_priority(kw_session* s, int priority, kw_status* status) {
  return guarded(status, [&] {
    if (!s) throw KwError(KW_ERR_INVALID_ARGUMENT, "NULL session");
    s->s->set_priority(priority);
  });
}

int kw_session_query(kw_session* s, uint64_t* in_flight, kw_status* status) {
  return guarded(status, [&] {
    if (!s || !in_flight) throw KwError(KW_ERR_INVALID_ARGUMENT, "NULL argument");
    *in_flight = s->s->in_flight();
  });
}

int kw_session_read(kw_session* s, kw_output* out, kw_status* status) {
  return guarded(status, [&] {
    if (!s) throw KwError(KW_ERR_INVALID_ARGUMENT, "NULL session");
    s->s->read(out);
  });
}

void* kw_session_stream(kw_session* s) { return s ? (void*)s->s->st : nullptr; }

uint64_t kw_session_launches_per_step(const kw_session* s) { return s ? s->s->last_launches_per_step() : 0; }

void kw_session_destroy(kw_session* s) { delete s; }

int kw_session_schedule(const kw_session* s, kw_schedule* sched) {
  if (!s || !sched) return KW_ERR_INVALID_ARGUMENT;
  const kwb::Schedule c = s->s->schedule();
  std::memset(sched, 0, sizeof(*sched));
  sched->slab_planes = c.slab;
  sched->streams = c.streams;
  sched->row_lines = c.row_lines;
  sched->col_lines = c.col_lines;
  sched->radix_plan = c.radix;
  return KW_OK;
}

int kw_solve(const kw_input* in, const kw_options* opt, kw_output* out, kw_status* status) {
  return guarded(status, [&] {
    select_device(opt);
    Session s;
    s.setup(in, opt, /*allow_ring=*/true);
    if (!s.ring_rows) {
      s.advance(s.Nt);
    } else {  // streamed raw series: advance a ring's worth of steps, drain, repeat
      while (s.t_done < s.Nt) {
        s.advance(std::min<uint64_t>(s.Nt - s.t_done, (uint64_t)s.ring_rows));
        s.drain_raw(out);
      }
    }
    s.read(out);
  });
}

}  // extern "C"
