// kw_fft3d_*: a plain 2D / 3D real-to-complex transform (and its inverse)
// run by the solver's own FFT passes, so they can be compared with a
// library transform (cuFFT) and checked against numpy on their own.
//
// The time loop never calls this: it fuses each pass with the physics (the
// x transform into the row kernels, the last axis into the operator
// kernels).  Here the same kernels run bare, one pass per axis:
//   forward:  x  R2C   row kernel (k_x_r2c: two real rows per complex line)
//             y        column pass, in place (TMA-fed k_col_tma for the
//                      lengths it supports, else k_col_fft)
//             z        column pass along z, in place (3D only)
//   inverse:  z, y inverse column passes in place, then x C2R.
// The spectrum is the solver's half-spectrum layout [nz][ny][nxp] of complex
// FP32 values, kx in [0, nx/2], row pitch nxp = nx/2 + 1 rounded up to even.
// The inverse is unnormalised (inverse(forward(f)) = nx ny nz f), as the
// solver folds 1 / (nx ny nz) into its operators, and it overwrites the
// spectrum it reads.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "kernels.cuh"
#include "kernels_tma.cuh"
#include "kwave_b200.h"

namespace kwb {
cudaError_t launch_col_fft(bool inv, const ColArgs& a, int nfields, long long nouter, const FFTPlan& plan,
                           const float2* tw, cudaStream_t st);
cudaError_t launch_x_r2c(const float* f, float2* S, const Dims& d, const FFTPlan& plan, const float2* tw, int L,
                         cudaStream_t st);
cudaError_t launch_x_c2r(const float2* S, float* out, int accumulate, const Dims& d, const FFTPlan& plan,
                         const float2* tw, int L, cudaStream_t st);
bool tma_col_supported(int n);
int tma_lines(int n);
bool make_spec_map(CUtensorMap* m, void* base, const Dims& d, int yaxis, int n);
cudaError_t launch_col_tma(bool inv, int n, const ColTmaArgs& a, const float2* tw, cudaStream_t st);
}  // namespace kwb

using namespace kwb;

struct kw_fft3d_plan {
  Dims d{};
  FFTPlan plan[3]{};
  float2* tw[3]{};
  int rowL = 1;
  int col_tl[3]{};
  int* err = nullptr;  // the TMA passes' error word
  int device = 0;
};

namespace {

int fft_status(kw_status* st, int code, const std::string& msg) {
  if (st) {
    st->code = code;
    std::snprintf(st->message, sizeof(st->message), "%s", msg.c_str());
  }
  return code;
}

void fck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

// One column pass (axis 1: y, axis 2: z) over the whole spectrum, in place.
void column_pass(const kw_fft3d_plan& p, int axis, bool inv, float2* S, cudaStream_t st) {
  const Dims& d = p.d;
  const int n = axis == 1 ? d.ny : d.nz;
  if (tma_col_supported(n)) {
    ColTmaArgs ca;
    std::memset(&ca, 0, sizeof(ca));
    if (!make_spec_map(&ca.map[0], S, d, axis, n)) throw std::runtime_error("tensor map of the spectrum");
    ca.nfields = 1;
    ca.dual_field = ca.dual_src = -1;
    ca.ncx = (d.nxh + tma_lines(n) - 1) / tma_lines(n);
    ca.nouter = axis == 1 ? d.nz : d.ny;
    ca.outer0 = 0;
    ca.yaxis = axis;
    ca.err = p.err;
    ca.wait = TmaWaitArgs{2000000000ull, -1};
    fck(launch_col_tma(inv, n, ca, p.tw[axis], st), "column pass");
  } else {
    ColArgs ca{};
    ca.buf[0] = S;
    ca.outer0 = 0;
    ca.ncols = d.nxh;
    ca.lstride = axis == 1 ? d.nxp : (long long)d.nxp * d.ny;
    ca.ostride = axis == 1 ? (long long)d.nxp * d.ny : d.nxp;
    ca.tl = p.col_tl[axis];
    fck(launch_col_fft(inv, ca, 1, axis == 1 ? d.nz : d.ny, p.plan[axis], p.tw[axis], st), "column pass");
  }
}

}  // namespace

extern "C" {

int kw_fft3d_create(uint64_t nx, uint64_t ny, uint64_t nz, kw_fft3d_plan** out, kw_status* status) {
  if (!out) return fft_status(status, KW_ERR_INVALID_ARGUMENT, "plan pointer must not be NULL");
  *out = nullptr;
  if (nx < 2 || ny < 2 || nz < 1 || nx > 4096 || ny > 4096 || nz > 4096 || nx % 2)
    return fft_status(status, KW_ERR_INVALID_ARGUMENT, "grid must be nx x ny x nz with even nx, 2..4096 per edge");
  kw_fft3d_plan* p = new (std::nothrow) kw_fft3d_plan();
  if (!p) return fft_status(status, KW_ERR_OUT_OF_MEMORY, "host allocation failed");
  Dims& d = p->d;
  d.nx = (int)nx;
  d.ny = (int)ny;
  d.nz = (int)nz;
  d.dim = nz == 1 ? 2 : 3;
  d.nxh = d.nx / 2 + 1;
  d.nxp = (d.nxh + 1) / 2 * 2;
  d.nrows = (long long)d.ny * d.nz;
  d.npts = (long long)d.nx * d.nrows;
  d.row0 = 0;
  d.row1 = d.nrows;
  const int ns[3] = {d.nx, d.ny, d.nz};
  try {
    fck(cudaGetDevice(&p->device), "cudaGetDevice");
    for (int a = 0; a < d.dim; ++a) {
      if (!make_fft_plan(ns[a], &p->plan[a])) {
        kw_fft3d_destroy(p);
        return fft_status(status, KW_ERR_UNSUPPORTED, "edges must factor into 2, 3, 5 and 7");
      }
      std::vector<float2> tw(ns[a]);
      for (int k = 0; k < ns[a]; ++k) {
        const double ang = -2.0 * M_PI * (double)k / ns[a];
        tw[k] = make_float2((float)std::cos(ang), (float)std::sin(ang));
      }
      fck(cudaMalloc(&p->tw[a], sizeof(float2) * ns[a]), "cudaMalloc");
      fck(cudaMemcpy(p->tw[a], tw.data(), sizeof(float2) * ns[a], cudaMemcpyHostToDevice), "cudaMemcpy");
      int tl = 16;
      while (tl > 1 && (size_t)tl * ns[a] * 3 * 8 + ns[a] * 8 > 160 * 1024) tl /= 2;
      p->col_tl[a] = tl;
    }
    p->rowL = std::max(1, std::min(8, 2048 / d.nx));
    fck(cudaMalloc(&p->err, sizeof(int)), "cudaMalloc");
    fck(cudaMemset(p->err, 0, sizeof(int)), "cudaMemset");
  } catch (const std::exception& e) {
    kw_fft3d_destroy(p);
    return fft_status(status, KW_ERR_CUDA, e.what());
  }
  *out = p;
  return fft_status(status, KW_OK, "");
}

int kw_fft3d_exec(kw_fft3d_plan* p, int inverse, unsigned passes, float* d_real, void* d_spec, void* stream,
                  kw_status* status) {
  if (!p || !d_spec || (!d_real && (passes & 1u)))
    return fft_status(status, KW_ERR_INVALID_ARGUMENT, "plan, d_spec and (for the x pass) d_real are required");
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev != p->device)
    return fft_status(status, KW_ERR_INVALID_ARGUMENT, "the plan was made on another device");
  cudaStream_t st = (cudaStream_t)stream;
  float2* S = (float2*)d_spec;
  const bool x = passes & 1u, y = passes & 2u, z = (passes & 4u) && p->d.dim == 3;
  try {
    if (!inverse) {
      if (x) fck(launch_x_r2c(d_real, S, p->d, p->plan[0], p->tw[0], p->rowL, st), "x pass");
      if (y) column_pass(*p, 1, false, S, st);
      if (z) column_pass(*p, 2, false, S, st);
    } else {
      if (z) column_pass(*p, 2, true, S, st);
      if (y) column_pass(*p, 1, true, S, st);
      if (x) fck(launch_x_c2r(S, d_real, 0, p->d, p->plan[0], p->tw[0], p->rowL, st), "x pass");
    }
  } catch (const std::exception& e) {
    return fft_status(status, KW_ERR_CUDA, e.what());
  }
  return fft_status(status, KW_OK, "");
}

int kw_fft3d_check(kw_fft3d_plan* p, kw_status* status) {
  if (!p) return fft_status(status, KW_ERR_INVALID_ARGUMENT, "plan must not be NULL");
  int e = 0;
  if (cudaMemcpy(&e, p->err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
    return fft_status(status, KW_ERR_CUDA, "reading the error word");
  if (e) return fft_status(status, KW_ERR_CUDA, "a device-side wait timed out (error " + std::to_string(e) + ")");
  return fft_status(status, KW_OK, "");
}

void kw_fft3d_destroy(kw_fft3d_plan* p) {
  if (!p) return;
  for (float2* t : p->tw)
    if (t) cudaFree(t);
  if (p->err) cudaFree(p->err);
  delete p;
}

}  // extern "C"
