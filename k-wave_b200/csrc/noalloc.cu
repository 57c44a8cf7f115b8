// kw_kspace_gradient_noalloc: the k-space staggered gradient of a 2D field
// (the operator that turns an initial pressure into the first particle
// velocity, kspaceFirstOrder2D.m:911-921), computed without allocating any
// device memory.
//
// Who needs this: a host application that owns all device memory itself --
// MATLAB holding gpuArray data in its own pool, a PyTorch program on its
// caching allocator, or a real-time loop where a cudaMalloc / cudaFree
// (which may synchronise the whole device) is not acceptable -- can call
// this with buffers it already holds.  The solver entry points (kw_solve,
// kw_session_*) allocate their fields and spectra per call and so cannot
// serve such callers.
//
// Where the memory comes from: the intermediate half spectra live in one
// file-scope __device__ array of fixed size (g_scratch below, 8 MiB: two
// spectra of the largest accepted grid, 1024 x 1024).  Every call looks up
// its address on the current device with cudaGetSymbolAddress and raises the
// kernel's shared-memory limit (cheap once the module is loaded, and never
// stale: a device reset or a new primary context gives a new address).  The
// first call on a device may load this module onto it, so make that first
// call, e.g. on a small grid, before any stream capture begins.
// Twiddle factors and operator values are generated inside the kernel, so
// nothing is copied from the host either.
//
// Nothing in the scratch has to start at zero: every element a phase reads
// was written by the previous phase of the same call, so it is never cleared.
//
// One scratch array per device means calls that overlap on a device -- two
// host threads, or two streams without an event between the calls -- race on
// it and corrupt each other's results.  Serialise them on one stream.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>

#include "fft_engine.cuh"
#include "kwave_b200.h"

namespace {

using namespace kwb;

constexpr int MAX_EDGE = KW_NOALLOC_MAX_EDGE;
constexpr int MAX_NXH = MAX_EDGE / 2 + 1;
constexpr int TL = 8;           // kx columns per CTA in the y pass
constexpr int THREADS = 256;
// y pass: twiddles + three column tiles; x passes need far less
constexpr size_t MAX_SMEM = sizeof(float2) * ((size_t)MAX_EDGE + 3ull * MAX_EDGE * TL);

// Two half spectra of the largest grid: [component][ky][kx], kx fastest.
static __device__ __align__(256) float2 g_scratch[2 * MAX_EDGE * MAX_NXH];

struct GradArgs {
  const float* f;    // input field [ny][nx]
  float* g[2];       // gradient components (g[1] may be null)
  float2* S[2];      // half spectra in the scratch
  FFTPlan px, py;
  int nx, ny, nxh, ngrad;
  float kx_step, ky_step;  // 2 pi / (N d)
  float half_cdt;          // c_ref dt / 2
  float inv_n;             // 1 / (nx ny)
};

// w_k = exp(-2 pi i k / n), evaluated in FP64 and rounded once.
__device__ void twiddles(float2* tw, int n) {
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    double s, c;
    sincospi(-2.0 * k / n, &s, &c);
    tw[k] = make_float2((float)c, (float)s);
  }
}

// k-Wave's wavenumber ordering: index j of an n-point axis is j for
// j <= (n-1)/2 and j - n above (so the Nyquist bin of an even axis is -n/2).
__device__ __forceinline__ int signed_index(int j, int n) { return j <= (n - 1) / 2 ? j : j - n; }

// i k exp(i k d / 2) for k = 2 pi m / (n d): the phase k d / 2 is pi m / n.
__device__ __forceinline__ float2 shifted_derivative(int m, int n, float kstep) {
  float s, c;
  sincospif((float)m / (float)n, &s, &c);
  const float k = m * kstep;
  return make_float2(-k * s, k * c);
}

__device__ __forceinline__ float sinc(float x) { return x == 0.f ? 1.f : sinf(x) / x; }

// Phase 0: R2C along x of row pairs into S[0].
// Phase 1: along y per group of TL kx columns: forward FFT, multiply by
//          kappa and the two shifted derivatives, inverse FFTs into S[0], S[1].
// Phase 2: C2R along x of S[c] into g[c] (blockIdx.y = component c).
__global__ void __launch_bounds__(THREADS) k_grad2d_noalloc(GradArgs a, int phase) {
  extern __shared__ float2 sm[];
  if (phase == 0) {
    const int n = a.nx, r = 2 * blockIdx.x;
    const RowLayout L{row_layout_stride(n)};
    float2* tw = sm;
    float2* b0 = tw + n;
    float2* b1 = b0 + L.ls;
    twiddles(tw, n);
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      const float re = a.f[(size_t)r * n + i];
      const float im = r + 1 < a.ny ? a.f[(size_t)(r + 1) * n + i] : 0.f;
      b0[L(0, i)] = make_float2(re, im);
    }
    __syncthreads();
    const float2* R = fft_lines<false, false>(b0, b1, tw, a.px, 1, L);
    for (int m = threadIdx.x; m < a.nxh; m += blockDim.x) {
      const float2 z = R[L(0, m)];
      const float2 zc = c_conj(R[L(0, m == 0 ? 0 : n - m)]);
      a.S[0][(size_t)r * a.nxh + m] = make_float2(0.5f * (z.x + zc.x), 0.5f * (z.y + zc.y));
      if (r + 1 < a.ny) a.S[0][(size_t)(r + 1) * a.nxh + m] = make_float2(0.5f * (z.y - zc.y), -0.5f * (z.x - zc.x));
    }
  } else if (phase == 1) {
    const int n = a.ny, m0 = blockIdx.x * TL;
    const ColLayout C{TL};
    float2* tw = sm;
    float2* b0 = tw + n;
    float2* b1 = b0 + n * TL;
    float2* b2 = b1 + n * TL;
    twiddles(tw, n);
    for (int i = threadIdx.x; i < n * TL; i += blockDim.x) {
      const int l = i % TL, j = i / TL, m = m0 + l;
      b0[C(l, j)] = m < a.nxh ? a.S[0][(size_t)j * a.nxh + m] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    float2* R = fft_lines<false, true>(b0, b1, tw, a.py, TL, C);
    float2* O = R == b0 ? b1 : b0;
    for (int i = threadIdx.x; i < n * TL; i += blockDim.x) {
      const int l = i % TL, j = i / TL;
      const int mx = signed_index(m0 + l, a.nx), my = signed_index(j, n);
      const float kx = mx * a.kx_step, ky = my * a.ky_step;
      const float kap = sinc(a.half_cdt * sqrtf(kx * kx + ky * ky));
      const float2 v = c_scale(R[C(l, j)], kap);
      R[C(l, j)] = c_mul(shifted_derivative(mx, a.nx, a.kx_step), v);
      if (a.ngrad == 2) O[C(l, j)] = c_mul(shifted_derivative(my, n, a.ky_step), v);
    }
    __syncthreads();
    const float2* r1 = fft_lines<true, true>(R, b2, tw, a.py, TL, C);
    for (int i = threadIdx.x; i < n * TL; i += blockDim.x) {
      const int l = i % TL, j = i / TL, m = m0 + l;
      if (m < a.nxh) a.S[0][(size_t)j * a.nxh + m] = r1[C(l, j)];
    }
    if (a.ngrad == 2) {
      __syncthreads();
      float2* freeb = r1 == R ? b2 : R;
      const float2* r2 = fft_lines<true, true>(O, freeb, tw, a.py, TL, C);
      for (int i = threadIdx.x; i < n * TL; i += blockDim.x) {
        const int l = i % TL, j = i / TL, m = m0 + l;
        if (m < a.nxh) a.S[1][(size_t)j * a.nxh + m] = r2[C(l, j)];
      }
    }
  } else {
    const int n = a.nx, r = 2 * blockIdx.x, c = blockIdx.y;
    const RowLayout L{row_layout_stride(n)};
    const float2* S = a.S[c];
    float* g = a.g[c];
    float2* tw = sm;
    float2* b0 = tw + n;
    float2* b1 = b0 + L.ls;
    twiddles(tw, n);
    const bool pair = r + 1 < a.ny;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
      const bool direct = k < a.nxh;
      const int m = direct ? k : n - k;
      float2 A = S[(size_t)r * a.nxh + m];
      float2 B = pair ? S[(size_t)(r + 1) * a.nxh + m] : make_float2(0.f, 0.f);
      if (m == 0 || 2 * m == n) {  // Hermitian projection: real(ifft(...))
        A.y = 0.f;
        B.y = 0.f;
      }
      if (!direct) {
        A = c_conj(A);
        B = c_conj(B);
      }
      b0[L(0, k)] = make_float2(A.x - B.y, A.y + B.x);
    }
    __syncthreads();
    const float2* R = fft_lines<true, false>(b0, b1, tw, a.px, 1, L);
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      const float2 z = R[L(0, i)];
      g[(size_t)r * n + i] = z.x * a.inv_n;
      if (pair) g[(size_t)(r + 1) * n + i] = z.y * a.inv_n;
    }
  }
}

int fail(kw_status* st, int code, const char* fmt, ...) __attribute__((format(printf, 3, 4)));
int fail(kw_status* st, int code, const char* fmt, ...) {
  if (st) {
    st->code = code;
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(st->message, sizeof(st->message), fmt, ap);
    va_end(ap);
  }
  return code;
}

// A pointer the kernel may dereference on device `dev`.
bool on_device(const void* p, int dev) {
  cudaPointerAttributes at{};
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (at.type == cudaMemoryTypeManaged) return true;
  return at.type == cudaMemoryTypeDevice && at.device == dev;
}

}  // namespace

extern "C" int kw_kspace_gradient_noalloc(const float* d_f, float* d_gx, float* d_gy, uint64_t nx, uint64_t ny,
                                          float dx, float dy, float c_ref, float dt, void* stream,
                                          kw_status* status) {
  if (status) {
    status->code = KW_OK;
    status->message[0] = 0;
  }
  if (!d_f || !d_gx) return fail(status, KW_ERR_INVALID_ARGUMENT, "d_f and d_gx must be device pointers");
  if (nx < 2 || ny < 2 || nx > (uint64_t)MAX_EDGE || ny > (uint64_t)MAX_EDGE)
    return fail(status, KW_ERR_INVALID_ARGUMENT,
                "grid %llu x %llu is outside 2..%d per edge, the size of the static scratch",
                (unsigned long long)nx, (unsigned long long)ny, MAX_EDGE);
  GradArgs a{};
  if (!make_fft_plan((int)nx, &a.px) || !make_fft_plan((int)ny, &a.py))
    return fail(status, KW_ERR_UNSUPPORTED, "grid edges must be products of 2, 3, 5 and 7 (got %llu x %llu)",
                (unsigned long long)nx, (unsigned long long)ny);
  if (!(dx > 0.f) || !(dy > 0.f) || !(dt > 0.f) || !(c_ref >= 0.f) || !std::isfinite(dx) || !std::isfinite(dy) ||
      !std::isfinite(dt) || !std::isfinite(c_ref))
    return fail(status, KW_ERR_INVALID_ARGUMENT, "dx, dy and dt must be positive and c_ref non-negative");

  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(status, KW_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
  if (!on_device(d_f, dev) || !on_device(d_gx, dev) || (d_gy && !on_device(d_gy, dev)))
    return fail(status, KW_ERR_INVALID_ARGUMENT, "d_f, d_gx and d_gy must be memory of the current device %d", dev);
  cudaStream_t st = (cudaStream_t)stream;
  if (st) {  // work enqueued on another device's stream would read this device's scratch address there
    int sdev = -1;
    e = cudaStreamGetDevice(st, &sdev);
    if (e != cudaSuccess) return fail(status, KW_ERR_INVALID_ARGUMENT, "stream: %s", cudaGetErrorString(e));
    if (sdev != dev)
      return fail(status, KW_ERR_INVALID_ARGUMENT, "the stream belongs to device %d, the current device is %d", sdev,
                  dev);
  }

  // the scratch array's address on the current device, looked up on every
  // call, with that device current
  void* scratch = nullptr;
  e = cudaGetSymbolAddress(&scratch, g_scratch);
  if (e != cudaSuccess) return fail(status, KW_ERR_CUDA, "cudaGetSymbolAddress(scratch): %s", cudaGetErrorString(e));
  e = cudaFuncSetAttribute(k_grad2d_noalloc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MAX_SMEM);
  if (e != cudaSuccess) return fail(status, KW_ERR_CUDA, "cudaFuncSetAttribute: %s", cudaGetErrorString(e));

  const int NX = (int)nx, NY = (int)ny;
  a.f = d_f;
  a.g[0] = d_gx;
  a.g[1] = d_gy;
  a.nx = NX;
  a.ny = NY;
  a.nxh = NX / 2 + 1;
  a.ngrad = d_gy ? 2 : 1;
  a.S[0] = (float2*)scratch;
  a.S[1] = (float2*)scratch + (size_t)MAX_EDGE * MAX_NXH;
  a.kx_step = (float)(2.0 * M_PI / (NX * (double)dx));
  a.ky_step = (float)(2.0 * M_PI / (NY * (double)dy));
  a.half_cdt = 0.5f * c_ref * dt;
  a.inv_n = (float)(1.0 / ((double)NX * NY));

  const size_t row_smem = sizeof(float2) * (NX + 2 * row_layout_stride(NX));
  const size_t col_smem = sizeof(float2) * ((size_t)NY + 3ull * NY * TL);
  const unsigned row_pairs = (unsigned)((NY + 1) / 2);
  k_grad2d_noalloc<<<row_pairs, THREADS, row_smem, st>>>(a, 0);
  k_grad2d_noalloc<<<(unsigned)((a.nxh + TL - 1) / TL), THREADS, col_smem, st>>>(a, 1);
  k_grad2d_noalloc<<<dim3(row_pairs, (unsigned)a.ngrad), THREADS, row_smem, st>>>(a, 2);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(status, KW_ERR_CUDA, "kernel launch: %s", cudaGetErrorString(e));
  return KW_OK;
}
