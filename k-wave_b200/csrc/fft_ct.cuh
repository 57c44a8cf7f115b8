// Compile-time-sized line FFTs (the fast path of the solver's FFT engine).
//
// For a transform length N known at compile time, the radix plan, the
// per-stage butterfly counts, the thread -> butterfly mapping and every
// index division fold to constants.  T = N / RMAX threads cooperate on one
// line; in stage s each thread runs ceil((N / R_s) / T) radix-R_s butterflies
// held in registers.  Stages run in place: all butterfly inputs of a thread
// are loaded to registers, the block synchronises, and the outputs are
// written back to the same buffer, so a transform needs a single shared-
// memory tile (one buffer per field instead of a ping-pong pair).
#pragma once
#include "fft_engine.cuh"

namespace kwb {

// The compile-time plan, chosen so the largest radix sets T = N / RMAX
// threads per line: 16-point stages first, then 8 / 4 / 2, then 5, 3.
__host__ __device__ constexpr int ct_stage_count(int n) {
  if (n <= 0) return -1;
  int m = n, s = 0;
  while (m % 16 == 0) { m /= 16; ++s; }
  const int rs[5] = {8, 4, 2, 5, 3};
  for (int i = 0; i < 5; ++i)
    while (m % rs[i] == 0) { m /= rs[i]; ++s; }
  return m == 1 ? s : -1;
}

__host__ __device__ constexpr int ct_radix(int n, int stage) {
  if (n <= 0) return 1;
  int m = n, s = 0;
  while (m % 16 == 0) {
    if (s == stage) return 16;
    m /= 16;
    ++s;
  }
  const int rs[5] = {8, 4, 2, 5, 3};
  for (int i = 0; i < 5; ++i)
    while (m % rs[i] == 0) {
      if (s == stage) return rs[i];
      m /= rs[i];
      ++s;
    }
  return 1;
}

__host__ __device__ constexpr int ct_ns(int n, int stage) {  // product of the radices before `stage`
  int p = 1;
  for (int s = 0; s < stage; ++s) p *= ct_radix(n, s);
  return p;
}

__host__ __device__ constexpr int ct_rmax(int n) {
  int r = 1;
  for (int s = 0; s < ct_stage_count(n); ++s) r = ct_radix(n, s) > r ? ct_radix(n, s) : r;
  return r;
}

template <int N>
struct Ct {
  static constexpr int S = ct_stage_count(N);
  static constexpr int RMAX = ct_rmax(N);
  static constexpr int T = N / RMAX;  // threads per line
  static_assert(S > 0, "transform length must factor into 2, 3 and 5");
};

// Lines per thread block for a compile-time length: about 256 threads, at
// least 4 lines (a 32-byte sector of complex values per column tile row).
__host__ __device__ constexpr int ct_lines_of(int n) {
  if (n <= 0) return 0;
  int l = 256 / (n / ct_rmax(n));
  if (l < 4) l = 4;
  if (l > 32) l = 32;
  return l;
}
__host__ __device__ constexpr int ct_threads_of(int n) { return n <= 0 ? 0 : (n / ct_rmax(n)) * ct_lines_of(n); }

template <int N, int STAGE, bool INV, class L>
__device__ __forceinline__ void ct_stage(float2* buf, const float2* __restrict__ tw, int l, int tid, L lay) {
  constexpr int R = ct_radix(N, STAGE);
  constexpr int NS = ct_ns(N, STAGE);
  constexpr int NR = N / R;
  constexpr int T = Ct<N>::T;
  constexpr int NB = (NR + T - 1) / T;
  constexpr int TWS = N / (NS * R);
  float2 v[NB][R];
#pragma unroll
  for (int i = 0; i < NB; ++i) {
    const int j = tid + i * T;
    if (NR % T == 0 || j < NR) {
#pragma unroll
      for (int r = 0; r < R; ++r) v[i][r] = buf[lay(l, j + r * NR)];
      if constexpr (NS > 1) {
        const int k = j % NS;
#pragma unroll
        for (int r = 1; r < R; ++r) {
          float2 w = tw[k * r * TWS];
          if (INV) w.y = -w.y;
          v[i][r] = c_mul(v[i][r], w);
        }
      }
      dft<R, INV>(v[i]);
    }
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < NB; ++i) {
    const int j = tid + i * T;
    if (NR % T == 0 || j < NR) {
      const int k = j % NS;
      const int idx = (j / NS) * NS * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) buf[lay(l, idx + r * NS)] = v[i][r];
    }
  }
  __syncthreads();
}

// One stage with caller-supplied element access: ld(l, pos) returns the
// input element, st(l, pos, v) stores an output element.  No barriers: the
// caller synchronises (between the loads and stores when they alias, and
// before the outputs are read).
template <int N, int STAGE, bool INV, class LD, class ST>
__device__ __forceinline__ void ct_stage_io(const float2* __restrict__ tw, int l, int tid, LD ld, ST st) {
  constexpr int R = ct_radix(N, STAGE);
  constexpr int NS = ct_ns(N, STAGE);
  constexpr int NR = N / R;
  constexpr int T = Ct<N>::T;
  constexpr int NB = (NR + T - 1) / T;
  constexpr int TWS = N / (NS * R);
#pragma unroll
  for (int i = 0; i < NB; ++i) {
    const int j = tid + i * T;
    if (NR % T == 0 || j < NR) {
      float2 v[R];
#pragma unroll
      for (int r = 0; r < R; ++r) v[r] = ld(l, j + r * NR);
      const int k = j % NS;
      if constexpr (NS > 1) {
#pragma unroll
        for (int r = 1; r < R; ++r) {
          float2 w = tw[k * r * TWS];
          if (INV) w.y = -w.y;
          v[r] = c_mul(v[r], w);
        }
      }
      dft<R, INV>(v);
      const int idx = (j / NS) * NS * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) st(l, idx + r * NS, v[r]);
    }
  }
}

// The first stage with a caller-supplied loader: ld(l, pos) returns input
// element pos of line l from wherever the caller keeps it (the row kernels
// build each packed line from two raw half-spectrum rows on the fly).  In
// place like ct_stage: every input is loaded before the block barrier and
// every output stored after it, so the inputs may alias the output buffer.
template <int N, bool INV, class L, class LD>
__device__ __forceinline__ void ct_stage0_ld(float2* buf, int l, int tid, L lay, LD ld) {
  constexpr int R = ct_radix(N, 0);
  constexpr int NR = N / R;
  constexpr int T = Ct<N>::T;
  constexpr int NB = (NR + T - 1) / T;
  float2 v[NB][R];
#pragma unroll
  for (int i = 0; i < NB; ++i) {
    const int j = tid + i * T;
    if (NR % T == 0 || j < NR) {
#pragma unroll
      for (int r = 0; r < R; ++r) v[i][r] = ld(l, j + r * NR);
      dft<R, INV>(v[i]);  // first stage: no twiddles
    }
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < NB; ++i) {
    const int j = tid + i * T;
    if (NR % T == 0 || j < NR) {
#pragma unroll
      for (int r = 0; r < R; ++r) buf[lay(l, j * R + r)] = v[i][r];
    }
  }
  __syncthreads();
}

template <int N, int STAGE, bool INV, class L>
__device__ __forceinline__ void ct_stages(float2* buf, const float2* __restrict__ tw, int l, int tid, L lay) {
  if constexpr (STAGE < Ct<N>::S) {
    ct_stage<N, STAGE, INV>(buf, tw, l, tid, lay);
    ct_stages<N, STAGE + 1, INV>(buf, tw, l, tid, lay);
  }
}

// Register hand-off between a forward transform and an inverse one of the
// same line.  Thread `tid` of a line owns positions tid + T*m, m < N/T, in
// two places: they are the outputs of its butterflies in the last stage
// (position j + r*NS, NS = N / R_last, j = tid + i*T) and the inputs of its
// butterflies in the first stage (position j + r*N/R_0), provided T divides
// N / R_last and N / R_0 (the largest radix is a multiple of the first and
// last ones: 64 = 16*4, 128 = 16*8, 256 = 16*16).  A spectral operator can
// then be applied in registers between the forward transform's last stage
// and the inverse transform's first, without a shared-memory round trip.
template <int N>
struct CtHandoff {
  static constexpr int S = Ct<N>::S;
  static constexpr int T = Ct<N>::T;
  static constexpr int M = N / T;  // positions per thread
  static constexpr bool OK = S >= 2 && (ct_ns(N, S - 1) % T == 0) && ((N / ct_radix(N, 0)) % T == 0);
};

// Forward last stage of line `l` read from `src`; u[m] receives position tid + T*m.
template <int N, class L>
__device__ __forceinline__ void ct_fwd_last_to_regs(const float2* __restrict__ src, const float2* __restrict__ tw,
                                                    int l, int tid, L lay, float2 (&u)[CtHandoff<N>::M]) {
  static_assert(CtHandoff<N>::OK, "no register hand-off for this plan");
  constexpr int STAGE = Ct<N>::S - 1;
  constexpr int R = ct_radix(N, STAGE);
  constexpr int NS = ct_ns(N, STAGE);  // = N / R: the stride of the outputs
  constexpr int NR = N / R;
  constexpr int T = Ct<N>::T;
  constexpr int TWS = N / (NS * R);
#pragma unroll
  for (int i = 0; i < NR / T; ++i) {
    const int j = tid + i * T;
    float2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = src[lay(l, j + r * NR)];
#pragma unroll
    for (int r = 1; r < R; ++r) v[r] = c_mul(v[r], tw[j * r * TWS]);  // k = j % NS = j
    dft<R, false>(v);
#pragma unroll
    for (int r = 0; r < R; ++r) u[i + r * (NS / T)] = v[r];  // position j + r * NS
  }
}

// Inverse first stage from registers (u[m] = position tid + T*m); stores its
// outputs to `dst` in the order the next stage reads (as ct_stage does).
template <int N, class L>
__device__ __forceinline__ void ct_inv_first_from_regs(const float2 (&u)[CtHandoff<N>::M], float2* __restrict__ dst,
                                                       int l, int tid, L lay) {
  static_assert(CtHandoff<N>::OK, "no register hand-off for this plan");
  constexpr int R = ct_radix(N, 0);
  constexpr int NR = N / R;
  constexpr int T = Ct<N>::T;
#pragma unroll
  for (int i = 0; i < NR / T; ++i) {
    const int j = tid + i * T;
    float2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = u[i + r * (NR / T)];  // position j + r * NR
    dft<R, true>(v);
#pragma unroll
    for (int r = 0; r < R; ++r) dst[lay(l, j * R + r)] = v[r];
  }
}

// In-place transform of LINES lines by T * LINES threads.  LINE_FAST maps
// consecutive threads to consecutive lines (column tiles, whose lines are
// adjacent in shared memory); otherwise to consecutive butterflies of one
// line (row tiles).  Must be called by every thread of the block (it
// synchronises); the caller synchronises before the call.
template <int N, bool INV, bool LINE_FAST, int LINES, class L>
__device__ __forceinline__ void ct_fft(float2* buf, const float2* __restrict__ tw, L lay) {
  constexpr int T = Ct<N>::T;
  int l, tid;
  if (LINE_FAST) {
    l = threadIdx.x % LINES;
    tid = threadIdx.x / LINES;
  } else {
    l = threadIdx.x / T;
    tid = threadIdx.x - l * T;
  }
  ct_stages<N, 0, INV>(buf, tw, l, tid, lay);
}

// Row tiles (consecutive threads on consecutive butterflies of a line): the
// first stage reads its inputs through `ld`, the others run in place.
template <int N, bool INV, class L, class LD>
__device__ __forceinline__ void ct_fft_rows_ld(float2* buf, const float2* __restrict__ tw, L lay, LD ld) {
  constexpr int T = Ct<N>::T;
  const int l = threadIdx.x / T, tid = threadIdx.x - l * T;
  ct_stage0_ld<N, INV>(buf, l, tid, lay, ld);
  ct_stages<N, 1, INV>(buf, tw, l, tid, lay);
}

}  // namespace kwb
