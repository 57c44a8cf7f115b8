// Solver kernels: per-axis FFT passes fused with the k-space operators and
// the split-field PML / conservation updates of k-Wave's fluid time loop
// (k-Wave/kspaceFirstOrder3D.m:767-1206, kspaceFirstOrder2D.m:710-1042).
//
// One time step is a pipeline of three spectral operations, each a forward
// transform, a k-space multiply and inverse transform(s):
//   grad p   -> u update          (kspaceFirstOrder3D.m:790-801)
//   div u    -> rho update, EOS   (:905-925, :963-1017)
//   absorption (power-law EOS)    (:970-977)
// The x axis is always the first forward / last inverse transform and is
// done by the row kernels (k_x_*), which fuse C2R -> elementwise physics ->
// R2C so each field row is read and written once.  The y axis (3D) is a
// column pass (k_col_fft) and the last axis (z in 3D, y in 2D) is done by
// k_fused_last: forward, operator multiply, inverse, in one kernel.
//
// Every FFT-carrying kernel is a template on NC, the length of the axis it
// transforms: NC > 0 selects the compile-time engine (fft_ct.cuh: in-place
// register-staged stages, one shared-memory buffer per field, index math
// folded to constants); NC == 0 is the runtime-plan engine for any other
// 2^a 3^b 5^c length.
#pragma once
#include "fft_ct.cuh"
#include "kernels.cuh"
#include "spec_ops.cuh"
#include "tma.cuh"

namespace kwb {

// Lines per block / threads per block of a kernel instantiation.
template <int NC>
struct Tile {
  static constexpr int LINES = ct_lines_of(NC);
  static constexpr int THREADS = NC > 0 ? ct_threads_of(NC) : kThreads;
};
// Row (x) tiles use half as many lines: smaller blocks, more of them per SM,
// so their load / transform / store phases overlap.
// The row kernels' 4-wide epilogue loops and their spectrum load / store
// loops run without unrolling: at 256 points per row this cut registers
// (k_x_rho 118 -> 90, k_x_u 72 -> 64) and instruction-fetch stalls, and the
// 256^3 step went from 1.43 to 1.36 ms against unroll factors of 2-4.
constexpr int kRowLoopUnroll = 1;

template <int NC>
struct RTile {
  static constexpr int LINES = NC > 0 ? (ct_lines_of(NC) / 2 > 0 ? ct_lines_of(NC) / 2 : 1) : 0;
  static constexpr int THREADS = NC > 0 ? (NC / ct_rmax(NC)) * LINES : kThreads;
  // blocks per SM the register budget is sized for (about 512 threads)
  static constexpr int MIN_BLOCKS = THREADS <= 128 ? 4 : (THREADS <= 256 ? 2 : 1);
};

// Transform the lines of a tile.  Compile-time lengths run in place in `a`;
// the runtime engine ping-pongs with `b`.  Returns the result buffer.
template <int NC, bool INV, bool COL, class L>
__device__ __forceinline__ float2* tile_fft(float2* a, float2* b, const float2* __restrict__ tw,
                                            const FFTPlan& plan, int nlines, L lay) {
  if constexpr (NC > 0) {
    ct_fft<NC, INV, COL, Tile<NC>::LINES>(a, tw, lay);
    return a;
  } else {
    return fft_lines<INV, COL>(a, b, tw, plan, nlines, lay);
  }
}

// ---------------------------------------------------------------------------
// column passes
// ---------------------------------------------------------------------------
template <int NC, bool INV>
__global__ void __launch_bounds__(Tile<NC>::THREADS) k_col_fft(ColArgs a, const __grid_constant__ FFTPlan plan,
                                                               const float2* __restrict__ tw_g) {
  extern __shared__ __align__(16) float2 sm[];
  constexpr bool CT = NC > 0;
  const int n = CT ? NC : plan.n;
  const int tl = CT ? Tile<NC>::LINES : a.tl;
  float2* tw = sm;
  float2* b0 = sm + n;
  float2* b1 = CT ? nullptr : b0 + tl * n;
  for (int i = threadIdx.x; i < n; i += blockDim.x) tw[i] = tw_g[i];
  float2* g = a.buf[blockIdx.z] + (long long)(a.outer0 + blockIdx.y) * a.ostride;
  const int c0 = blockIdx.x * tl;
  const int total = tl * n;
#pragma unroll 4
  for (int i = threadIdx.x; i < total; i += blockDim.x) {
    const int l = i % tl, p = i / tl, c = c0 + l;
    b0[i] = (c < a.ncols) ? g[p * a.lstride + c] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  float2* r = tile_fft<NC, INV, true>(b0, b1, tw, plan, tl, ColLayout{tl});
#pragma unroll 4
  for (int i = threadIdx.x; i < total; i += blockDim.x) {
    const int l = i % tl, p = i / tl, c = c0 + l;
    if (c < a.ncols) g[p * a.lstride + c] = r[i];
  }
}

// Last axis: forward transform, multiply by `fanout` operators, inverse
// transform each product.
template <int NC>
__global__ void __launch_bounds__(Tile<NC>::THREADS) k_fused_last(const __grid_constant__ FusedArgs a,
                                                                  const __grid_constant__ FFTPlan plan,
                                                                  const float2* __restrict__ tw_g,
                                                                  const __grid_constant__ SpecTables T, int dim) {
  extern __shared__ __align__(16) float2 sm[];
  constexpr bool CT = NC > 0;
  const int n = CT ? NC : plan.n;
  const int tl = CT ? Tile<NC>::LINES : a.tl;
  float2* tw = sm;
  float2* A = sm + n;
  float2* B = A + tl * n;
  float2* C = CT ? nullptr : B + tl * n;
  for (int i = threadIdx.x; i < n; i += blockDim.x) tw[i] = tw_g[i];
  const int g = blockIdx.z;
  const int outer = blockIdx.y;
  const long long off = (long long)outer * a.ostride;
  const float2* src = a.in[g] + off;
  const int c0 = blockIdx.x * tl;
  const int total = tl * n;
#pragma unroll 4
  for (int i = threadIdx.x; i < total; i += blockDim.x) {
    const int l = i % tl, p = i / tl, c = c0 + l;
    A[i] = (c < a.ncols) ? src[p * a.lstride + c] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  const ColLayout lay{tl};
  float2* F = tile_fft<NC, false, true>(A, B, tw, plan, tl, lay);
  float2* W1 = (F == A) ? B : A;
  float2* W2 = C;
  for (int o = 0; o < a.fanout; ++o) {
    const SpecOp op = a.op[g * a.fanout + o];
    for (int i = threadIdx.x; i < total; i += blockDim.x) {
      const int l = i % tl, p = i / tl;
      int c = c0 + l;
      if (c >= a.ncols) c = 0;
      const int iy = (dim == 3) ? outer : p;
      const int iz = (dim == 3) ? p : 0;
      W1[i] = c_mul(F[i], eval_op(op, T, dim, c, iy, iz));
    }
    __syncthreads();
    float2* R = tile_fft<NC, true, true>(W1, W2, tw, plan, tl, lay);
    float2* dst = a.out[g * a.fanout + o] + off;
    float2* dst2 = a.dual_out[g * a.fanout + o];
    const float2 dsc = dst2 ? __ldg(a.dual_tab[g * a.fanout + o] + outer) : make_float2(0.f, 0.f);
    if (dst2) dst2 += off;
#pragma unroll 4
    for (int i = threadIdx.x; i < total; i += blockDim.x) {
      const int l = i % tl, p = i / tl, c = c0 + l;
      if (c < a.ncols) {
        dst[p * a.lstride + c] = R[i];
        if (dst2) dst2[p * a.lstride + c] = c_mul(R[i], dsc);
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// row (x axis) helpers.  A row tile holds 2L consecutive rows packed two per
// complex line (row 2l in the real part, row 2l+1 in the imaginary part).
// ---------------------------------------------------------------------------
__device__ __forceinline__ float get_comp(const float2* b, RowLayout lay, int q, int x) {
  const float2& v = b[lay(q >> 1, x)];
  return (q & 1) ? v.y : v.x;
}
__device__ __forceinline__ void set_comp(float2* b, RowLayout lay, int q, int x, float v) {
  float* f = reinterpret_cast<float*>(b + lay(q >> 1, x));
  f[q & 1] = v;
}

// Build the full complex spectrum of each packed line from two half spectra
// (C2R).  The imaginary parts of the k = 0 and Nyquist bins are dropped,
// which is the Hermitian projection that real(ifftn(.)) performs.
template <int NC>
__device__ __forceinline__ void load_c2r(const float2* __restrict__ S, float2* buf, RowLayout lay, const Dims& d,
                                         long long r0, int L, const float2* __restrict__ kmul = nullptr,
                                         const float2* __restrict__ S2 = nullptr) {
  if constexpr (NC > 0 && NC % 4 == 0) {
    // paired 16-byte loads; each loaded bin k also fills its mirror n - k
    constexpr int n = NC, np = NC / 4 + 1;  // bin pairs (k, k+1), k even, k <= n/2
    const int total = L * np;
#pragma unroll (kRowLoopUnroll)
    for (int i = threadIdx.x; i < total; i += blockDim.x) {
      const int l = i / np, k = 2 * (i - l * np);
      const long long ra = r0 + 2 * l, rb = ra + 1;
      float4 A = make_float4(0.f, 0.f, 0.f, 0.f), B = A;
      if (ra < d.row1) A = *reinterpret_cast<const float4*>(S + ra * d.nxp + k);
      if (rb < d.row1) B = *reinterpret_cast<const float4*>(S + rb * d.nxp + k);
      if (S2) {
        float4 A2 = make_float4(0.f, 0.f, 0.f, 0.f), B2 = A2;
        if (ra < d.row1) A2 = *reinterpret_cast<const float4*>(S2 + ra * d.nxp + k);
        if (rb < d.row1) B2 = *reinterpret_cast<const float4*>(S2 + rb * d.nxp + k);
        A = make_float4(A.x + A2.x, A.y + A2.y, A.z + A2.z, A.w + A2.w);
        B = make_float4(B.x + B2.x, B.y + B2.y, B.z + B2.z, B.w + B2.w);
      }
      if (kmul) {
        const float2 m0 = __ldg(kmul + k), m1 = __ldg(kmul + min(k + 1, n / 2));
        float2 t = c_mul(make_float2(A.x, A.y), m0), u = c_mul(make_float2(A.z, A.w), m1);
        A = make_float4(t.x, t.y, u.x, u.y);
        t = c_mul(make_float2(B.x, B.y), m0);
        u = c_mul(make_float2(B.z, B.w), m1);
        B = make_float4(t.x, t.y, u.x, u.y);
      }
      if (k == 0) {
        A.y = 0.f;
        B.y = 0.f;
      }
      if (2 * k == n) {
        A.y = 0.f;
        B.y = 0.f;
      }
      buf[lay(l, k)] = make_float2(A.x - B.y, A.y + B.x);
      if (k > 0 && 2 * k < n) buf[lay(l, n - k)] = make_float2(A.x + B.y, B.x - A.y);
      if (2 * (k + 1) < n) {
        buf[lay(l, k + 1)] = make_float2(A.z - B.w, A.w + B.z);
        buf[lay(l, n - k - 1)] = make_float2(A.z + B.w, B.z - A.w);
      }
    }
    return;
  }
  const int n = NC > 0 ? NC : d.nx;
  const int total = L * n;
#pragma unroll 4
  for (int i = threadIdx.x; i < total; i += blockDim.x) {
    const int l = i / n, k = i - l * n;
    const long long ra = r0 + 2 * l, rb = ra + 1;
    const int kk = (2 * k <= n) ? k : n - k;
    float2 A = make_float2(0.f, 0.f), B = make_float2(0.f, 0.f);
    if (ra < d.row1) A = S[ra * d.nxp + kk];
    if (rb < d.row1) B = S[rb * d.nxp + kk];
    if (S2) {
      if (ra < d.row1) A = c_add(A, S2[ra * d.nxp + kk]);
      if (rb < d.row1) B = c_add(B, S2[rb * d.nxp + kk]);
    }
    if (kmul) {
      const float2 m = __ldg(kmul + kk);
      A = c_mul(A, m);
      B = c_mul(B, m);
    }
    if (2 * k > n) {
      A.y = -A.y;
      B.y = -B.y;
    } else if (k == 0 || 2 * k == n) {
      A.y = 0.f;
      B.y = 0.f;
    }
    buf[lay(l, k)] = make_float2(A.x - B.y, A.y + B.x);
  }
}

// Split each packed line's spectrum Z = FFT(a + i b) into the half spectra
// of a and b (R2C) and store them.
template <int NC>
__device__ __forceinline__ void store_r2c(const float2* buf, float2* __restrict__ S, RowLayout lay, const Dims& d,
                                          long long r0, int L) {
  if constexpr (NC > 0 && NC % 4 == 0) {
    constexpr int n = NC, nh = NC / 2 + 1, np = NC / 4 + 1;
    const int total = L * np;
#pragma unroll (kRowLoopUnroll)
    for (int i = threadIdx.x; i < total; i += blockDim.x) {
      const int l = i / np, k = 2 * (i - l * np);
      const long long ra = r0 + 2 * l, rb = ra + 1;
      const float2 z0 = buf[lay(l, k)], m0 = buf[lay(l, k == 0 ? 0 : n - k)];
      const float2 z1 = buf[lay(l, k + 1)], m1 = buf[lay(l, n - k - 1)];
      const float4 A = make_float4(0.5f * (z0.x + m0.x), 0.5f * (z0.y - m0.y), 0.5f * (z1.x + m1.x),
                                   0.5f * (z1.y - m1.y));
      const float4 B = make_float4(0.5f * (z0.y + m0.y), -0.5f * (z0.x - m0.x), 0.5f * (z1.y + m1.y),
                                   -0.5f * (z1.x - m1.x));
      if (k + 1 < nh) {
        if (ra < d.row1) *reinterpret_cast<float4*>(S + ra * d.nxp + k) = A;
        if (rb < d.row1) *reinterpret_cast<float4*>(S + rb * d.nxp + k) = B;
      } else {
        if (ra < d.row1) S[ra * d.nxp + k] = make_float2(A.x, A.y);
        if (rb < d.row1) S[rb * d.nxp + k] = make_float2(B.x, B.y);
      }
    }
    return;
  }
  const int n = NC > 0 ? NC : d.nx;
  const int nh = n / 2 + 1;
  const int total = L * nh;
#pragma unroll 4
  for (int i = threadIdx.x; i < total; i += blockDim.x) {
    const int l = i / nh, k = i - l * nh;
    const long long ra = r0 + 2 * l, rb = ra + 1;
    const float2 zk = buf[lay(l, k)];
    const float2 zn = buf[lay(l, k == 0 ? 0 : n - k)];
    const float2 A = make_float2(0.5f * (zk.x + zn.x), 0.5f * (zk.y - zn.y));
    const float2 B = make_float2(0.5f * (zk.y + zn.y), -0.5f * (zk.x - zn.x));
    if (ra < d.row1) S[ra * d.nxp + k] = A;
    if (rb < d.row1) S[rb * d.nxp + k] = B;
  }
}

__device__ __forceinline__ int lower_bound_i(const int* a, int n, long long v) {
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if ((long long)__ldg(a + mid) < v)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

// Range [lo, hi) of sorted indices that fall inside the tile's rows.
__device__ __forceinline__ void tile_range(const int* idx, int n, long long a, long long b, int* sh) {
  if (threadIdx.x == 0) {
    sh[0] = lower_bound_i(idx, n, a);
    sh[1] = lower_bound_i(idx, n, b);
  }
  __syncthreads();
}

// Row of the raw series that record index fi (1-based) goes to: a ring of
// s.ring rows when the series is streamed to the host in blocks.
__device__ __forceinline__ long long raw_row(const Sensor& s, int fi) {
  return s.ring ? (long long)((fi - 1) % s.ring) : (long long)(fi - 1);
}

// Kahan-compensated addition of x to {sum, compensation}.
__device__ __forceinline__ float2 kahan_acc(float2 acc, float x) {
  const float y = x - acc.y;
  const float t = acc.x + y;
  acc.y = (t - acc.x) - y;
  acc.x = t;
  return acc;
}

// Position of record index fi in its rms block, and whether fi ends it.
__device__ __forceinline__ int rms_pos(int fi) { return (fi - 1) % kRmsBlock; }

// The block partial sum after adding v^2 (b: the partial sum so far, unread
// at a block's first step).
__device__ __forceinline__ float rms_step(int j, float b, float v) {
  return j == 0 ? __fmul_rn(v, v) : __fmaf_rn(v, v, b);
}

// One recorded value into the blocked rms accumulators of `slot` (kRmsBlock).
__device__ __forceinline__ void rms_put(const Sensor& s, int fi, long long slot, float v) {
  const int j = rms_pos(fi);
  const float b = rms_step(j, j ? s.rms_blk[slot] : 0.f, v);
  if (j == kRmsBlock - 1)
    s.rms[slot] = kahan_acc(fi == kRmsBlock ? make_float2(0.f, 0.f) : s.rms[slot], b);
  else
    s.rms_blk[slot] = b;
}

__device__ __forceinline__ void sensor_put(const Sensor& s, int fi, long long slot, float v) {
  if (s.raw) s.raw[raw_row(s, fi) * s.ns + slot] = v;
  if (s.vmax) s.vmax[slot] = (fi == 1) ? v : fmaxf(s.vmax[slot], v);
  if (s.vmin) s.vmin[slot] = (fi == 1) ? v : fminf(s.vmin[slot], v);
  if (s.rms) rms_put(s, fi, slot, v);
}

__device__ __forceinline__ void sensor_all(const Sensor& s, int fi, long long gi, float v) {
  if (s.max_all) s.max_all[gi] = (fi == 1) ? v : fmaxf(s.max_all[gi], v);
  if (s.min_all) s.min_all[gi] = (fi == 1) ? v : fminf(s.min_all[gi], v);
}

__device__ __forceinline__ int record_index(const Clock& c) {
  const int t = *c.t;
  return (t >= c.start) ? (t - c.start + 1) : 0;
}

// Dense sensors for one grid point (mode 1) and full-grid reductions.
__device__ __forceinline__ void sensor_dense(const Sensor& s, int fi, long long gi, float v) {
  if (fi <= 0) return;
  if (s.mode == 1) sensor_put(s, fi, gi, v);
  sensor_all(s, fi, gi, v);
}

// ----- 4-wide (16-byte) variants for the compile-time path -----
__device__ __forceinline__ float4 ld4(const float* p, long long i) { return *reinterpret_cast<const float4*>(p + i); }
__device__ __forceinline__ void st4(float* p, long long i, float4 v) { *reinterpret_cast<float4*>(p + i) = v; }
__device__ __forceinline__ float4 map4(const Map& m, long long i) {
  return m.p ? __ldg(reinterpret_cast<const float4*>(m.p + i)) : make_float4(m.s, m.s, m.s, m.s);
}
__device__ __forceinline__ float4 max4(float4 a, float4 b) {
  return make_float4(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z), fmaxf(a.w, b.w));
}
__device__ __forceinline__ float4 min4(float4 a, float4 b) {
  return make_float4(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z), fminf(a.w, b.w));
}
// Dense sensors and full-grid reductions for 4 consecutive points, split
// into a load and a store part so that an epilogue issues every load of an
// iteration (its own inputs and the accumulators) before any store: a store
// through another pointer (p, say) would otherwise keep the accumulator loads
// behind it, a second memory round trip per iteration.
struct Acc4 {  // the accumulators loaded ahead: per-point max and the rms block partial sums
  float4 mx{}, bl{};
};
__device__ __forceinline__ void rms_load4(const Sensor& s, int fi, long long gi, Acc4& c) {
  if (rms_pos(fi) != 0) c.bl = ld4(s.rms_blk, gi);
}
// (at a block's end the Kahan pairs are loaded here, once per kRmsBlock steps)
__device__ __forceinline__ void rms_store4(const Sensor& s, int fi, long long gi, float4 v, const Acc4& c) {
  const int j = rms_pos(fi);
  const float4 b = make_float4(rms_step(j, c.bl.x, v.x), rms_step(j, c.bl.y, v.y), rms_step(j, c.bl.z, v.z),
                               rms_step(j, c.bl.w, v.w));
  if (j != kRmsBlock - 1) {
    st4(s.rms_blk, gi, b);
    return;
  }
  float4* r = reinterpret_cast<float4*>(s.rms + gi);
  const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
  const float4 a = (fi == kRmsBlock) ? z : r[0], a2 = (fi == kRmsBlock) ? z : r[1];
  const float2 t0 = kahan_acc(make_float2(a.x, a.y), b.x), t1 = kahan_acc(make_float2(a.z, a.w), b.y);
  const float2 t2 = kahan_acc(make_float2(a2.x, a2.y), b.z), t3 = kahan_acc(make_float2(a2.z, a2.w), b.w);
  r[0] = make_float4(t0.x, t0.y, t1.x, t1.y);
  r[1] = make_float4(t2.x, t2.y, t3.x, t3.y);
}
__device__ __forceinline__ void sensor_dense4_load(const Sensor& s, int fi, long long gi, Acc4& c) {
  if (fi <= 1 || s.mode != 1) return;  // fi 1: the accumulators start here; <= 0: nothing recorded yet
  if (s.vmax) c.mx = ld4(s.vmax, gi);
  if (s.rms) rms_load4(s, fi, gi, c);
}
// (the less common accumulators -- per-point min, full-grid max / min -- are
// loaded here, where they are updated)
__device__ __forceinline__ void sensor_dense4_store(const Sensor& s, int fi, long long gi, float4 v, const Acc4& c) {
  if (fi <= 0) return;
  if (s.mode == 1) {
    if (s.raw) st4(s.raw, raw_row(s, fi) * s.ns + gi, v);
    if (s.vmax) st4(s.vmax, gi, fi == 1 ? v : max4(c.mx, v));
    if (s.vmin) st4(s.vmin, gi, fi == 1 ? v : min4(ld4(s.vmin, gi), v));
    if (s.rms) rms_store4(s, fi, gi, v, c);
  }
  if (s.max_all) st4(s.max_all, gi, fi == 1 ? v : max4(ld4(s.max_all, gi), v));
  if (s.min_all) st4(s.min_all, gi, fi == 1 ? v : min4(ld4(s.min_all, gi), v));
}

// Both parts at once, each accumulator loaded where it is updated (fewer
// live registers; used where the loads need not run ahead of a store).
__device__ __forceinline__ void sensor_dense4(const Sensor& s, int fi, long long gi, float4 v) {
  if (fi <= 0) return;
  if (s.mode == 1) {
    if (s.raw) st4(s.raw, raw_row(s, fi) * s.ns + gi, v);
    if (s.vmax) st4(s.vmax, gi, fi == 1 ? v : max4(ld4(s.vmax, gi), v));
    if (s.vmin) st4(s.vmin, gi, fi == 1 ? v : min4(ld4(s.vmin, gi), v));
    if (s.rms) {
      Acc4 c;
      rms_load4(s, fi, gi, c);
      rms_store4(s, fi, gi, v, c);
    }
  }
  if (s.max_all) st4(s.max_all, gi, fi == 1 ? v : max4(ld4(s.max_all, gi), v));
  if (s.min_all) st4(s.min_all, gi, fi == 1 ? v : min4(ld4(s.min_all, gi), v));
}

// Sparse sensors (mode 2) of a row tile, values read from the packed buffer.
static __device__ void sensor_sparse_tile(const Sensor& s, int fi, const float2* buf, RowLayout lay, const Dims& d,
                                   long long r0, int L, int* sh) {
  if (s.mode != 2 || fi <= 0) return;
  const long long rend = min(r0 + 2LL * L, d.row1);
  tile_range(s.idx, s.ns, r0 * d.nx, rend * d.nx, sh);
  const int lo = sh[0], hi = sh[1];
  for (int j = lo + threadIdx.x; j < hi; j += blockDim.x) {
    const long long local = (long long)__ldg(s.idx + j) - r0 * d.nx;
    const int q = (int)(local / d.nx), x = (int)(local - (long long)q * d.nx);
    sensor_put(s, fi, __ldg(s.slot + j), get_comp(buf, lay, q, x));
  }
}

__device__ __forceinline__ float src_value(const SparseSource& s, const float* sig, int j, int t) {
  const int row = (s.nrows_sig == 1) ? 0 : __ldg(s.slot + j);
  const int off = s.delay ? __ldg(s.delay + j) : 0;
  const float v = __ldg(sig + (long long)(t - 1 + off) * s.nrows_sig + row);
  return s.weight ? __ldg(s.weight + j) * v : v;
}

template <int NC>
__device__ __forceinline__ int row_lines(int L) {
  return NC > 0 ? RTile<NC>::LINES : L;
}

// ---------------------------------------------------------------------------
// L2 prefetch of a row tile's inputs.  Issued when the tile starts, so DRAM
// streams everything the tile will read while the block is still in its
// first phase; the later loads then hit L2.  Bulk prefetches need 16-byte
// aligned addresses and sizes: real fields with nx % 4 == 0 and half-spectrum
// rows rounded up to an even number of bins (the pitch nxp is that even
// count, so the rounded row stays inside it).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void prefetch_l2(const void* p, unsigned bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

struct TilePrefetch {
  long long r0;
  int rows;  // rows of the tile inside [row0, row1)
  int nx;
  int nxp;
  int nxh2;  // half-spectrum bins per row, rounded up to even
  int slot;  // prefetch slots are dealt to the block's threads round robin

  __device__ TilePrefetch(const Dims& d, long long r, int L)
      : r0(r), rows((int)min(2LL * L, d.row1 - r)), nx(d.nx), nxp(d.nxp), nxh2((d.nxh + 1) & ~1), slot(0) {}
  __device__ bool mine() { return (int)threadIdx.x == (slot++ % (int)blockDim.x); }
  // a real field (x fastest): one contiguous range
  __device__ void field(const void* f, int elem_bytes = 4) {
    if (!f || rows <= 0) return;
    if (mine()) prefetch_l2(static_cast<const char*>(f) + r0 * nx * elem_bytes, (unsigned)rows * nx * elem_bytes);
  }
  // a half spectrum: one range per row, padding bins skipped
  __device__ void spectrum(const float2* S) {
    if (!S) return;
    for (int t = 0; t < rows; ++t)
      if (mine()) prefetch_l2(S + (r0 + t) * nxp, (unsigned)nxh2 * 8u);
  }
  __device__ void sensor(const Sensor& s, int fi) {
    if (s.mode != 1 || fi <= 1) return;
    field(s.vmax);
    field(s.vmin);
    if (s.rms) {
      const int j = rms_pos(fi);
      if (j != 0) field(s.rms_blk);
      if (j == kRmsBlock - 1 && fi != kRmsBlock) field(s.rms, 8);
    }
  }
};

// ---------------------------------------------------------------------------
// Bulk-copied spectrum rows.  A row tile's input half spectra are fetched by
// cp.async.bulk straight into the tile's own transform buffer, raw (tile row
// r at r * nxp), every field of the tile requested when the block starts, so
// the loads overlap one another and the first transform instead of
// stalling each phase.  The first inverse stage then builds each packed line
// (rows 2l and 2l + 1 as real and imaginary parts) from the raw rows as it
// reads them (RawRows), in place: all its inputs are read before the block
// barrier that precedes its stores.
// Needs: NC % 4 == 0 (an even pitch nxp = nx / 2 + 2, so rows are 16-byte
// multiples), 2 nxp <= the packed line stride (the raw rows fit the buffer),
// and buffers at 16-byte boundaries (an even lines x stride product).
// ---------------------------------------------------------------------------
template <int NC>
struct RowBulk {
  static constexpr int LS = NC + NC / 16 + 1;  // row_layout_stride(NC)
  static constexpr bool OK = NC > 0 && NC % 4 == 0 && 2 * (NC / 2 + 2) <= LS &&
                             (RTile<NC>::LINES * LS) % 2 == 0 && NC % 2 == 0;
};

__device__ __forceinline__ void bulk_load_1d(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// Issued by warp 0: `rows` spectrum rows from row r0 into raw, completion on bar.
__device__ __forceinline__ void bulk_rows(float2* raw, const float2* S, const Dims& d, long long r0, int rows,
                                          uint64_t* bar) {
  const unsigned bytes = (unsigned)d.nxp * 8u;
  const int lane = threadIdx.x & 31;
  if (lane == 0) mbar_expect_tx(bar, bytes * (unsigned)rows);
  __syncwarp();
  for (int r = lane; r < rows; r += 32) bulk_load_1d(raw + (long long)r * d.nxp, S + (r0 + r) * d.nxp, bytes, bar);
}

__device__ __forceinline__ int tile_rows(const Dims& d, long long r0, int L) {
  return (int)min(2LL * L, d.row1 - r0);
}

__device__ __forceinline__ uint64_t wait_limit(const WaitCtl& w) { return w.limit_ns ? w.limit_ns : kWaitNs; }

// Wait for one field's rows; false (for every thread) if any thread's wait ran out.
__device__ __forceinline__ bool rows_ready(uint64_t* bar, const WaitCtl& w) {
  const bool ok = mbar_wait(bar, 0, w.err, wait_limit(w));
  return !__syncthreads_or(!ok);
}

// After a failed wait: thread 0 waits (bounded) for the copies still in
// flight, so they land before the block's shared memory is released.
__device__ __forceinline__ void drain_rows(uint64_t* bars, int from, int to, const WaitCtl& w) {
  if (threadIdx.x == 0)
    for (int f = from; f < to; ++f) mbar_wait(&bars[f], 0, nullptr, wait_limit(w));
}

// Element n of packed line l, read from raw rows 2l and 2l + 1: the full
// spectrum of row 2l plus i times that of row 2l + 1, each from its half
// spectrum (Hermitian), with the imaginary parts of the k = 0 and Nyquist
// bins dropped, as load_c2r builds it.  `kmul` (optional) multiplies bin k.
template <int NC>
struct RawRows {
  const float2* raw;
  int nxp;
  int rows;
  const float2* kmul;
  __device__ __forceinline__ float2 operator()(int l, int n) const {
    const bool lo = 2 * n <= NC;
    const int k = lo ? n : NC - n;
    const int ra = 2 * l;
    float2 A = make_float2(0.f, 0.f), B = A;
    if (ra < rows) A = raw[ra * nxp + k];
    if (ra + 1 < rows) B = raw[(ra + 1) * nxp + k];
    if (kmul) {
      const float2 m = __ldg(kmul + k);
      A = c_mul(A, m);
      B = c_mul(B, m);
    }
    if (k == 0 || 2 * k == NC) {
      A.y = 0.f;
      B.y = 0.f;
    }
    return lo ? make_float2(A.x - B.y, A.y + B.x) : make_float2(A.x + B.y, B.x - A.y);
  }
};

// ---------------------------------------------------------------------------
// u update: C2R of the gradient, split-PML momentum update, velocity
// sources, velocity sensors, R2C of the new velocity.  blockIdx.y = axis.
// ---------------------------------------------------------------------------
// LEAN: the variant for steps with no velocity source and no velocity sensor
// after the first (no source, sensor or initial-pressure code: a smaller
// kernel body); otherwise every case.  At 256 points the lean variant is
// held to 64 registers a thread (8 blocks of 128 threads per SM) and the
// general one to 72 (7 blocks); other lengths keep the compiler's own
// choice (a minimum block count of 0 sets no bound), which caps would push
// into spills (96, 128, 160, 192 points).
template <int NC, bool LEAN>
__global__ void __launch_bounds__(RTile<NC>::THREADS, NC == 256 ? (LEAN ? 8 : 7) : 0)
    k_x_u(const __grid_constant__ UArgs a, Dims d,
                                                           const __grid_constant__ FFTPlan plan,
                                                           const float2* __restrict__ tw_g, int Lrt) {
  extern __shared__ __align__(16) float2 sm[];
  __shared__ int sh[2];
  constexpr bool CT = NC > 0;
  const int nx = CT ? NC : d.nx;
  const int L = row_lines<NC>(Lrt);
  const int ax = blockIdx.y;
  const RowLayout lay{row_layout_stride(nx)};
  float2* tw = sm;
  float2* B0 = sm + nx;
  float2* B1 = CT ? nullptr : B0 + L * lay.ls;
  const long long r0 = d.row0 + (long long)blockIdx.x * 2 * L;
  for (int i = threadIdx.x; i < nx; i += blockDim.x) tw[i] = tw_g[i];
  __shared__ uint64_t rbar[1];
  if constexpr (RowBulk<NC>::OK) {
    if (threadIdx.x == 0) {
      mbar_init(&rbar[0], 1);
      fence_mbar_init();
    }
  }
  pdl_wait();  // everything below reads or writes the predecessors' data
  pdl_trigger();
  if constexpr (RowBulk<NC>::OK) {  // the tile's spectrum rows are requested first
    __syncthreads();
    if (threadIdx.x < 32) bulk_rows(B0, a.S[ax], d, r0, tile_rows(d, r0, L), &rbar[0]);
  }
  const int t = *a.clk.t;
  const int fi = LEAN ? 0 : record_index(a.clk);
  const bool init = !LEAN && a.init;
  float2* G;
  if constexpr (RowBulk<NC>::OK) {
    {  // the epilogue's inputs stream in during the wait and the FFT
      TilePrefetch pf(d, r0, L);
      if (!init) pf.field(a.u[ax]);
      pf.field(a.rinv[ax].p);
      pf.sensor(a.sens[ax], fi);
    }
    if (!rows_ready(&rbar[0], a.wait)) {
      drain_rows(rbar, 0, 1, a.wait);
      return;
    }
    ct_fft_rows_ld<NC, true>(B0, tw, lay, RawRows<NC>{B0, d.nxp, tile_rows(d, r0, L), a.kmul[ax]});
    G = B0;
  } else {
    load_c2r<NC>(a.S[ax], B0, lay, d, r0, L, a.kmul[ax]);
    __syncthreads();
    if constexpr (NC > 0 && NC % 4 == 0) {  // the epilogue's inputs stream in during the FFT
      TilePrefetch pf(d, r0, L);
      if (!init) pf.field(a.u[ax]);
      pf.field(a.rinv[ax].p);
      pf.sensor(a.sens[ax], fi);
    }
    G = tile_fft<NC, true, false>(B0, B1, tw, plan, L, lay);
  }
  float2* W = (G == B0) ? B1 : B0;
  float* u = a.u[ax];
  const float* pml = a.pml_sg[ax];
  const Map rinv = a.rinv[ax];
  const DenseSource ds = a.dsrc[ax];
  const bool dense_on = !LEAN && ds.field && t <= ds.len;
  const float damp = dense_on ? (ds.sig ? __ldg(ds.sig + t - 1) : 1.f) : 0.f;
  const int total = 2 * L * nx;
  constexpr bool VEC = NC > 0 && NC % 4 == 0;
  if constexpr (VEC) {
    // 4 consecutive points per iteration, 16-byte global accesses
#pragma unroll (kRowLoopUnroll)
    for (int i = 4 * threadIdx.x; i < total; i += 4 * blockDim.x) {
      const int q = i / nx, x = i - q * nx;
      const long long row = r0 + q;
      if (row >= d.row1) {
#pragma unroll
        for (int j = 0; j < 4; ++j) set_comp(G, lay, q, x + j, 0.f);
        continue;
      }
      const long long gi = row * nx + x;
      float4 pm;
      if (ax == 0) {
        pm = __ldg(reinterpret_cast<const float4*>(pml + x));
      } else {
        const float v = __ldg(pml + (ax == 1 ? (int)(row % d.ny) : (int)(row / d.ny)));
        pm = make_float4(v, v, v, v);
      }
      const float4 rv = map4(rinv, gi);
      const float4 uo = init ? make_float4(0.f, 0.f, 0.f, 0.f) : ld4(u, gi);
      const float4 sv = dense_on ? __ldg(reinterpret_cast<const float4*>(ds.field + gi)) : make_float4(0.f, 0.f, 0.f, 0.f);
      const float pmv[4] = {pm.x, pm.y, pm.z, pm.w}, rvv[4] = {rv.x, rv.y, rv.z, rv.w};
      const float uov[4] = {uo.x, uo.y, uo.z, uo.w}, svv[4] = {sv.x, sv.y, sv.z, sv.w};
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const float g = get_comp(G, lay, q, x + j);
        float un;
        if (init)
          un = a.dt * rvv[j] * g / 2.f;
        else
          un = pmv[j] * (pmv[j] * uov[j] - a.dt * rvv[j] * g);
        if (dense_on) un = un + damp * svv[j];
        set_comp(G, lay, q, x + j, un);
      }
    }
  } else {
#pragma unroll 4
    for (int i = threadIdx.x; i < total; i += blockDim.x) {
      const int q = i / nx, x = i - q * nx;
      const long long row = r0 + q;
      if (row >= d.row1) {
        set_comp(G, lay, q, x, 0.f);
        continue;
      }
      const long long gi = row * nx + x;
      const float g = get_comp(G, lay, q, x);
      int coord = x;
      if (ax == 1) coord = (int)(row % d.ny);
      if (ax == 2) coord = (int)(row / d.ny);
      const float pm = __ldg(pml + coord);
      const float rv = rinv.at(gi);
      float un;
      if (init)
        un = a.dt * rv * g / 2.f;
      else
        un = pm * (pm * u[gi] - a.dt * rv * g);
      if (dense_on) un = un + damp * __ldg(ds.field + gi);
      set_comp(G, lay, q, x, un);
    }
  }
  __syncthreads();
  // sparse velocity sources (dirichlet / additive without correction; a
  // transducer is an additive x source with per-point delays and weights)
  const float* ssig = a.src_sig[ax];
  if (!LEAN && a.src.n > 0 && ssig && t <= a.src_len[ax] && !init) {
    const long long rend = min(r0 + 2LL * L, d.row1);
    tile_range(a.src.idx, a.src.n, r0 * nx, rend * nx, sh);
    const int lo = sh[0], hi = sh[1];
    for (int j = lo + threadIdx.x; j < hi; j += blockDim.x) {
      const long long local = (long long)__ldg(a.src.idx + j) - r0 * nx;
      const int q = (int)(local / nx), x = (int)(local - (long long)q * nx);
      const float v = src_value(a.src, ssig, j, t);
      const float cur = get_comp(G, lay, q, x);
      set_comp(G, lay, q, x, a.src.mode == 0 ? v : cur + v);
    }
    __syncthreads();
  }
  const Sensor& s = a.sens[ax];
  if constexpr (VEC) {
#pragma unroll (kRowLoopUnroll)
    for (int i = 4 * threadIdx.x; i < total; i += 4 * blockDim.x) {
      const int q = i / nx, x = i - q * nx;
      const long long row = r0 + q;
      if (row >= d.row1) continue;
      const long long gi = row * nx + x;
      const float4 v = make_float4(get_comp(G, lay, q, x), get_comp(G, lay, q, x + 1), get_comp(G, lay, q, x + 2),
                                   get_comp(G, lay, q, x + 3));
      st4(u, gi, v);
      if (!LEAN) sensor_dense4(s, fi, gi, v);
    }
  } else {
#pragma unroll 4
    for (int i = threadIdx.x; i < total; i += blockDim.x) {
      const int q = i / nx, x = i - q * nx;
      const long long row = r0 + q;
      if (row >= d.row1) continue;
      const long long gi = row * nx + x;
      const float v = get_comp(G, lay, q, x);
      u[gi] = v;
      sensor_dense(s, fi, gi, v);
    }
  }
  if (!LEAN) sensor_sparse_tile(s, fi, G, lay, d, r0, L, sh);
  if (a.do_r2c) {
    __syncthreads();
    float2* F = tile_fft<NC, false, false>(G, W, tw, plan, L, lay);
    store_r2c<NC>(F, a.Sout[ax], lay, d, r0, L);
  }
}

// ---------------------------------------------------------------------------
// rho update and equation of state.  C2R of du_i/dx_i for every axis, split
// mass conservation (linear / nonlinear), pressure sources, then either the
// lossless / Stokes EOS (p, sensors, R2C of p) or, for power-law absorption,
// the local part of p plus the R2C of rho0 * sum(du) and sum(rho).
// ---------------------------------------------------------------------------
// EOSK 1: the variant for power-law absorption without sparse pressure
// sources (no sensor, Stokes, lossless-EOS or source-pass code: a smaller
// kernel body); -1: every case, the equation of state read from a.eos.
template <int NC, int DIM, int EOSK>
__global__ void __launch_bounds__(RTile<NC>::THREADS, RTile<NC>::MIN_BLOCKS) k_x_rho(const __grid_constant__ RhoArgs a, Dims d,
                                                             const __grid_constant__ FFTPlan plan,
                                                             const float2* __restrict__ tw_g, int Lrt) {
  extern __shared__ __align__(16) float2 sm[];
  __shared__ int sh[2];
  constexpr bool CT = NC > 0;
  const int nx = CT ? NC : d.nx;
  const int L = row_lines<NC>(Lrt);
  constexpr int dim = DIM;
  const int eos = EOSK >= 0 ? EOSK : a.eos;
  const RowLayout lay{row_layout_stride(nx)};
  float2* tw = sm;
  float2* pool[4];
  for (int b = 0; b < 4; ++b) pool[b] = sm + nx + b * L * lay.ls;
  const long long r0 = d.row0 + (long long)blockIdx.x * 2 * L;
  for (int i = threadIdx.x; i < nx; i += blockDim.x) tw[i] = tw_g[i];
  // every divergence component's spectrum rows are requested first (not on
  // axisymmetric grids, whose u_r / r spectrum is summed in as S[1] is read)
  __shared__ uint64_t rbar[3];
  const bool bulk = RowBulk<NC>::OK && !a.S_rr;
  if constexpr (RowBulk<NC>::OK) {
    if (bulk && threadIdx.x == 0) {
      _Pragma("unroll") for (int f = 0; f < dim; ++f) mbar_init(&rbar[f], 1);
      fence_mbar_init();
    }
  }
  pdl_wait();  // everything below reads or writes the predecessors' data
  pdl_trigger();
  if constexpr (RowBulk<NC>::OK) {
    if (bulk) {
      __syncthreads();
      if (threadIdx.x < 32) {
        const int rows = tile_rows(d, r0, L);
        _Pragma("unroll") for (int f = 0; f < dim; ++f) bulk_rows(pool[f], a.S[f], d, r0, rows, &rbar[f]);
      }
    }
  }
  const int t = *a.clk.t;
  const int fi = record_index(a.clk);
  // inverse x transforms of the divergence components
  float2* D[3] = {nullptr, nullptr, nullptr};
  float2* Wk = nullptr;
  if constexpr (CT) {
#pragma unroll 1
    for (int f = 0; f < dim; ++f) {
      if (!bulk) {
        load_c2r<NC>(a.S[f], pool[f], lay, d, r0, L, nullptr, f == 1 ? a.S_rr : nullptr);
        __syncthreads();
      }
      if constexpr (NC % 4 == 0) {  // what the next phase reads streams in during this FFT
        TilePrefetch pf(d, r0, L);
        if (f + 1 < dim) {
          if (!bulk) pf.spectrum(a.S[f + 1]);
        } else {
          pf.field(a.rho[0]);
          // rho_y, rho_z only where the tile has rows in the y or z PML (rows
          // outside it read them at the x-PML ends only; a heuristic from
          // the first and last row: it decides prefetching, not results)
          const long long rl = r0 + tile_rows(d, r0, L) - 1;
          if (!a.box.row((int)(r0 % d.ny), (int)(r0 / d.ny), dim) || !a.box.row((int)(rl % d.ny), (int)(rl / d.ny), dim))
            _Pragma("unroll") for (int g = 1; g < dim; ++g) pf.field(a.rho[g]);
          pf.field(a.rho0.p);
          pf.field(a.c0sq.p);
          if (a.nonlinear) pf.field(a.bona.p);
          if (eos == 2) pf.field(a.tau.p);
          if (eos != 1) pf.sensor(a.sens, fi);
        }
      }
      if constexpr (RowBulk<NC>::OK) {
        if (bulk) {
          if (!rows_ready(&rbar[f], a.wait)) {
            drain_rows(rbar, f, dim, a.wait);
            return;
          }
          ct_fft_rows_ld<NC, true>(pool[f], tw, lay, RawRows<NC>{pool[f], d.nxp, tile_rows(d, r0, L), nullptr});
          continue;
        }
      }
      tile_fft<NC, true, false>(pool[f], nullptr, tw, plan, L, lay);
    }
    _Pragma("unroll") for (int f = 0; f < dim; ++f) D[f] = pool[f];
  } else {
    bool used[4] = {false, false, false, false};
    _Pragma("unroll") for (int f = 0; f < dim; ++f) {
      int ia = -1, ib = -1;
      _Pragma("unroll") for (int b = 0; b <= dim; ++b) {
        if (!used[b]) {
          if (ia < 0)
            ia = b;
          else if (ib < 0)
            ib = b;
        }
      }
      load_c2r<NC>(a.S[f], pool[ia], lay, d, r0, L, nullptr, f == 1 ? a.S_rr : nullptr);
      __syncthreads();
      D[f] = tile_fft<NC, true, false>(pool[ia], pool[ib], tw, plan, L, lay);
      used[(D[f] == pool[ia]) ? ia : ib] = true;
    }
    _Pragma("unroll") for (int b = 0; b <= dim; ++b)
      if (!used[b]) Wk = pool[b];
  }

  const bool sp = EOSK < 0 && (a.src.n > 0) && (t <= a.src.len);
  const bool dense_on = a.dsrc.field && t <= a.dsrc.len;
  const float damp = dense_on ? (a.dsrc.sig ? __ldg(a.dsrc.sig + t - 1) : 1.f) : 0.f;
  const int total = 2 * L * nx;
  const bool absorbing = (eos == 1);

  constexpr bool VEC = NC > 0 && NC % 4 == 0;
  if (VEC && !sp) {
    // 4 consecutive points per iteration, 16-byte global accesses
#pragma unroll (kRowLoopUnroll)
    for (int i = 4 * threadIdx.x; i < total; i += 4 * blockDim.x) {
      const int q = i / nx, x = i - q * nx;
      const long long row = r0 + q;
      if (row >= d.row1) {
#pragma unroll
        for (int j = 0; j < 4; ++j)
          _Pragma("unroll") for (int f = 0; f < dim; ++f) set_comp(D[f], lay, q, x + j, 0.f);
        continue;
      }
      const long long gi = row * nx + x;
      const int y = (int)(row % d.ny), z = (int)(row / d.ny);
      float4 ro[3], pm4[3];
      pm4[0] = __ldg(reinterpret_cast<const float4*>(a.pml[0] + x));
      {
        const float vy = __ldg(a.pml[1] + y);
        pm4[1] = make_float4(vy, vy, vy, vy);
        if (dim == 3) {
          const float vz = __ldg(a.pml[2] + z);
          pm4[2] = make_float4(vz, vz, vz, vz);
        }
      }
      const bool merged = a.box.at(x, y, z, dim);  // the density stored merged (RhoBox)
      if (merged) {
        ro[0] = ld4(a.rho[0], gi);
      } else {
        _Pragma("unroll") for (int f = 0; f < dim; ++f) ro[f] = ld4(a.rho[f], gi);
      }
      const float4 r0v4 = map4(a.rho0, gi);
      const float4 c24 = map4(a.c0sq, gi);
      const float4 bn4 = a.nonlinear ? map4(a.bona, gi) : make_float4(0.f, 0.f, 0.f, 0.f);
      const float4 ta4 = (eos == 2) ? map4(a.tau, gi) : make_float4(0.f, 0.f, 0.f, 0.f);
      const float4 ds4 = dense_on ? __ldg(reinterpret_cast<const float4*>(a.dsrc.field + gi))
                                  : make_float4(0.f, 0.f, 0.f, 0.f);
      Acc4 acc;  // the sensor accumulators (lossless / Stokes), loaded before any store
      if (!absorbing) sensor_dense4_load(a.sens, fi, gi, acc);
      float rn[3][4], outp[4], outq[4], outr[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        auto c = [&](const float4& v) { return j == 0 ? v.x : (j == 1 ? v.y : (j == 2 ? v.z : v.w)); };
        float du[3];
        _Pragma("unroll") for (int f = 0; f < dim; ++f) du[f] = get_comp(D[f], lay, q, x + j);
        float dsum = du[0] + du[1];
        if (dim == 3) dsum += du[2];
        const float r0v = c(r0v4);
        float rsum;
        if (merged) {
          // the split update summed over the axes, each PML factor 1
          const float rold = c(ro[0]);
          const float rpr = a.nonlinear ? 2.f * rold + r0v : r0v;
          rsum = rold - a.dt * rpr * dsum;
          if (dense_on) rsum = rsum + (float)dim * (damp * c(ds4));
          rn[0][j] = rsum;
        } else {
          float rold[3];
          _Pragma("unroll") for (int f = 0; f < dim; ++f) rold[f] = c(ro[f]);
          float rpr = r0v;
          if (a.nonlinear) {
            float rs = rold[0] + rold[1];
            if (dim == 3) rs += rold[2];
            rpr = 2.f * rs + r0v;
          }
          _Pragma("unroll") for (int f = 0; f < dim; ++f) {
            const float pm = c(pm4[f]);
            rn[f][j] = pm * (pm * rold[f] - a.dt * rpr * du[f]);
            if (dense_on) rn[f][j] = rn[f][j] + damp * c(ds4);
          }
          rsum = rn[0][j] + rn[1][j];
          if (dim == 3) rsum += rn[2][j];
        }
        float term = rsum;
        if (eos == 2) term = term + c(ta4) * r0v * dsum;
        if (a.nonlinear) term = term + c(bn4) * rsum * rsum / (2.f * r0v);
        outp[j] = c(c24) * term;
        outq[j] = r0v * dsum;
        outr[j] = rsum;
      }
      if (merged) {
        st4(a.rho[0], gi, make_float4(rn[0][0], rn[0][1], rn[0][2], rn[0][3]));
      } else {
        _Pragma("unroll") for (int f = 0; f < dim; ++f) st4(a.rho[f], gi, make_float4(rn[f][0], rn[f][1], rn[f][2], rn[f][3]));
      }
      const float4 pv4 = make_float4(outp[0], outp[1], outp[2], outp[3]);
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        if (absorbing) {
          set_comp(D[0], lay, q, x + j, outq[j]);
          set_comp(D[1], lay, q, x + j, outr[j]);
        } else {
          set_comp(D[0], lay, q, x + j, outp[j]);
        }
      }
      if (absorbing) {
        st4(a.p_loc, gi, pv4);
      } else {
        if (a.p_out) st4(a.p_out, gi, pv4);
        sensor_dense4_store(a.sens, fi, gi, pv4, acc);
      }
    }
  } else {
  // Phase A: rho update (stored to global before the EOS when sparse
  // sources must be applied first).
  float rnew[3];
  for (int pass = 0; pass < (sp ? 2 : 1); ++pass) {
    if (sp && pass == 1) {
      // apply sparse pressure sources to every rho component in global memory
      __syncthreads();
      const long long rend = min(r0 + 2LL * L, d.row1);
      tile_range(a.src.idx, a.src.n, r0 * nx, rend * nx, sh);
      const int lo = sh[0], hi = sh[1];
      for (int j = lo + threadIdx.x; j < hi; j += blockDim.x) {
        const long long gi = __ldg(a.src.idx + j);
        const float v = src_value(a.src, a.src.sig, j, t);
        const long long grow = gi / nx;
        if (a.box.at((int)(gi - grow * nx), (int)(grow % d.ny), (int)(grow / d.ny), dim)) {
          const float vt = (float)dim * v;  // every component set to / increased by v
          a.rho[0][gi] = (a.src.mode == 0) ? vt : a.rho[0][gi] + vt;
        } else {
          _Pragma("unroll") for (int f = 0; f < dim; ++f) a.rho[f][gi] = (a.src.mode == 0) ? v : a.rho[f][gi] + v;
        }
      }
      __syncthreads();
    }
#pragma unroll 2
    for (int i = threadIdx.x; i < total; i += blockDim.x) {
      const int q = i / nx, x = i - q * nx;
      const long long row = r0 + q;
      if (row >= d.row1) {
        _Pragma("unroll") for (int f = 0; f < dim; ++f) set_comp(D[f], lay, q, x, 0.f);
        continue;
      }
      const long long gi = row * nx + x;
      float du[3];
      _Pragma("unroll") for (int f = 0; f < dim; ++f) du[f] = get_comp(D[f], lay, q, x);
      float dsum = du[0] + du[1];
      if (dim == 3) dsum += du[2];
      const float r0v = a.rho0.at(gi);
      const int y = (int)(row % d.ny), z = (int)(row / d.ny);
      const bool merged = a.box.at(x, y, z, dim);
      float rsum;
      if (merged) {
        if (pass == 0) {  // the split update summed over the axes, each PML factor 1
          const float rold = a.rho[0][gi];
          const float rpr = a.nonlinear ? 2.f * rold + r0v : r0v;
          rsum = rold - a.dt * rpr * dsum;
          if (dense_on) rsum = rsum + (float)dim * (damp * __ldg(a.dsrc.field + gi));
          a.rho[0][gi] = rsum;
          if (sp) continue;
        } else {
          rsum = a.rho[0][gi];
        }
      } else {
        if (pass == 0) {
          float rold[3];
          _Pragma("unroll") for (int f = 0; f < dim; ++f) rold[f] = a.rho[f][gi];
          float rpr = r0v;
          if (a.nonlinear) {
            float rs = rold[0] + rold[1];
            if (dim == 3) rs += rold[2];
            rpr = 2.f * rs + r0v;
          }
          const int coord[3] = {x, y, z};
          _Pragma("unroll") for (int f = 0; f < dim; ++f) {
            const float pm = __ldg(a.pml[f] + coord[f]);
            rnew[f] = pm * (pm * rold[f] - a.dt * rpr * du[f]);
            if (dense_on) rnew[f] = rnew[f] + damp * __ldg(a.dsrc.field + gi);
            a.rho[f][gi] = rnew[f];
          }
          if (sp) continue;
        } else {
          _Pragma("unroll") for (int f = 0; f < dim; ++f) rnew[f] = a.rho[f][gi];
        }
        rsum = rnew[0] + rnew[1];
        if (dim == 3) rsum += rnew[2];
      }
      // equation of state (kspaceFirstOrder3D.m:963-1017)
      const float c2 = a.c0sq.at(gi);
      float term = rsum;
      if (eos == 2) term = term + a.tau.at(gi) * r0v * dsum;
      if (a.nonlinear) term = term + a.bona.at(gi) * rsum * rsum / (2.f * r0v);
      const float pv = c2 * term;
      if (absorbing) {
        a.p_loc[gi] = pv;
        set_comp(D[0], lay, q, x, r0v * dsum);
        set_comp(D[1], lay, q, x, rsum);
      } else {
        set_comp(D[0], lay, q, x, pv);
        if (a.p_out) a.p_out[gi] = pv;
        sensor_dense(a.sens, fi, gi, pv);
      }
    }
  }
  }
  __syncthreads();
  if (absorbing) {
    if constexpr (CT) {
#pragma unroll 1
      for (int f = 0; f < 2; ++f) {
        if (f) __syncthreads();
        tile_fft<NC, false, false>(D[f], nullptr, tw, plan, L, lay);
        store_r2c<NC>(D[f], f == 0 ? a.S_q : a.S_r, lay, d, r0, L);
      }
    } else {
      float2* F = tile_fft<NC, false, false>(D[0], Wk, tw, plan, L, lay);
      store_r2c<NC>(F, a.S_q, lay, d, r0, L);
      __syncthreads();
      float2* Wk2 = (F == D[0]) ? Wk : D[0];
      F = tile_fft<NC, false, false>(D[1], Wk2, tw, plan, L, lay);
      store_r2c<NC>(F, a.S_r, lay, d, r0, L);
    }
  } else {
    sensor_sparse_tile(a.sens, fi, D[0], lay, d, r0, L, sh);
    __syncthreads();
    float2* F = tile_fft<NC, false, false>(D[0], Wk, tw, plan, L, lay);
    store_r2c<NC>(F, a.S_p, lay, d, r0, L);
  }
}

// ---------------------------------------------------------------------------
// power-law absorbing EOS: p = p_loc + c0^2 tau A - c0^2 eta B, sensors, R2C.
// ---------------------------------------------------------------------------
template <int NC>
__global__ void __launch_bounds__(RTile<NC>::THREADS) k_x_eos(const __grid_constant__ EosArgs a, Dims d,
                                                             const __grid_constant__ FFTPlan plan,
                                                             const float2* __restrict__ tw_g, int Lrt) {
  extern __shared__ __align__(16) float2 sm[];
  __shared__ int sh[2];
  constexpr bool CT = NC > 0;
  const int nx = CT ? NC : d.nx;
  const int L = row_lines<NC>(Lrt);
  const RowLayout lay{row_layout_stride(nx)};
  float2* tw = sm;
  float2* P0 = sm + nx;
  float2* P1 = P0 + L * lay.ls;
  float2* P2 = CT ? nullptr : P1 + L * lay.ls;
  const long long r0 = d.row0 + (long long)blockIdx.x * 2 * L;
  for (int i = threadIdx.x; i < nx; i += blockDim.x) tw[i] = tw_g[i];
  __shared__ uint64_t rbar[2];
  if constexpr (RowBulk<NC>::OK) {
    if (threadIdx.x == 0) {
      mbar_init(&rbar[0], 1);
      mbar_init(&rbar[1], 1);
      fence_mbar_init();
    }
  }
  pdl_wait();  // everything below reads or writes the predecessors' data
  pdl_trigger();
  if constexpr (RowBulk<NC>::OK) {  // both spectra's rows are requested first
    __syncthreads();
    if (threadIdx.x < 32) {
      const int rows = tile_rows(d, r0, L);
      bulk_rows(P0, a.S_a, d, r0, rows, &rbar[0]);
      bulk_rows(P1, a.S_b, d, r0, rows, &rbar[1]);
    }
  }
  const int fi = record_index(a.clk);
  float2 *RA, *RB, *Wk;
  if constexpr (RowBulk<NC>::OK) {
    {  // the epilogue's inputs stream in during the waits and the FFTs
      TilePrefetch pf(d, r0, L);
      pf.field(a.p_loc);
      pf.field(a.c2tau.p);
      pf.field(a.c2eta.p);
      pf.sensor(a.sens, fi);
    }
#pragma unroll 1
    for (int f = 0; f < 2; ++f) {
      if (!rows_ready(&rbar[f], a.wait)) {
        drain_rows(rbar, f, 2, a.wait);
        return;
      }
      float2* P = f ? P1 : P0;
      ct_fft_rows_ld<NC, true>(P, tw, lay, RawRows<NC>{P, d.nxp, tile_rows(d, r0, L), nullptr});
    }
    RA = P0;
    RB = P1;
    Wk = nullptr;
  } else if constexpr (CT) {
    load_c2r<NC>(a.S_a, P0, lay, d, r0, L);
    load_c2r<NC>(a.S_b, P1, lay, d, r0, L);
    __syncthreads();
    if constexpr (NC % 4 == 0) {  // the epilogue's inputs stream in during the FFTs
      TilePrefetch pf(d, r0, L);
      pf.field(a.p_loc);
      pf.field(a.c2tau.p);
      pf.field(a.c2eta.p);
      pf.sensor(a.sens, fi);
    }
#pragma unroll 1
    for (int f = 0; f < 2; ++f) tile_fft<NC, true, false>(f ? P1 : P0, nullptr, tw, plan, L, lay);
    RA = P0;
    RB = P1;
    Wk = nullptr;
  } else {
    load_c2r<NC>(a.S_a, P0, lay, d, r0, L);
    __syncthreads();
    RA = tile_fft<NC, true, false>(P0, P1, tw, plan, L, lay);
    float2* f1 = (RA == P0) ? P1 : P0;
    load_c2r<NC>(a.S_b, f1, lay, d, r0, L);
    __syncthreads();
    RB = tile_fft<NC, true, false>(f1, P2, tw, plan, L, lay);
    Wk = (RB == f1) ? P2 : f1;
  }
  const int total = 2 * L * nx;
  if constexpr (NC > 0 && NC % 4 == 0) {
    // 4 points per iteration: every load (inputs and sensor accumulators)
    // is issued before any store
    struct In {
      float4 pl, ct, ce;
      Acc4 acc;
      long long gi;
      int q, x;
      bool ok;
    };
    auto load = [&](int i, In& v) {
      v.q = i / nx;
      v.x = i - v.q * nx;
      const long long row = r0 + v.q;
      v.ok = row < d.row1;
      if (!v.ok) return;
      v.gi = row * nx + v.x;
      v.pl = ld4(a.p_loc, v.gi);
      v.ct = map4(a.c2tau, v.gi);
      v.ce = map4(a.c2eta, v.gi);
      sensor_dense4_load(a.sens, fi, v.gi, v.acc);
    };
    auto update = [&](const In& v) {
      if (!v.ok) {
#pragma unroll
        for (int j = 0; j < 4; ++j) set_comp(RA, lay, v.q, v.x + j, 0.f);
        return;
      }
      const float plv[4] = {v.pl.x, v.pl.y, v.pl.z, v.pl.w}, ctv[4] = {v.ct.x, v.ct.y, v.ct.z, v.ct.w};
      const float cev[4] = {v.ce.x, v.ce.y, v.ce.z, v.ce.w};
      float pv[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        pv[j] = plv[j] + ctv[j] * get_comp(RA, lay, v.q, v.x + j) - cev[j] * get_comp(RB, lay, v.q, v.x + j);
        set_comp(RA, lay, v.q, v.x + j, pv[j]);
      }
      const float4 p4 = make_float4(pv[0], pv[1], pv[2], pv[3]);
      if (a.p_out) st4(a.p_out, v.gi, p4);
      sensor_dense4_store(a.sens, fi, v.gi, p4, v.acc);
    };
    // (issuing two iterations' loads together measured the same: 1.2622
    // against 1.2616 ms per 256^3 step, at 113 instead of 72 registers)
#pragma unroll 1
    for (int i = 4 * threadIdx.x; i < total; i += 4 * blockDim.x) {
      In v;
      load(i, v);
      update(v);
    }
  } else {
#pragma unroll 4
    for (int i = threadIdx.x; i < total; i += blockDim.x) {
      const int q = i / nx, x = i - q * nx;
      const long long row = r0 + q;
      if (row >= d.row1) {
        set_comp(RA, lay, q, x, 0.f);
        continue;
      }
      const long long gi = row * nx + x;
      const float A = get_comp(RA, lay, q, x);
      const float B = get_comp(RB, lay, q, x);
      const float pv = a.p_loc[gi] + a.c2tau.at(gi) * A - a.c2eta.at(gi) * B;
      set_comp(RA, lay, q, x, pv);
      if (a.p_out) a.p_out[gi] = pv;
      sensor_dense(a.sens, fi, gi, pv);
    }
  }
  __syncthreads();
  sensor_sparse_tile(a.sens, fi, RA, lay, d, r0, L, sh);
  __syncthreads();
  float2* F = tile_fft<NC, false, false>(RA, Wk, tw, plan, L, lay);
  store_r2c<NC>(F, a.S_p, lay, d, r0, L);
}

// ---------------------------------------------------------------------------
// plain x transforms (setup work, sources with k-space correction)
// ---------------------------------------------------------------------------
template <int NC>
__global__ void __launch_bounds__(RTile<NC>::THREADS) k_x_r2c(const float* __restrict__ f, float2* S, Dims d,
                                                             const __grid_constant__ FFTPlan plan,
                                                             const float2* __restrict__ tw_g, int Lrt) {
  extern __shared__ __align__(16) float2 sm[];
  constexpr bool CT = NC > 0;
  const int nx = CT ? NC : d.nx;
  const int L = row_lines<NC>(Lrt);
  const RowLayout lay{row_layout_stride(nx)};
  float2* tw = sm;
  float2* B0 = sm + nx;
  float2* B1 = CT ? nullptr : B0 + L * lay.ls;
  for (int i = threadIdx.x; i < nx; i += blockDim.x) tw[i] = tw_g[i];
  const long long r0 = d.row0 + (long long)blockIdx.x * 2 * L;
  const int total = 2 * L * nx;
  for (int i = threadIdx.x; i < total; i += blockDim.x) {
    const int q = i / nx, x = i - q * nx;
    const long long row = r0 + q;
    set_comp(B0, lay, q, x, row < d.row1 ? f[row * nx + x] : 0.f);
  }
  __syncthreads();
  float2* F = tile_fft<NC, false, false>(B0, B1, tw, plan, L, lay);
  store_r2c<NC>(F, S, lay, d, r0, L);
}

// out = v (accumulate == 0) or out += v
template <int NC>
__global__ void __launch_bounds__(RTile<NC>::THREADS) k_x_c2r(const float2* __restrict__ S, float* out,
                                                             int accumulate, Dims d,
                                                             const __grid_constant__ FFTPlan plan,
                                                             const float2* __restrict__ tw_g, int Lrt) {
  extern __shared__ __align__(16) float2 sm[];
  constexpr bool CT = NC > 0;
  const int nx = CT ? NC : d.nx;
  const int L = row_lines<NC>(Lrt);
  const RowLayout lay{row_layout_stride(nx)};
  float2* tw = sm;
  float2* B0 = sm + nx;
  float2* B1 = CT ? nullptr : B0 + L * lay.ls;
  for (int i = threadIdx.x; i < nx; i += blockDim.x) tw[i] = tw_g[i];
  const long long r0 = d.row0 + (long long)blockIdx.x * 2 * L;
  load_c2r<NC>(S, B0, lay, d, r0, L);
  __syncthreads();
  float2* G = tile_fft<NC, true, false>(B0, B1, tw, plan, L, lay);
  const int total = 2 * L * nx;
  for (int i = threadIdx.x; i < total; i += blockDim.x) {
    const int q = i / nx, x = i - q * nx;
    const long long row = r0 + q;
    if (row >= d.row1) continue;
    const long long gi = row * nx + x;
    const float v = get_comp(G, lay, q, x);
    out[gi] = accumulate ? out[gi] + v : v;
  }
}



// ---------------------------------------------------------------------------
// host-side launchers of one transform length NC (0: runtime plan).  Each
// compile-time length is instantiated in a translation unit of its own
// (generated at build time), so the lengths compile in parallel.
// ---------------------------------------------------------------------------
static inline size_t smem_col(int n, int tl, int nbuf) { return sizeof(float2) * ((size_t)n + (size_t)nbuf * tl * n); }
static inline size_t smem_row(int nx, int L, int nbuf) {
  return sizeof(float2) * ((size_t)nx + (size_t)nbuf * L * row_layout_stride(nx));
}

template <class K>
static inline void set_smem(K k, size_t sm) {
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
}

static inline unsigned row_tiles(const Dims& d, int L) { return (unsigned)((d.row1 - d.row0 + 2 * L - 1) / (2 * L)); }

template <int NC, bool INV>
static void col_fft_t(const ColArgs& a0, int nfields, long long nouter, const FFTPlan& plan, const float2* tw,
                      cudaStream_t st) {
  ColArgs a = a0;
  const int tl = NC > 0 ? Tile<NC>::LINES : a.tl;
  a.tl = tl;
  dim3 grid((a.ncols + tl - 1) / tl, (unsigned)nouter, nfields);
  const size_t sm = smem_col(plan.n, tl, NC > 0 ? 1 : 2);
  set_smem(k_col_fft<NC, INV>, sm);
  k_col_fft<NC, INV><<<grid, Tile<NC>::THREADS, sm, st>>>(a, plan, tw);
}

template <int NC>
static void fused_t(const FusedArgs& a0, int ninputs, long long nouter, const FFTPlan& plan, const float2* tw,
                    const SpecTables& T, int dim, cudaStream_t st) {
  FusedArgs a = a0;
  const int tl = NC > 0 ? Tile<NC>::LINES : a.tl;
  a.tl = tl;
  dim3 grid((a.ncols + tl - 1) / tl, (unsigned)nouter, ninputs);
  const size_t sm = smem_col(plan.n, tl, NC > 0 ? 2 : 3);
  set_smem(k_fused_last<NC>, sm);
  k_fused_last<NC><<<grid, Tile<NC>::THREADS, sm, st>>>(a, plan, tw, T, dim);
}

template <int NC>
static void x_u_t(const UArgs& a, const Dims& d, const FFTPlan& plan, const float2* tw, int Lrt, cudaStream_t st) {
  const int L = NC > 0 ? RTile<NC>::LINES : Lrt;
  const size_t sm = smem_row(d.nx, L, NC > 0 ? 1 : 2);
  bool lean = !a.init && a.src.n == 0;
  for (int ax = 0; ax < d.dim; ++ax) lean = lean && !a.dsrc[ax].field && a.sens[ax].mode == 0;
  auto go = [&](auto k) {
    set_smem(k, sm);
    launch_pdl(k, dim3(row_tiles(d, L), d.dim), dim3(RTile<NC>::THREADS), sm, st, a, d, plan, tw, L);
  };
  lean ? go(k_x_u<NC, true>) : go(k_x_u<NC, false>);
}

template <int NC>
static void x_rho_t(const RhoArgs& a, const Dims& d, const FFTPlan& plan, const float2* tw, int Lrt,
                    cudaStream_t st) {
  const int L = NC > 0 ? RTile<NC>::LINES : Lrt;
  const size_t sm = smem_row(d.nx, L, NC > 0 ? d.dim : d.dim + 1);
  auto go = [&](auto k) {
    set_smem(k, sm);
    launch_pdl(k, dim3(row_tiles(d, L)), dim3(RTile<NC>::THREADS), sm, st, a, d, plan, tw, L);
  };
  const bool lean = a.eos == 1 && a.src.n == 0;
  if (d.dim == 3)
    lean ? go(k_x_rho<NC, 3, 1>) : go(k_x_rho<NC, 3, -1>);
  else
    lean ? go(k_x_rho<NC, 2, 1>) : go(k_x_rho<NC, 2, -1>);
}

template <int NC>
static void x_eos_t(const EosArgs& a, const Dims& d, const FFTPlan& plan, const float2* tw, int Lrt,
                    cudaStream_t st) {
  const int L = NC > 0 ? RTile<NC>::LINES : Lrt;
  const size_t sm = smem_row(d.nx, L, NC > 0 ? 2 : 3);
  set_smem(k_x_eos<NC>, sm);
  launch_pdl(k_x_eos<NC>, dim3(row_tiles(d, L)), dim3(RTile<NC>::THREADS), sm, st, a, d, plan, tw, L);
}

template <int NC>
static void x_r2c_t(const float* f, float2* S, const Dims& d, const FFTPlan& plan, const float2* tw, int Lrt,
                    cudaStream_t st) {
  const int L = NC > 0 ? RTile<NC>::LINES : Lrt;
  const size_t sm = smem_row(d.nx, L, NC > 0 ? 1 : 2);
  set_smem(k_x_r2c<NC>, sm);
  k_x_r2c<NC><<<row_tiles(d, L), RTile<NC>::THREADS, sm, st>>>(f, S, d, plan, tw, L);
}

template <int NC>
static void x_c2r_t(const float2* S, float* out, int acc, const Dims& d, const FFTPlan& plan, const float2* tw,
                    int Lrt, cudaStream_t st) {
  const int L = NC > 0 ? RTile<NC>::LINES : Lrt;
  const size_t sm = smem_row(d.nx, L, NC > 0 ? 1 : 2);
  set_smem(k_x_c2r<NC>, sm);
  k_x_c2r<NC><<<row_tiles(d, L), RTile<NC>::THREADS, sm, st>>>(S, out, acc, d, plan, tw, L);
}

// The launchers of one length.  Member functions are defined out of class
// (so not inline), which lets `extern template` in kernels.cu keep every
// length out of that translation unit.
template <int NC>
struct CtKernels {
  static void col_fft(bool inv, const ColArgs& a, int nfields, long long nouter, const FFTPlan& plan,
                      const float2* tw, cudaStream_t st);
  static void fused(const FusedArgs& a, int ninputs, long long nouter, const FFTPlan& plan, const float2* tw,
                    const SpecTables& T, int dim, cudaStream_t st);
  static void x_u(const UArgs& a, const Dims& d, const FFTPlan& plan, const float2* tw, int L, cudaStream_t st);
  static void x_rho(const RhoArgs& a, const Dims& d, const FFTPlan& plan, const float2* tw, int L,
                    cudaStream_t st);
  static void x_eos(const EosArgs& a, const Dims& d, const FFTPlan& plan, const float2* tw, int L,
                    cudaStream_t st);
  static void x_r2c(const float* f, float2* S, const Dims& d, const FFTPlan& plan, const float2* tw, int L,
                    cudaStream_t st);
  static void x_c2r(const float2* S, float* out, int acc, const Dims& d, const FFTPlan& plan, const float2* tw,
                    int L, cudaStream_t st);
};

template <int NC>
void CtKernels<NC>::col_fft(bool inv, const ColArgs& a, int nfields, long long nouter, const FFTPlan& plan,
                            const float2* tw, cudaStream_t st) {
  if (inv)
    col_fft_t<NC, true>(a, nfields, nouter, plan, tw, st);
  else
    col_fft_t<NC, false>(a, nfields, nouter, plan, tw, st);
}
template <int NC>
void CtKernels<NC>::fused(const FusedArgs& a, int ninputs, long long nouter, const FFTPlan& plan,
                          const float2* tw, const SpecTables& T, int dim, cudaStream_t st) {
  fused_t<NC>(a, ninputs, nouter, plan, tw, T, dim, st);
}
template <int NC>
void CtKernels<NC>::x_u(const UArgs& a, const Dims& d, const FFTPlan& plan, const float2* tw, int L,
                        cudaStream_t st) {
  x_u_t<NC>(a, d, plan, tw, L, st);
}
template <int NC>
void CtKernels<NC>::x_rho(const RhoArgs& a, const Dims& d, const FFTPlan& plan, const float2* tw, int L,
                          cudaStream_t st) {
  x_rho_t<NC>(a, d, plan, tw, L, st);
}
template <int NC>
void CtKernels<NC>::x_eos(const EosArgs& a, const Dims& d, const FFTPlan& plan, const float2* tw, int L,
                          cudaStream_t st) {
  x_eos_t<NC>(a, d, plan, tw, L, st);
}
template <int NC>
void CtKernels<NC>::x_r2c(const float* f, float2* S, const Dims& d, const FFTPlan& plan, const float2* tw,
                          int L, cudaStream_t st) {
  x_r2c_t<NC>(f, S, d, plan, tw, L, st);
}
template <int NC>
void CtKernels<NC>::x_c2r(const float2* S, float* out, int acc, const Dims& d, const FFTPlan& plan,
                          const float2* tw, int L, cudaStream_t st) {
  x_c2r_t<NC>(S, out, acc, d, plan, tw, L, st);
}

}  // namespace kwb

