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
#include "kernels.cuh"

namespace kwb {

// ---------------------------------------------------------------------------
// spectral operators generated per point from 1D tables
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 eval_op(const SpecOp& op, const SpecTables& T, int dim, int ix,
                                          int iy, int iz) {
  float k2 = __ldg(T.k2[0] + ix) + __ldg(T.k2[1] + iy);
  if (dim == 3) k2 += __ldg(T.k2[2] + iz);
  const float k = sqrtf(k2);
  switch (op.kind) {
    case OP_GRAD_POS:
    case OP_GRAD_NEG: {
      // kappa = sinc(c_ref k dt / 2), sinc(x) = sin(x) / x (k-Wave/private/sinc.m:38-39)
      const float x = T.cdt2 * k;
      const float kap = (x == 0.f) ? 1.f : sinf(x) / x;
      const int id = op.axis == 0 ? ix : (op.axis == 1 ? iy : iz);
      const float2* tab = (op.kind == OP_GRAD_POS) ? T.ddk_pos[op.axis] : T.ddk_neg[op.axis];
      const float2 d = tab[id];
      const float s = kap * T.scale;
      return make_float2(d.x * s, d.y * s);
    }
    case OP_NABLA1:
    case OP_NABLA2: {
      // k.^(y-2) / k.^(y-1) with the infinite value at k = 0 set to zero
      // (kspaceFirstOrder_createAbsorptionVariables.m:37-39, 49-51)
      const float e = (op.kind == OP_NABLA1) ? T.ym2 : T.ym1;
      float v;
      if (k == 0.f)
        v = (e == 0.f) ? 1.f : 0.f;
      else
        v = powf(k, e);
      return make_float2(v * T.scale, 0.f);
    }
    case OP_SRC_KAPPA: {
      const float x = T.cdt2 * k;
      return make_float2(cosf(x) * T.scale, 0.f);
    }
    default:
      return make_float2(T.scale, 0.f);
  }
}

// ---------------------------------------------------------------------------
// column passes
// ---------------------------------------------------------------------------
template <bool INV>
__global__ void __launch_bounds__(kThreads) k_col_fft(ColArgs a, FFTPlan plan,
                                                      const float2* __restrict__ tw_g) {
  extern __shared__ float2 sm[];
  const int n = plan.n, tl = a.tl;
  float2* tw = sm;
  float2* b0 = sm + n;
  float2* b1 = b0 + tl * n;
  for (int i = threadIdx.x; i < n; i += blockDim.x) tw[i] = tw_g[i];
  float2* g = a.buf[blockIdx.z] + (long long)blockIdx.y * a.ostride;
  const int c0 = blockIdx.x * tl;
  const int total = tl * n;
  for (int i = threadIdx.x; i < total; i += blockDim.x) {
    const int l = i % tl, p = i / tl, c = c0 + l;
    b0[i] = (c < a.ncols) ? g[p * a.lstride + c] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  float2* r = fft_lines<INV, true>(b0, b1, tw, plan, tl, ColLayout{tl});
  for (int i = threadIdx.x; i < total; i += blockDim.x) {
    const int l = i % tl, p = i / tl, c = c0 + l;
    if (c < a.ncols) g[p * a.lstride + c] = r[i];
  }
}

// Last axis: forward transform, multiply by `fanout` operators, inverse
// transform each product.
__global__ void __launch_bounds__(kThreads) k_fused_last(FusedArgs a, FFTPlan plan,
                                                         const float2* __restrict__ tw_g,
                                                         SpecTables T, int dim) {
  extern __shared__ float2 sm[];
  const int n = plan.n, tl = a.tl;
  float2* tw = sm;
  float2* A = sm + n;
  float2* B = A + tl * n;
  float2* C = B + tl * n;
  for (int i = threadIdx.x; i < n; i += blockDim.x) tw[i] = tw_g[i];
  const int g = blockIdx.z;
  const int outer = blockIdx.y;
  const long long off = (long long)outer * a.ostride;
  const float2* src = a.in[g] + off;
  const int c0 = blockIdx.x * tl;
  const int total = tl * n;
  for (int i = threadIdx.x; i < total; i += blockDim.x) {
    const int l = i % tl, p = i / tl, c = c0 + l;
    A[i] = (c < a.ncols) ? src[p * a.lstride + c] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  const ColLayout lay{tl};
  float2* F = fft_lines<false, true>(A, B, tw, plan, tl, lay);
  float2* W1 = (F == A) ? B : A;
  float2* W2 = C;
  for (int o = 0; o < a.fanout; ++o) {
    const SpecOp op = a.op[g * a.fanout + o];
    for (int i = threadIdx.x; i < total; i += blockDim.x) {
      const int l = i % tl, p = i / tl;
      int c = c0 + l;
      if (c >= a.ncols) c = 0;
      const int ix = c;
      const int iy = (dim == 3) ? outer : p;
      const int iz = (dim == 3) ? p : 0;
      W1[i] = c_mul(F[i], eval_op(op, T, dim, ix, iy, iz));
    }
    __syncthreads();
    float2* R = fft_lines<true, true>(W1, W2, tw, plan, tl, lay);
    float2* dst = a.out[g * a.fanout + o] + off;
    for (int i = threadIdx.x; i < total; i += blockDim.x) {
      const int l = i % tl, p = i / tl, c = c0 + l;
      if (c < a.ncols) dst[p * a.lstride + c] = R[i];
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
__device__ void load_c2r(const float2* __restrict__ S, float2* buf, RowLayout lay, const Dims& d,
                         long long r0, int L) {
  const int n = d.nx;
  const int total = L * n;
  for (int i = threadIdx.x; i < total; i += blockDim.x) {
    const int l = i / n, k = i - l * n;
    const long long ra = r0 + 2 * l, rb = ra + 1;
    const int kk = (2 * k <= n) ? k : n - k;
    float2 A = make_float2(0.f, 0.f), B = make_float2(0.f, 0.f);
    if (ra < d.nrows) A = S[ra * d.nxp + kk];
    if (rb < d.nrows) B = S[rb * d.nxp + kk];
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
__device__ void store_r2c(const float2* buf, float2* __restrict__ S, RowLayout lay, const Dims& d,
                          long long r0, int L) {
  const int n = d.nx, nh = d.nxh;
  const int total = L * nh;
  for (int i = threadIdx.x; i < total; i += blockDim.x) {
    const int l = i / nh, k = i - l * nh;
    const long long ra = r0 + 2 * l, rb = ra + 1;
    const float2 zk = buf[lay(l, k)];
    const float2 zn = buf[lay(l, k == 0 ? 0 : n - k)];
    const float2 A = make_float2(0.5f * (zk.x + zn.x), 0.5f * (zk.y - zn.y));
    const float2 B = make_float2(0.5f * (zk.y + zn.y), -0.5f * (zk.x - zn.x));
    if (ra < d.nrows) S[ra * d.nxp + k] = A;
    if (rb < d.nrows) S[rb * d.nxp + k] = B;
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

__device__ __forceinline__ void sensor_put(const Sensor& s, int fi, long long slot, float v) {
  if (s.raw) s.raw[(long long)(fi - 1) * s.ns + slot] = v;
  if (s.vmax) s.vmax[slot] = (fi == 1) ? v : fmaxf(s.vmax[slot], v);
  if (s.vmin) s.vmin[slot] = (fi == 1) ? v : fminf(s.vmin[slot], v);
  if (s.rms) {
    // compensated (Kahan) running sum of squares
    float2 acc = (fi == 1) ? make_float2(0.f, 0.f) : s.rms[slot];
    const float y = v * v - acc.y;
    const float t = acc.x + y;
    acc.y = (t - acc.x) - y;
    acc.x = t;
    s.rms[slot] = acc;
  }
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

// Sparse sensors (mode 2) of a row tile, values read from the packed buffer.
__device__ void sensor_sparse_tile(const Sensor& s, int fi, const float2* buf, RowLayout lay,
                                   const Dims& d, long long r0, int L, int* sh) {
  if (s.mode != 2 || fi <= 0) return;
  const long long rend = min(r0 + 2LL * L, d.nrows);
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
  return __ldg(sig + (long long)(t - 1) * s.nrows_sig + row);
}

// ---------------------------------------------------------------------------
// u update: C2R of the gradient, split-PML momentum update, velocity
// sources, velocity sensors, R2C of the new velocity.  blockIdx.y = axis.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) k_x_u(UArgs a, Dims d, FFTPlan plan,
                                                  const float2* __restrict__ tw_g, int L) {
  extern __shared__ float2 sm[];
  __shared__ int sh[2];
  const int nx = d.nx;
  const int ax = blockIdx.y;
  const RowLayout lay{row_layout_stride(nx)};
  float2* tw = sm;
  float2* B0 = sm + nx;
  float2* B1 = B0 + L * lay.ls;
  for (int i = threadIdx.x; i < nx; i += blockDim.x) tw[i] = tw_g[i];
  const long long r0 = (long long)blockIdx.x * 2 * L;
  const int t = *a.clk.t;
  const int fi = record_index(a.clk);
  load_c2r(a.S[ax], B0, lay, d, r0, L);
  __syncthreads();
  float2* G = fft_lines<true, false>(B0, B1, tw, plan, L, lay);
  float2* W = (G == B0) ? B1 : B0;
  float* u = a.u[ax];
  const float* pml = a.pml_sg[ax];
  const Map rinv = a.rinv[ax];
  const DenseSource ds = a.dsrc[ax];
  const bool dense_on = ds.field && t <= ds.len;
  const float damp = dense_on ? (ds.sig ? __ldg(ds.sig + t - 1) : 1.f) : 0.f;
  const int total = 2 * L * nx;
  for (int i = threadIdx.x; i < total; i += blockDim.x) {
    const int q = i / nx, x = i - q * nx;
    const long long row = r0 + q;
    if (row >= d.nrows) {
      set_comp(G, lay, q, x, 0.f);
      continue;
    }
    const long long gi = row * nx + x;
    const float g = get_comp(G, lay, q, x);
    const int y = (int)(row % d.ny), z = (int)(row / d.ny);
    const int coord = (ax == 0) ? x : ((ax == 1) ? y : z);
    const float pm = __ldg(pml + coord);
    const float rv = rinv.at(gi);
    float un;
    if (a.init)
      un = a.dt * rv * g / 2.f;
    else
      un = pm * (pm * u[gi] - a.dt * rv * g);
    if (dense_on) un = un + damp * __ldg(ds.field + gi);
    set_comp(G, lay, q, x, un);
  }
  __syncthreads();
  // sparse velocity sources (dirichlet / additive without correction)
  const float* ssig = a.src_sig[ax];
  if (a.src.n > 0 && ssig && t <= a.src_len[ax] && !a.init) {
    const long long rend = min(r0 + 2LL * L, d.nrows);
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
  for (int i = threadIdx.x; i < total; i += blockDim.x) {
    const int q = i / nx, x = i - q * nx;
    const long long row = r0 + q;
    if (row >= d.nrows) continue;
    const long long gi = row * nx + x;
    const float v = get_comp(G, lay, q, x);
    u[gi] = v;
    sensor_dense(s, fi, gi, v);
  }
  sensor_sparse_tile(s, fi, G, lay, d, r0, L, sh);
  if (a.do_r2c) {
    __syncthreads();
    float2* F = fft_lines<false, false>(G, W, tw, plan, L, lay);
    store_r2c(F, a.Sout[ax], lay, d, r0, L);
  }
}

// ---------------------------------------------------------------------------
// rho update and equation of state.  C2R of du_i/dx_i for every axis, split
// mass conservation (linear / nonlinear), pressure sources, then either the
// lossless / Stokes EOS (p, sensors, R2C of p) or, for power-law absorption,
// the local part of p plus the R2C of rho0 * sum(du) and sum(rho).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) k_x_rho(RhoArgs a, Dims d, FFTPlan plan,
                                                    const float2* __restrict__ tw_g, int L) {
  extern __shared__ float2 sm[];
  __shared__ int sh[2];
  const int nx = d.nx, dim = d.dim;
  const RowLayout lay{row_layout_stride(nx)};
  float2* tw = sm;
  float2* pool[4];
  for (int b = 0; b <= dim; ++b) pool[b] = sm + nx + b * L * lay.ls;
  for (int i = threadIdx.x; i < nx; i += blockDim.x) tw[i] = tw_g[i];
  const long long r0 = (long long)blockIdx.x * 2 * L;
  const int t = *a.clk.t;
  const int fi = record_index(a.clk);
  // inverse x transforms of the three divergence components
  float2* D[3] = {nullptr, nullptr, nullptr};
  bool used[4] = {false, false, false, false};
  for (int f = 0; f < dim; ++f) {
    int ia = -1, ib = -1;
    for (int b = 0; b <= dim; ++b) {
      if (!used[b]) {
        if (ia < 0)
          ia = b;
        else if (ib < 0)
          ib = b;
      }
    }
    load_c2r(a.S[f], pool[ia], lay, d, r0, L);
    __syncthreads();
    D[f] = fft_lines<true, false>(pool[ia], pool[ib], tw, plan, L, lay);
    used[(D[f] == pool[ia]) ? ia : ib] = true;
  }
  float2* Wk = nullptr;
  for (int b = 0; b <= dim; ++b)
    if (!used[b]) Wk = pool[b];

  const bool sp = (a.src.n > 0) && (t <= a.src.len);
  const bool dense_on = a.dsrc.field && t <= a.dsrc.len;
  const float damp = dense_on ? (a.dsrc.sig ? __ldg(a.dsrc.sig + t - 1) : 1.f) : 0.f;
  const int total = 2 * L * nx;
  const bool absorbing = (a.eos == 1);

  // Phase A: rho update (stored to global when sparse sources must be
  // applied before the equation of state).
  float rnew[3];
  for (int pass = 0; pass < (sp ? 2 : 1); ++pass) {
    if (sp && pass == 1) {
      // apply sparse pressure sources to every rho component in global memory
      __syncthreads();
      const long long rend = min(r0 + 2LL * L, d.nrows);
      tile_range(a.src.idx, a.src.n, r0 * nx, rend * nx, sh);
      const int lo = sh[0], hi = sh[1];
      for (int j = lo + threadIdx.x; j < hi; j += blockDim.x) {
        const long long gi = __ldg(a.src.idx + j);
        const float v = src_value(a.src, a.src.sig, j, t);
        for (int f = 0; f < dim; ++f) a.rho[f][gi] = (a.src.mode == 0) ? v : a.rho[f][gi] + v;
      }
      __syncthreads();
    }
    for (int i = threadIdx.x; i < total; i += blockDim.x) {
      const int q = i / nx, x = i - q * nx;
      const long long row = r0 + q;
      if (row >= d.nrows) {
        for (int f = 0; f < dim; ++f) set_comp(D[f], lay, q, x, 0.f);
        continue;
      }
      const long long gi = row * nx + x;
      const int y = (int)(row % d.ny), z = (int)(row / d.ny);
      float du[3];
      for (int f = 0; f < dim; ++f) du[f] = get_comp(D[f], lay, q, x);
      const float r0v = a.rho0.at(gi);
      if (pass == 0) {
        float rold[3];
        for (int f = 0; f < dim; ++f) rold[f] = a.rho[f][gi];
        float rpr = r0v;
        if (a.nonlinear) {
          float rs = rold[0] + rold[1];
          if (dim == 3) rs += rold[2];
          rpr = 2.f * rs + r0v;
        }
        const int coord[3] = {x, y, z};
        for (int f = 0; f < dim; ++f) {
          const float pm = __ldg(a.pml[f] + coord[f]);
          rnew[f] = pm * (pm * rold[f] - a.dt * rpr * du[f]);
          if (dense_on) rnew[f] = rnew[f] + damp * __ldg(a.dsrc.field + gi);
        }
        if (sp) {
          for (int f = 0; f < dim; ++f) a.rho[f][gi] = rnew[f];
          continue;
        }
        for (int f = 0; f < dim; ++f) a.rho[f][gi] = rnew[f];
      } else {
        for (int f = 0; f < dim; ++f) rnew[f] = a.rho[f][gi];
      }
      // equation of state (kspaceFirstOrder3D.m:963-1017)
      float rsum = rnew[0] + rnew[1];
      if (dim == 3) rsum += rnew[2];
      float dsum = du[0] + du[1];
      if (dim == 3) dsum += du[2];
      const float c2 = a.c0sq.at(gi);
      float term = rsum;
      if (a.eos == 2) term = term + a.tau.at(gi) * r0v * dsum;
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
  __syncthreads();
  if (absorbing) {
    float2* F = fft_lines<false, false>(D[0], Wk, tw, plan, L, lay);
    store_r2c(F, a.S_q, lay, d, r0, L);
    __syncthreads();
    float2* Wk2 = (F == D[0]) ? Wk : D[0];
    F = fft_lines<false, false>(D[1], Wk2, tw, plan, L, lay);
    store_r2c(F, a.S_r, lay, d, r0, L);
  } else {
    sensor_sparse_tile(a.sens, fi, D[0], lay, d, r0, L, sh);
    __syncthreads();
    float2* F = fft_lines<false, false>(D[0], Wk, tw, plan, L, lay);
    store_r2c(F, a.S_p, lay, d, r0, L);
  }
}

// ---------------------------------------------------------------------------
// power-law absorbing EOS: p = p_loc + c0^2 tau A - c0^2 eta B, sensors, R2C.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) k_x_eos(EosArgs a, Dims d, FFTPlan plan,
                                                    const float2* __restrict__ tw_g, int L) {
  extern __shared__ float2 sm[];
  __shared__ int sh[2];
  const int nx = d.nx;
  const RowLayout lay{row_layout_stride(nx)};
  float2* tw = sm;
  float2* P0 = sm + nx;
  float2* P1 = P0 + L * lay.ls;
  float2* P2 = P1 + L * lay.ls;
  for (int i = threadIdx.x; i < nx; i += blockDim.x) tw[i] = tw_g[i];
  const long long r0 = (long long)blockIdx.x * 2 * L;
  const int fi = record_index(a.clk);
  load_c2r(a.S_a, P0, lay, d, r0, L);
  __syncthreads();
  float2* RA = fft_lines<true, false>(P0, P1, tw, plan, L, lay);
  float2* f1 = (RA == P0) ? P1 : P0;
  load_c2r(a.S_b, f1, lay, d, r0, L);
  __syncthreads();
  float2* RB = fft_lines<true, false>(f1, P2, tw, plan, L, lay);
  float2* Wk = (RB == f1) ? P2 : f1;
  const int total = 2 * L * nx;
  for (int i = threadIdx.x; i < total; i += blockDim.x) {
    const int q = i / nx, x = i - q * nx;
    const long long row = r0 + q;
    if (row >= d.nrows) {
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
  __syncthreads();
  sensor_sparse_tile(a.sens, fi, RA, lay, d, r0, L, sh);
  __syncthreads();
  float2* F = fft_lines<false, false>(RA, Wk, tw, plan, L, lay);
  store_r2c(F, a.S_p, lay, d, r0, L);
}

// ---------------------------------------------------------------------------
// plain x transforms (setup work, sources with k-space correction)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) k_x_r2c(const float* __restrict__ f, float2* S, Dims d,
                                                    FFTPlan plan, const float2* __restrict__ tw_g,
                                                    int L) {
  extern __shared__ float2 sm[];
  const int nx = d.nx;
  const RowLayout lay{row_layout_stride(nx)};
  float2* tw = sm;
  float2* B0 = sm + nx;
  float2* B1 = B0 + L * lay.ls;
  for (int i = threadIdx.x; i < nx; i += blockDim.x) tw[i] = tw_g[i];
  const long long r0 = (long long)blockIdx.x * 2 * L;
  const int total = 2 * L * nx;
  for (int i = threadIdx.x; i < total; i += blockDim.x) {
    const int q = i / nx, x = i - q * nx;
    const long long row = r0 + q;
    set_comp(B0, lay, q, x, row < d.nrows ? f[row * nx + x] : 0.f);
  }
  __syncthreads();
  float2* F = fft_lines<false, false>(B0, B1, tw, plan, L, lay);
  store_r2c(F, S, lay, d, r0, L);
}

// out = v (accumulate == 0) or out += v
__global__ void __launch_bounds__(kThreads) k_x_c2r(const float2* __restrict__ S, float* out,
                                                    int accumulate, Dims d, FFTPlan plan,
                                                    const float2* __restrict__ tw_g, int L) {
  extern __shared__ float2 sm[];
  const int nx = d.nx;
  const RowLayout lay{row_layout_stride(nx)};
  float2* tw = sm;
  float2* B0 = sm + nx;
  float2* B1 = B0 + L * lay.ls;
  for (int i = threadIdx.x; i < nx; i += blockDim.x) tw[i] = tw_g[i];
  const long long r0 = (long long)blockIdx.x * 2 * L;
  load_c2r(S, B0, lay, d, r0, L);
  __syncthreads();
  float2* G = fft_lines<true, false>(B0, B1, tw, plan, L, lay);
  const int total = 2 * L * nx;
  for (int i = threadIdx.x; i < total; i += blockDim.x) {
    const int q = i / nx, x = i - q * nx;
    const long long row = r0 + q;
    if (row >= d.nrows) continue;
    const long long gi = row * nx + x;
    const float v = get_comp(G, lay, q, x);
    out[gi] = accumulate ? out[gi] + v : v;
  }
}

// ---------------------------------------------------------------------------
// small elementwise kernels
// ---------------------------------------------------------------------------
// scatter one time sample of a source into a zeroed field
__global__ void k_scatter(float* f, const int* __restrict__ idx, const int* __restrict__ slot, int n,
                          const float* __restrict__ sig, int nrows_sig, int t) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const int row = (nrows_sig == 1) ? 0 : slot[j];
  f[idx[j]] = sig[(long long)(t - 1) * nrows_sig + row];
}

// rho_i = p0 / (dim c0^2) (kspaceFirstOrder3D.m:1027-1030, 2D.m:915-916)
__global__ void k_rho_init(float* r0, float* r1, float* r2, const float* __restrict__ p0, Map c0sq,
                           int dim, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const float v = p0[i] / ((float)dim * c0sq.at(i));
    r0[i] = v;
    r1[i] = v;
    if (dim == 3) r2[i] = v;
  }
}

// sensors from a materialised real field (initial-pressure step)
__global__ void k_record_field(const float* __restrict__ f, Sensor s, Clock clk, long long n) {
  const int fi = record_index(clk);
  if (fi <= 0) return;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const float v = f[i];
    if (s.mode == 1) sensor_put(s, fi, i, v);
    sensor_all(s, fi, i, v);
  }
  if (s.mode == 2) {
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < s.ns;
         j += (long long)gridDim.x * blockDim.x)
      sensor_put(s, fi, s.slot[j], f[s.idx[j]]);
  }
}

__global__ void k_advance(int* t) { *t += 1; }

__global__ void k_rms_final(const float2* __restrict__ acc, float* out, long long n, float inv_n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = sqrtf(acc[i].x * inv_n);
}

// ---------------------------------------------------------------------------
// host-side launch helpers
// ---------------------------------------------------------------------------
size_t smem_col(int n, int tl, int nbuf) { return sizeof(float2) * ((size_t)n + (size_t)nbuf * tl * n); }
size_t smem_row(int nx, int L, int nbuf) {
  return sizeof(float2) * ((size_t)nx + (size_t)nbuf * L * row_layout_stride(nx));
}

cudaError_t launch_col_fft(bool inv, const ColArgs& a, int nfields, long long nouter, const FFTPlan& plan,
                           const float2* tw, cudaStream_t st) {
  dim3 grid((a.ncols + a.tl - 1) / a.tl, (unsigned)nouter, nfields);
  const size_t sm = smem_col(plan.n, a.tl, 2);
  if (inv) {
    cudaFuncSetAttribute(k_col_fft<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_col_fft<true><<<grid, kThreads, sm, st>>>(a, plan, tw);
  } else {
    cudaFuncSetAttribute(k_col_fft<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_col_fft<false><<<grid, kThreads, sm, st>>>(a, plan, tw);
  }
  return cudaGetLastError();
}

cudaError_t launch_fused_last(const FusedArgs& a, int ninputs, long long nouter, const FFTPlan& plan,
                              const float2* tw, const SpecTables& T, int dim, cudaStream_t st) {
  dim3 grid((a.ncols + a.tl - 1) / a.tl, (unsigned)nouter, ninputs);
  const size_t sm = smem_col(plan.n, a.tl, 3);
  cudaFuncSetAttribute(k_fused_last, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  k_fused_last<<<grid, kThreads, sm, st>>>(a, plan, tw, T, dim);
  return cudaGetLastError();
}

static inline unsigned row_tiles(const Dims& d, int L) { return (unsigned)((d.nrows + 2 * L - 1) / (2 * L)); }

cudaError_t launch_x_u(const UArgs& a, const Dims& d, const FFTPlan& plan, const float2* tw, int L,
                       cudaStream_t st) {
  const size_t sm = smem_row(d.nx, L, 2);
  cudaFuncSetAttribute(k_x_u, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  k_x_u<<<dim3(row_tiles(d, L), d.dim), kThreads, sm, st>>>(a, d, plan, tw, L);
  return cudaGetLastError();
}

cudaError_t launch_x_rho(const RhoArgs& a, const Dims& d, const FFTPlan& plan, const float2* tw, int L,
                         cudaStream_t st) {
  const size_t sm = smem_row(d.nx, L, d.dim + 1);
  cudaFuncSetAttribute(k_x_rho, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  k_x_rho<<<row_tiles(d, L), kThreads, sm, st>>>(a, d, plan, tw, L);
  return cudaGetLastError();
}

cudaError_t launch_x_eos(const EosArgs& a, const Dims& d, const FFTPlan& plan, const float2* tw, int L,
                         cudaStream_t st) {
  const size_t sm = smem_row(d.nx, L, 3);
  cudaFuncSetAttribute(k_x_eos, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  k_x_eos<<<row_tiles(d, L), kThreads, sm, st>>>(a, d, plan, tw, L);
  return cudaGetLastError();
}

cudaError_t launch_x_r2c(const float* f, float2* S, const Dims& d, const FFTPlan& plan, const float2* tw,
                         int L, cudaStream_t st) {
  const size_t sm = smem_row(d.nx, L, 2);
  cudaFuncSetAttribute(k_x_r2c, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  k_x_r2c<<<row_tiles(d, L), kThreads, sm, st>>>(f, S, d, plan, tw, L);
  return cudaGetLastError();
}

cudaError_t launch_x_c2r(const float2* S, float* out, int accumulate, const Dims& d, const FFTPlan& plan,
                         const float2* tw, int L, cudaStream_t st) {
  const size_t sm = smem_row(d.nx, L, 2);
  cudaFuncSetAttribute(k_x_c2r, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  k_x_c2r<<<row_tiles(d, L), kThreads, sm, st>>>(S, out, accumulate, d, plan, tw, L);
  return cudaGetLastError();
}

static inline unsigned ew_blocks(long long n) {
  long long b = (n + kThreads - 1) / kThreads;
  if (b > 148LL * 16) b = 148LL * 16;
  if (b < 1) b = 1;
  return (unsigned)b;
}

cudaError_t launch_scatter(float* f, const int* idx, const int* slot, int n, const float* sig,
                           int nrows_sig, int t, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  k_scatter<<<(n + kThreads - 1) / kThreads, kThreads, 0, st>>>(f, idx, slot, n, sig, nrows_sig, t);
  return cudaGetLastError();
}

cudaError_t launch_rho_init(float* r0, float* r1, float* r2, const float* p0, Map c0sq, int dim,
                            long long n, cudaStream_t st) {
  k_rho_init<<<ew_blocks(n), kThreads, 0, st>>>(r0, r1, r2, p0, c0sq, dim, n);
  return cudaGetLastError();
}

cudaError_t launch_record_field(const float* f, const Sensor& s, const Clock& clk, long long n,
                                cudaStream_t st) {
  k_record_field<<<ew_blocks(n), kThreads, 0, st>>>(f, s, clk, n);
  return cudaGetLastError();
}

cudaError_t launch_advance(int* t, cudaStream_t st) {
  k_advance<<<1, 1, 0, st>>>(t);
  return cudaGetLastError();
}

cudaError_t launch_rms_final(const float2* acc, float* out, long long n, float inv_n, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  k_rms_final<<<ew_blocks(n), kThreads, 0, st>>>(acc, out, n, inv_n);
  return cudaGetLastError();
}

}  // namespace kwb
