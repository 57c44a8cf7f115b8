// Shared-memory line FFT engine for the k-space solver (sm_100a).
//
// The solver's spectral work is a sequence of 1D transforms along one grid
// axis at a time: a batch of "lines" (rows along x, or columns along y / z)
// is staged in shared memory and transformed there with a mixed-radix
// Stockham auto-sort FFT (radices 16, 8, 4, 2, 5, 3; grid edges of the form
// 2^a 3^b 5^c up to 1024).  Each stage loads R points per butterfly into
// registers, applies the inter-stage twiddles from a table built in FP64 on
// the host, runs a register-resident radix-R codelet and writes the result
// to the other half of a ping-pong buffer.
//
// Two tile layouts are used:
//   * column tile (Y / Z passes): element (line l, position n) at n*TL + l,
//     lines are consecutive kx columns, so global loads and stores of a tile
//     are 128-byte coalesced rows;
//   * row tile (X passes): element (l, n) at l*LS + n + (n >> 4), a padded
//     row layout that keeps the strided butterfly stores bank-conflict free.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace kwb {

#define KWB_MAX_STAGES 12

struct FFTPlan {
  int n;                      // transform length
  int nst;                    // number of stages
  int rad[KWB_MAX_STAGES];    // radix of each stage
};

// On sm_100 the complex additions and scalings issue as packed FP32x2
// instructions (one instruction for both components; per component the
// same IEEE rounding as the scalar form: a - b as fma(b, -1, a) is exact
// before its one rounding).
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000 && !defined(KWB_NO_F32X2)
#define KWB_F32X2 1
#endif
__host__ __device__ inline float2 c_add(float2 a, float2 b) {
#ifdef KWB_F32X2
  return __fadd2_rn(a, b);
#else
  return make_float2(a.x + b.x, a.y + b.y);
#endif
}
__host__ __device__ inline float2 c_sub(float2 a, float2 b) {
#ifdef KWB_F32X2
  return __ffma2_rn(b, make_float2(-1.f, -1.f), a);
#else
  return make_float2(a.x - b.x, a.y - b.y);
#endif
}
__host__ __device__ inline float2 c_mul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ inline float2 c_scale(float2 a, float s) {
#ifdef KWB_F32X2
  return __fmul2_rn(a, make_float2(s, s));
#else
  return make_float2(a.x * s, a.y * s);
#endif
}
__host__ __device__ inline float2 c_conj(float2 a) { return make_float2(a.x, -a.y); }
// multiply by -i (forward) or +i (inverse)
template <bool INV>
__device__ __forceinline__ float2 c_rot(float2 a) {
  return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

// ---------------------------------------------------------------------------
// radix-R codelets: X[k] = sum_n x[n] exp(-+2 pi i n k / R)
// ---------------------------------------------------------------------------
template <bool INV>
__device__ __forceinline__ void dft2(float2& a, float2& b) {
  float2 t = a;
  a = c_add(t, b);
  b = c_sub(t, b);
}

template <bool INV>
__device__ __forceinline__ void dft4(float2& x0, float2& x1, float2& x2, float2& x3) {
  float2 t0 = c_add(x0, x2), t1 = c_sub(x0, x2);
  float2 t2 = c_add(x1, x3), t3 = c_rot<INV>(c_sub(x1, x3));
  x0 = c_add(t0, t2);
  x2 = c_sub(t0, t2);
  x1 = c_add(t1, t3);
  x3 = c_sub(t1, t3);
}

template <bool INV>
__device__ __forceinline__ void dft3(float2* v) {
  const float s = 0.866025403784438646763723170752936183f;  // sin(2 pi / 3)
  float2 t1 = c_add(v[1], v[2]);
  float2 t2 = c_sub(v[1], v[2]);
  float2 m = make_float2(v[0].x - 0.5f * t1.x, v[0].y - 0.5f * t1.y);
  v[0] = c_add(v[0], t1);
  float2 r = c_rot<INV>(c_scale(t2, s));  // -i s t2 (forward)
  v[1] = c_add(m, r);
  v[2] = c_sub(m, r);
}

template <bool INV>
__device__ __forceinline__ void dft5(float2* v) {
  const float c1 = 0.309016994374947424102293417182819059f;   // cos(2 pi / 5)
  const float c2 = -0.809016994374947424102293417182819059f;  // cos(4 pi / 5)
  const float s1 = 0.951056516295153572116439333379382143f;   // sin(2 pi / 5)
  const float s2 = 0.587785252292473129168705954639072769f;   // sin(4 pi / 5)
  float2 t1 = c_add(v[1], v[4]), t2 = c_add(v[2], v[3]);
  float2 t3 = c_sub(v[1], v[4]), t4 = c_sub(v[2], v[3]);
  float2 a1 = make_float2(v[0].x + c1 * t1.x + c2 * t2.x, v[0].y + c1 * t1.y + c2 * t2.y);
  float2 a2 = make_float2(v[0].x + c2 * t1.x + c1 * t2.x, v[0].y + c2 * t1.y + c1 * t2.y);
  float2 b1 = make_float2(s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y);
  float2 b2 = make_float2(s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y);
  v[0] = c_add(v[0], c_add(t1, t2));
  float2 r1 = c_rot<INV>(b1), r2 = c_rot<INV>(b2);
  v[1] = c_add(a1, r1);
  v[4] = c_sub(a1, r1);
  v[2] = c_add(a2, r2);
  v[3] = c_sub(a2, r2);
}

// 7-point: the symmetric / antisymmetric pair sums of samples n and 7 - n,
// X[k] = a_k -+ i b_k and X[7 - k] = a_k +- i b_k for k = 1..3, with
// a_k = x0 + sum_m cos(2 pi m k / 7) t_m and b_k = sum_m sin(2 pi m k / 7) d_m.
template <bool INV>
__device__ __forceinline__ void dft7(float2* v) {
  const float c1 = 0.623489801858733530525004884004239811f;   // cos(2 pi / 7)
  const float c2 = -0.222520933956314404288902564496794759f;  // cos(4 pi / 7)
  const float c3 = -0.900968867902419126236102319507445051f;  // cos(6 pi / 7)
  const float s1 = 0.781831482468029808708444526674057750f;   // sin(2 pi / 7)
  const float s2 = 0.974927912181823607018131682993931217f;   // sin(4 pi / 7)
  const float s3 = 0.433883739117558120475768332848358754f;   // sin(6 pi / 7)
  const float2 t1 = c_add(v[1], v[6]), t2 = c_add(v[2], v[5]), t3 = c_add(v[3], v[4]);
  const float2 d1 = c_sub(v[1], v[6]), d2 = c_sub(v[2], v[5]), d3 = c_sub(v[3], v[4]);
  const float2 x0 = v[0];
  const float ca[3][3] = {{c1, c2, c3}, {c2, c3, c1}, {c3, c1, c2}};
  const float sb[3][3] = {{s1, s2, s3}, {s2, -s3, -s1}, {s3, -s1, s2}};
  v[0] = c_add(x0, c_add(t1, c_add(t2, t3)));
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float2 a = make_float2(x0.x + ca[k][0] * t1.x + ca[k][1] * t2.x + ca[k][2] * t3.x,
                                 x0.y + ca[k][0] * t1.y + ca[k][1] * t2.y + ca[k][2] * t3.y);
    const float2 b = make_float2(sb[k][0] * d1.x + sb[k][1] * d2.x + sb[k][2] * d3.x,
                                 sb[k][0] * d1.y + sb[k][1] * d2.y + sb[k][2] * d3.y);
    const float2 r = c_rot<INV>(b);
    v[k + 1] = c_add(a, r);
    v[6 - k] = c_sub(a, r);
  }
}

// 8-point: two 4-point transforms of the even / odd samples, then one
// radix-2 layer with W8^k.
template <bool INV>
__device__ __forceinline__ void dft8(float2* v) {
  const float r = 0.707106781186547524400844362104849039f;
  float2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
  float2 o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
  dft4<INV>(e0, e1, e2, e3);
  dft4<INV>(o0, o1, o2, o3);
  // W8^1 = (r, -r) forward, (r, r) inverse; W8^2 = -i / +i; W8^3 = (-r, -r) / (-r, r)
  float2 w1 = INV ? make_float2(r * (o1.x - o1.y), r * (o1.x + o1.y))
                  : make_float2(r * (o1.x + o1.y), r * (o1.y - o1.x));
  float2 w2 = c_rot<INV>(o2);
  float2 w3 = INV ? make_float2(-r * (o3.x + o3.y), r * (o3.x - o3.y))
                  : make_float2(r * (o3.y - o3.x), -r * (o3.x + o3.y));
  v[0] = c_add(e0, o0);
  v[4] = c_sub(e0, o0);
  v[1] = c_add(e1, w1);
  v[5] = c_sub(e1, w1);
  v[2] = c_add(e2, w2);
  v[6] = c_sub(e2, w2);
  v[3] = c_add(e3, w3);
  v[7] = c_sub(e3, w3);
}

template <bool INV>
__device__ __forceinline__ void dft16(float2* v) {
  // cos / sin of k*pi/8
  const float c1 = 0.923879532511286756128183189396788933f;
  const float s1 = 0.382683432365089771728459984030398866f;
  const float r = 0.707106781186547524400844362104849039f;
  float2 e[8], o[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    e[i] = v[2 * i];
    o[i] = v[2 * i + 1];
  }
  dft8<INV>(e);
  dft8<INV>(o);
  // W16^k = exp(-+ i k pi / 8)
  const float wc[8] = {1.f, c1, r, s1, 0.f, -s1, -r, -c1};
  const float ws[8] = {0.f, s1, r, c1, 1.f, c1, r, s1};
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    float2 w = make_float2(wc[k], INV ? ws[k] : -ws[k]);
    float2 t = c_mul(o[k], w);
    v[k] = c_add(e[k], t);
    v[k + 8] = c_sub(e[k], t);
  }
}

template <int R, bool INV>
__device__ __forceinline__ void dft(float2* v) {
  if constexpr (R == 2) {
    dft2<INV>(v[0], v[1]);
  } else if constexpr (R == 3) {
    dft3<INV>(v);
  } else if constexpr (R == 4) {
    dft4<INV>(v[0], v[1], v[2], v[3]);
  } else if constexpr (R == 5) {
    dft5<INV>(v);
  } else if constexpr (R == 7) {
    dft7<INV>(v);
  } else if constexpr (R == 8) {
    dft8<INV>(v);
  } else if constexpr (R == 16) {
    dft16<INV>(v);
  }
}

// ---------------------------------------------------------------------------
// tile layouts
// ---------------------------------------------------------------------------
struct ColLayout {  // element (l, n) at n * tl + l
  int tl;
  __device__ __forceinline__ int operator()(int l, int n) const { return n * tl + l; }
};
struct RowLayout {  // element (l, n) at l * ls + n + n / 16
  int ls;
  __device__ __forceinline__ int operator()(int l, int n) const { return l * ls + n + (n >> 4); }
};
__host__ __device__ inline int row_layout_stride(int n) { return n + (n >> 4) + 1; }

// One Stockham stage on `nlines` lines of length n held in shared memory.
// LINE_FAST: consecutive threads take consecutive lines (column tiles);
// otherwise consecutive butterflies of one line (row tiles).
template <int R, bool INV, bool LINE_FAST, class L>
__device__ __forceinline__ void fft_stage(const float2* __restrict__ src, float2* __restrict__ dst,
                                          const float2* __restrict__ tw, int n, int ns, int nlines,
                                          L lay) {
  const int nr = n / R;
  const int nb = nlines * nr;
  const int twstep = n / (ns * R);
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
    int l, j;
    if (LINE_FAST) {
      l = b % nlines;
      j = b / nlines;
    } else {
      j = b % nr;
      l = b / nr;
    }
    float2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = src[lay(l, j + r * nr)];
    const int k = j % ns;
    if (ns > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) {
        float2 w = tw[k * r * twstep];
        if (INV) w.y = -w.y;
        v[r] = c_mul(v[r], w);
      }
    }
    dft<R, INV>(v);
    const int idx = (j / ns) * ns * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) dst[lay(l, idx + r * ns)] = v[r];
  }
}

// Full transform of `nlines` lines held in buffer `a` (ping-pong with `b`).
// Returns the buffer that holds the result.  Ends with a block barrier.
template <bool INV, bool LINE_FAST, class L>
__device__ float2* fft_lines(float2* a, float2* b, const float2* __restrict__ tw, const FFTPlan& plan,
                             int nlines, L lay) {
  int ns = 1;
  for (int s = 0; s < plan.nst; ++s) {
    const int R = plan.rad[s];
    switch (R) {
      case 16: fft_stage<16, INV, LINE_FAST>(a, b, tw, plan.n, ns, nlines, lay); break;
      case 8: fft_stage<8, INV, LINE_FAST>(a, b, tw, plan.n, ns, nlines, lay); break;
      case 4: fft_stage<4, INV, LINE_FAST>(a, b, tw, plan.n, ns, nlines, lay); break;
      case 2: fft_stage<2, INV, LINE_FAST>(a, b, tw, plan.n, ns, nlines, lay); break;
      case 5: fft_stage<5, INV, LINE_FAST>(a, b, tw, plan.n, ns, nlines, lay); break;
      case 3: fft_stage<3, INV, LINE_FAST>(a, b, tw, plan.n, ns, nlines, lay); break;
      case 7: fft_stage<7, INV, LINE_FAST>(a, b, tw, plan.n, ns, nlines, lay); break;
      default: break;
    }
    __syncthreads();
    float2* t = a;
    a = b;
    b = t;
    ns *= R;
  }
  return a;
}

// Host-side plan construction.  Radix orders (variant):
//   0: radix-16 stages first, then 8 / 4 / 2, then 7, 5, 3 (fewest stages);
//   1: the odd radices 7, 5, 3 first, then 16, 8, 4, 2;
//   2: no radix-16 stage (8 / 4 / 2, then 7, 5, 3): more stages, lighter
//      butterflies.
// Every order computes the same transform; they round differently.
// Returns false when n has a prime factor other than 2, 3, 5 or 7.
inline bool make_fft_plan(int n, FFTPlan* p, int variant = 0) {
  p->n = n;
  p->nst = 0;
  int m = n;
  if (n < 1 || variant < 0 || variant > 2) return false;
  const int order[3][7] = {{16, 8, 4, 2, 7, 5, 3}, {7, 5, 3, 16, 8, 4, 2}, {8, 4, 2, 7, 5, 3, 0}};
  for (int i = 0; i < 7 && order[variant][i]; ++i) {
    const int r = order[variant][i];
    while (m % r == 0) {
      if (p->nst >= KWB_MAX_STAGES) return false;
      p->rad[p->nst++] = r;
      m /= r;
    }
  }
  return m == 1;
}

}  // namespace kwb
