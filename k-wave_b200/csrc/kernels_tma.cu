// Persistent, TMA-fed column passes (the y pass and the fused last-axis
// operator) for compile-time transform lengths up to 256 (the y pass: every
// 2^a 3^b 5^c length from 64 to 256; the fused operator: the two-stage
// lengths 64, 128, 256, whose register hand-off it is built on).
//
// Each thread block loops over column tiles (TL adjacent kx columns x the
// whole line).  Tiles arrive by cp.async.bulk.tensor into a ring of shared
// memory stages while the previous tile is being transformed, and leave by
// bulk tensor stores, so the memory system streams continuously instead of
// stalling on each block's load phase.  The shared-memory tile layout
// [position][column] is exactly the TMA box layout and the column layout
// the in-place FFT engine uses.
#include <cudaTypedefs.h>

#include <algorithm>

#include "fft_ct.cuh"
#include "kernels.cuh"
#include "kernels_tma.cuh"
#include "spec_ops.cuh"
#include "tma.cuh"

namespace kwb {

// Lines per TMA tile: the compile-time tile's line count rounded down to an
// even number, so every tile starts at a bin index x = cx * LINES whose byte
// offset (8-byte bins) is a multiple of 16, as tensor copies require.
__host__ __device__ constexpr int tma_lines_of(int n) {
  return ct_lines_of(n) & ~1;  // ct_lines_of is at least 4
}

template <int NC>
struct TTile {
  static constexpr int LINES = tma_lines_of(NC);
  static constexpr int THREADS = Ct<NC>::T * LINES;
  static constexpr int ELEMS = LINES * NC;
  static constexpr unsigned BYTES = ELEMS * sizeof(float2);
  // Stage stride in elements: tensor copies read and write shared memory at
  // 128-byte aligned addresses, so each stage is padded to a multiple of 128
  // bytes (a tile of 14 lines of 90 points is 10080 bytes).
  static constexpr int STRIDE = (int)((BYTES + 127u) / 128u * 128u / sizeof(float2));
};

__device__ __forceinline__ void tile_coords(int yaxis, int cx, int o, int lines, int& x, int& y, int& z) {
  x = cx * lines;
  if (yaxis == 1) {
    y = 0;
    z = o;
  } else {
    y = o;
    z = 0;
  }
}

// Shared-memory stages of the y pass: tiles t + grid and t + 2 grid load
// while tile t is transformed and stored (two blocks per SM at 256 points).
// Two stages, three blocks per SM, measured slower at 256^3 (1.348 against
// 1.336 ms per step).
constexpr int kColStages = 3;

template <int NC, bool INV>
__global__ void __launch_bounds__(TTile<NC>::THREADS) k_col_tma(const __grid_constant__ ColTmaArgs a,
                                                                const float2* __restrict__ tw_g) {
  constexpr int TL = TTile<NC>::LINES;
  constexpr int E = TTile<NC>::STRIDE;  // stage stride (the tile, padded to 128 bytes)
  constexpr int ST = kColStages;
  extern __shared__ __align__(128) unsigned char smraw[];
  float2* bufs = reinterpret_cast<float2*>(smraw);
  float2* tw = bufs + ST * E;
  uint64_t* bar = reinterpret_cast<uint64_t*>(tw + NC);
  if (threadIdx.x == 0) {
    for (int s = 0; s < ST; ++s) mbar_init(&bar[s], 1);
    fence_mbar_init();
  }
  for (int i = threadIdx.x; i < NC; i += blockDim.x) tw[i] = tw_g[i];
  __syncthreads();
  const int per_field = a.ncx * a.nouter;
  const int ntiles = a.nfields * per_field;
  // Tiles are numbered f * per_field + r (field f, position r).  Without a
  // derived field, block b takes tiles b, b + grid, ...  With one, block b
  // takes positions b, b + grid, ... and at each position every field,
  // the derived field first: its load from the source field and the source
  // field's own load both come before the source tile is stored back in
  // place, in one block's program order, and the second load hits L2.
  const bool grouped = a.dual_field >= 0;
  auto tile_at = [&](int k) -> int {  // this block's k-th tile, -1 past the end
    if (!grouped) {
      const int t = blockIdx.x + k * gridDim.x;
      return t < ntiles ? t : -1;
    }
    const int q = k / a.nfields, j = k - q * a.nfields;
    const int r = blockIdx.x + q * gridDim.x;
    if (r >= per_field) return -1;
    const int f = (j == 0) ? a.dual_field : (j - 1 < a.dual_field ? j - 1 : j);
    return f * per_field + r;
  };
  auto coords = [&](int t, int& f, int& x, int& y, int& z) {
    f = t / per_field;
    const int r = t - f * per_field;
    const int o = r / a.ncx;
    tile_coords(a.yaxis, r - o * a.ncx, a.outer0 + o, TL, x, y, z);
  };
  // thread 0's record of the stages with a load in flight (bit s) and the
  // parity of each one's pending phase, for the drain after a failed wait
  // (in shared memory: it costs no registers in the transform loop)
  __shared__ unsigned inflight, parity_bits;
  if (threadIdx.x == 0) inflight = parity_bits = 0;
  auto issue = [&](int t, int j) {  // tile t, consumed at loop iteration j
    const int s = j % ST;
    int f, x, y, z;
    coords(t, f, x, y, z);
    mbar_expect_tx(&bar[s], TTile<NC>::BYTES);
    if (t == a.wait.skip_tile) return;  // test hook: announced, never issued
    tma_load_3d(bufs + s * E, &a.map[f == a.dual_field ? a.dual_src : f], x, y, z, &bar[s]);
    inflight |= 1u << s;
    parity_bits = (parity_bits & ~(1u << s)) | ((unsigned)((j / ST) & 1) << s);
  };
  if (threadIdx.x == 0)
    for (int f = 0; f < a.nfields; ++f) prefetch_tmap(&a.map[f]);
  pdl_wait();  // the fields are the predecessors' outputs
  pdl_trigger();
  if (threadIdx.x == 0) {
    const int t0 = tile_at(0), t1 = tile_at(1);
    if (t0 >= 0) issue(t0, 0);
    if (t1 >= 0) issue(t1, 1);
  }
  const ColLayout lay{TL};
  bool aborted = false;
  for (int it = 0;; ++it) {
    const int t = tile_at(it);
    if (t < 0) break;
    const int s = it % ST;
    float2* b = bufs + s * E;
    const bool ok = mbar_wait(&bar[s], (it / ST) & 1, a.err, a.wait.limit_ns);
    if (__syncthreads_or(!ok)) {  // every thread leaves together; nothing more is issued
      aborted = true;
      break;
    }
    if (threadIdx.x == 0) inflight &= ~(1u << s);
    int f, x, y, z;
    coords(t, f, x, y, z);
    if (f == a.dual_field) {  // the derived field: the first stage reads its input times the axis factor
      const int l = threadIdx.x % TL, tid = threadIdx.x / TL;
      const float2* tab = a.dual_tab;
      ct_stage0_ld<NC, INV>(b, l, tid, lay, [&](int ll, int n) { return c_mul(b[lay(ll, n)], __ldg(tab + n)); });
      ct_stages<NC, 1, INV>(b, tw, l, tid, lay);
    } else {
      ct_fft<NC, INV, true, TL>(b, tw, lay);
    }
    fence_async_smem();
    __syncthreads();
    if (threadIdx.x == 0) {
      tma_store_3d(&a.map[f], x, y, z, b);
      bulk_commit();
      const int t2 = tile_at(it + 2);
      if (t2 >= 0) {
        bulk_wait_read<ST - 2>();  // the store out of the stage being refilled has read it
        issue(t2, it + 2);
      }
    }
  }
  if (threadIdx.x == 0) {
    bulk_wait<0>();
    if (aborted)  // the loads still in flight land before the block's shared memory is released
      for (int s = 0; s < ST; ++s)
        if (inflight & (1u << s)) mbar_wait(&bar[s], (parity_bits >> s) & 1, nullptr, a.wait.limit_ns);
  }
}

// Operator classes of the fused kernel: one instantiation per class keeps
// only that operator's arithmetic in the kernel body.
enum FusedClass { FC_GRAD = 0, FC_NABLA = 1, FC_SRCK = 2 };

// MODE 1: every input has a single output (the register hand-off path, in
// place in the input stage: two tile buffers, three blocks per SM).
// MODE 0: the forward transform is kept and each output multiplied from it
// into a third buffer (two blocks per SM).  (The gradient's pair of outputs,
// kappa and kappa times the transform axis' derivative, also fits the
// in-place form with both taken from the hand-off registers, but at three
// blocks per SM that spills and measured slower: 1.338 against 1.330 ms.)
template <int NC, int CLS, int MODE>
__global__ void __launch_bounds__(TTile<NC>::THREADS, MODE ? 3 : 2) k_fused_tma(const __grid_constant__ FusedTmaArgs a,
                                                                     const float2* __restrict__ tw_g,
                                                                     const __grid_constant__ SpecTables T) {
  constexpr int TL = TTile<NC>::LINES;
  constexpr int E = TTile<NC>::ELEMS;
  constexpr int TH = TTile<NC>::THREADS;
  static_assert(Ct<NC>::S == 2, "the fused last-axis kernel assumes a two-stage plan");
  static_assert(TTile<NC>::STRIDE == E, "tile buffers must start at 128-byte aligned addresses");
  extern __shared__ __align__(128) unsigned char smraw[];
  float2* inb = reinterpret_cast<float2*>(smraw);  // 2 input stages
  float2* W = MODE ? nullptr : inb + 2 * E;        // product / inverse-transform buffer (MODE 0)
  float2* tw = inb + (MODE ? 2 : 3) * E;
  uint64_t* bar = reinterpret_cast<uint64_t*>(tw + NC);
  // per-line tables of the transform axis: shifted derivatives (+, -) and k^2
  float2* dpos = reinterpret_cast<float2*>(bar + 2);
  float2* dneg = dpos + NC;
  float2* dsh = dneg + NC;
  float* kl2 = reinterpret_cast<float*>(dsh + NC);
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  const int lax = (a.dim == 3) ? 2 : 1;
  for (int i = threadIdx.x; i < NC; i += blockDim.x) {
    tw[i] = tw_g[i];
    kl2[i] = T.k2[lax][i];
    if constexpr (CLS == FC_GRAD) {
      dpos[i] = T.ddk_pos[lax][i];
      dneg[i] = T.ddk_neg[lax][i];
      dsh[i] = T.shift_neg[lax] ? T.shift_neg[lax][i] : make_float2(1.f, 0.f);
    }
  }
  __syncthreads();
  const int main_in = a.ncx * a.nouter;  // column tiles of one input
  const int per_in = main_in + a.nrem;
  const int ntiles = a.nin * per_in;
  // tile t -> input g and, for a column tile, its first column cx and outer
  // index o; a remainder tile has cx = -1 and its first outer index in o
  auto decode = [&](int t, int& g, int& cx, int& o) {
    g = t / per_in;
    const int r = t - g * per_in;
    if (r < main_in) {
      o = r / a.ncx;
      cx = r - o * a.ncx;
    } else {
      cx = -1;
      o = (r - main_in) * a.rem_y;
    }
  };
  __shared__ unsigned inflight, parity_bits;  // thread 0: as in k_col_tma
  if (threadIdx.x == 0) inflight = parity_bits = 0;
  auto issue = [&](int t, int j) {  // tile t, consumed at loop iteration j
    const int s = j & 1;
    int g, cx, o, x, y, z;
    decode(t, g, cx, o);
    mbar_expect_tx(&bar[s], TTile<NC>::BYTES);  // a remainder box holds as many bytes
    if (t == a.wait.skip_tile) return;  // test hook: announced, never issued
    if (cx >= 0) {
      tile_coords(a.yaxis, cx, o, TL, x, y, z);
      tma_load_3d(inb + s * E, &a.in[g], x, y, z, &bar[s]);
    } else {
      tma_load_3d(inb + s * E, &a.in_rem[g], a.ncols - 1, o, 0, &bar[s]);
    }
    inflight |= 1u << s;
    parity_bits = (parity_bits & ~(1u << s)) | ((unsigned)((j >> 1) & 1) << s);
  };
  pdl_wait();  // the inputs are the predecessors' outputs
  pdl_trigger();
  if (threadIdx.x == 0) {
    if (blockIdx.x < ntiles) issue(blockIdx.x, 0);
    if (blockIdx.x + gridDim.x < ntiles) issue(blockIdx.x + gridDim.x, 1);
  }
  const ColLayout lay{TL};
  // the line mapping fixes this thread's column (kx) for every pass
  const int l = threadIdx.x % TL, tid = threadIdx.x / TL;
  const float cdt2sq = T.cdt2 * T.cdt2;
  constexpr int TPL = TH / TL;  // threads per line
  constexpr int M = CtHandoff<NC>::M;
  static_assert(TPL == Ct<NC>::T, "one line per group of T threads");
  bool aborted = false;
  int it = 0;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++it) {
    const int s = it & 1;
    float2* F = inb + s * E;
    int g, cx, o;
    decode(t, g, cx, o);
    // this thread's line: its column ix and outer index ol, where its
    // output goes (loff) and whether it is a real column (valid)
    int ix, ol;
    long long loff;
    bool valid;
    if (cx >= 0) {
      const int x0 = cx * TL;
      ix = min(x0 + l, a.ncols - 1);
      ol = o;
      loff = (long long)o * a.ostride + x0 + l;
      valid = (x0 + l) < a.ncols;
    } else {  // lines alternate the last column and the padding bin
      ix = a.ncols - 1;
      ol = o + (l >> 1);
      loff = (long long)ol * a.ostride + ix;
      valid = (l & 1) == 0;
    }
    const float kxy2 = __ldg(T.k2[0] + ix) + ((a.dim == 3) ? __ldg(T.k2[1] + ol) : 0.f);
    // the operator of output q: a real factor m(|k|^2), times a complex
    // factor that is constant along the line or read from a line table
    struct OpEval {
      float2 dconst;
      const float2* dline;
      float e;
      bool kappa;
    };
    auto setup = [&](int q) {
      const SpecOp op = a.op[g * a.fanout + q];
      OpEval ev{make_float2(1.f, 0.f), nullptr, 0.f, true};
      if constexpr (CLS == FC_GRAD) {
        if (op.kind != OP_KAPPA) {
          ev.kappa = op.kind != OP_SHIFT_NEG;  // the shift operator carries no kappa
          if (op.axis == lax) {
            ev.dline = (op.kind == OP_GRAD_POS) ? dpos : (op.kind == OP_GRAD_NEG ? dneg : dsh);
          } else {
            const float2* tab = (op.kind == OP_GRAD_POS)   ? T.ddk_pos[op.axis]
                                : (op.kind == OP_GRAD_NEG) ? T.ddk_neg[op.axis]
                                                           : T.shift_neg[op.axis];  // shift, kappa * shift
            ev.dconst = __ldg(tab + (op.axis == 0 ? ix : ol));
          }
        }
      } else if constexpr (CLS == FC_NABLA) {
        ev.e = 0.5f * ((op.kind == OP_NABLA1) ? T.ym2 : T.ym1);  // |k|^y = (|k|^2)^(y/2)
      }
      return ev;
    };
    // prescaled: u already holds kappa * scale times the transform (GRAD)
    auto apply = [&](const OpEval& ev, float2 (&u)[M], bool prescaled = false) {
#pragma unroll
      for (int m = 0; m < M; ++m) {
        const int p = tid + TPL * m;
        const float k2 = kxy2 + kl2[p];
        float f;
        if constexpr (CLS == FC_GRAD) {
          if (prescaled) {
            u[m] = c_mul(u[m], ev.dline ? ev.dline[p] : ev.dconst);
            continue;
          }
          f = ev.kappa ? sinc_sq(cdt2sq * k2) * T.scale : T.scale;
          u[m] = c_mul(c_scale(u[m], f), ev.dline ? ev.dline[p] : ev.dconst);
        } else if constexpr (CLS == FC_NABLA) {
          f = (k2 == 0.f) ? (ev.e == 0.f ? T.scale : 0.f) : exp2f(ev.e * log2f(k2)) * T.scale;
          u[m] = c_scale(u[m], f);
        } else {
          f = cos_sq(cdt2sq * k2) * T.scale;
          u[m] = c_scale(u[m], f);
        }
      }
    };
    // inverse last stage, straight from W to the output (and the optional
    // second output scaled by a factor constant along the line)
    auto finish = [&](int q, const float2* src) {
      float2* dst = a.outp[g * a.fanout + q] + loff;
      float2* dst2 = a.dual_outp[g * a.fanout + q];
      float2 dsc = make_float2(0.f, 0.f);
      if (dst2) {
        dst2 += loff;
        dsc = __ldg(a.dual_tab[g * a.fanout + q] + ol);
      }
      auto ld_w = [&](int ll, int pos) -> float2 { return src[lay(ll, pos)]; };
      auto st_g = [&](int, int pos, float2 v) {  // (the line is this thread's, folded into loff)
        if (valid) {
          dst[pos * a.lstride] = v;
          if (dst2) dst2[pos * a.lstride] = c_mul(v, dsc);
        }
      };
      ct_stage_io<NC, 1, true>(tw, l, tid, ld_w, st_g);
      fence_async_smem();  // the reads of src come before a TMA refill of it
      __syncthreads();     // src is reused by the next inverse
    };
    auto refill = [&]() {  // F is consumed: refill this input stage with the tile two ahead
      if (threadIdx.x == 0) {
        const int t2 = t + 2 * gridDim.x;
        if (t2 < ntiles) issue(t2, it + 2);
      }
    };
    const bool ok = mbar_wait(&bar[s], (it >> 1) & 1, a.err, a.wait.limit_ns);
    if (__syncthreads_or(!ok)) {  // every thread leaves together; nothing more is issued
      aborted = true;
      break;
    }
    if (threadIdx.x == 0) inflight &= ~(1u << s);
    if constexpr (MODE == 1) {
      float2 u[M];
      // forward first stage in place; last stage, operator and inverse first
      // stage in registers, the latter's outputs back into F once every
      // thread has read its inputs; inverse last stage to the output; then F
      // takes the tile two ahead
      ct_stage<NC, 0, false>(F, tw, l, tid, lay);
      ct_fwd_last_to_regs<NC>(F, tw, l, tid, lay, u);
      apply(setup(0), u);
      __syncthreads();
      ct_inv_first_from_regs<NC>(u, F, l, tid, lay);
      __syncthreads();
      finish(0, F);
      refill();
    } else {
      // several outputs of one input: the forward transform stays in F; each
      // output is read from it in the hand-off order, multiplied in registers
      // and given the inverse first stage on the way to W
      ct_fft<NC, false, true, TL>(F, tw, lay);
      // a first output of kappa alone (the gradient pass: kappa P, then kappa
      // P times the axis derivative) leaves kappa * scale * F in F, so the
      // later outputs carrying kappa skip its evaluation (c_mul by 1 + 0i is
      // exact, so each output's value is unchanged)
      bool kf = false;
#pragma unroll 1
      for (int q = 0; q < a.fanout; ++q) {
        float2 u[M];
#pragma unroll
        for (int m = 0; m < M; ++m) u[m] = F[lay(l, tid + TPL * m)];
        const OpEval ev = setup(q);
        apply(ev, u, kf && ev.kappa);
        if constexpr (CLS == FC_GRAD) {
          if (q == 0 && a.fanout > 1 && a.op[g * a.fanout].kind == OP_KAPPA) {
#pragma unroll
            for (int m = 0; m < M; ++m) F[lay(l, tid + TPL * m)] = u[m];  // this thread's own positions
            kf = true;
          }
        }
        ct_inv_first_from_regs<NC>(u, W, l, tid, lay);
        if (q + 1 == a.fanout) fence_async_smem();
        __syncthreads();
        if (q + 1 == a.fanout) refill();
        finish(q, W);
      }
    }
  }
  if (threadIdx.x == 0 && aborted)  // the loads still in flight land before shared memory is released
    for (int s = 0; s < 2; ++s)
      if (inflight & (1u << s)) mbar_wait(&bar[s], (parity_bits >> s) & 1, nullptr, a.wait.limit_ns);
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
static PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;

static bool get_encoder() {
  if (g_encode) return true;
  void* fn = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess || !fn)
    return false;
  g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  return true;
}

// TMA-fed y pass lengths (the box's line extent is at most 256 elements)
#define KWB_TMA_COL_SIZES(X)                                                                                   \
  X(64) X(72) X(75) X(80) X(81) X(90) X(96) X(100) X(108) X(120) X(125) X(128) X(135) X(144) X(150) X(160) \
  X(162) X(180) X(192) X(200) X(216) X(225) X(240) X(243) X(250) X(256)

bool tma_col_supported(int n) {
  switch (n) {
#define KWB_CASE(N) case N:
    KWB_TMA_COL_SIZES(KWB_CASE)
#undef KWB_CASE
    return true;
    default:
      return false;
  }
}

bool tma_fused_supported(int n) { return n == 64 || n == 128 || n == 256; }

// Tensor map over a half-spectrum buffer [nz][ny][nxp] (8-byte elements),
// box {lines, ny or 1, 1 or nz} for transforms along y (yaxis 1) or z (2).
// The x extent is the nxh bins in use, not the pitch: the last column tile
// of a row is loaded with zeros past bin nxh - 1 and stored clipped there,
// so padding costs no memory traffic.  Tiles start at x = cx * lines, a
// multiple of 16 bytes.
bool make_spec_map(CUtensorMap* m, void* base, const Dims& d, int yaxis, int n) {
  if (!get_encoder()) return false;
  const int lines = tma_lines_of(n);
  if (d.nxp % 2 != 0 || (lines * 8) % 16 != 0 || lines > 256 || n > 256) return false;
  cuuint64_t dims[3] = {(cuuint64_t)d.nxh, (cuuint64_t)d.ny, (cuuint64_t)d.nz};
  cuuint64_t strides[2] = {(cuuint64_t)d.nxp * 8, (cuuint64_t)d.nxp * d.ny * 8};
  cuuint32_t box[3] = {(cuuint32_t)lines, yaxis == 1 ? (cuuint32_t)d.ny : 1u, yaxis == 2 ? (cuuint32_t)d.nz : 1u};
  cuuint32_t es[3] = {1, 1, 1};
  CUresult r = g_encode(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, base, dims, strides, box, es,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

// Tensor map of the remainder tiles of the last-axis pass (3D): box {2,
// rows, nz} at x = nxh - 1, the lone last column and the bin past it (zero-
// filled on load; its lines are not stored).
bool make_spec_map_rem(CUtensorMap* m, void* base, const Dims& d, int n, int rows) {
  if (!get_encoder()) return false;
  if (d.nxp % 2 != 0 || (d.nxh - 1) % 2 != 0 || rows < 1 || rows > 256 || n > 256) return false;
  cuuint64_t dims[3] = {(cuuint64_t)d.nxh, (cuuint64_t)d.ny, (cuuint64_t)d.nz};
  cuuint64_t strides[2] = {(cuuint64_t)d.nxp * 8, (cuuint64_t)d.nxp * d.ny * 8};
  cuuint32_t box[3] = {2u, (cuuint32_t)rows, (cuuint32_t)n};
  cuuint32_t es[3] = {1, 1, 1};
  CUresult r = g_encode(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, base, dims, strides, box, es,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

static int g_num_sms = 0;
static int num_sms() {
  if (!g_num_sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev);
  }
  return g_num_sms;
}

template <int NC, bool INV>
static cudaError_t col_tma_t(const ColTmaArgs& a, const float2* tw, cudaStream_t st) {
  const size_t sm = kColStages * TTile<NC>::STRIDE * sizeof(float2) + NC * sizeof(float2) + kColStages * sizeof(uint64_t);
  auto k = k_col_tma<NC, INV>;
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  int per_sm = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, TTile<NC>::THREADS, sm);
  const int ntiles = a.nfields * a.ncx * a.nouter;
  const int grid = std::min(ntiles, std::max(1, per_sm) * num_sms());
  const cudaError_t e = launch_pdl(k, dim3(grid), dim3(TTile<NC>::THREADS), sm, st, a, tw);
  return e != cudaSuccess ? e : cudaGetLastError();
}

template <int NC, int CLS, int MODE>
static cudaError_t fused_tma_t(const FusedTmaArgs& a, const float2* tw, const SpecTables& T, cudaStream_t st) {
  const size_t sm = (MODE ? 2 : 3) * TTile<NC>::BYTES + NC * sizeof(float2) + 2 * sizeof(uint64_t) + 3 * NC * sizeof(float2) +
                    NC * sizeof(float);
  auto k = k_fused_tma<NC, CLS, MODE>;
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  int per_sm = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, TTile<NC>::THREADS, sm);
  const int ntiles = a.nin * (a.ncx * a.nouter + a.nrem);
  const int grid = std::min(ntiles, std::max(1, per_sm) * num_sms());
  const cudaError_t e = launch_pdl(k, dim3(grid), dim3(TTile<NC>::THREADS), sm, st, a, tw, T);
  return e != cudaSuccess ? e : cudaGetLastError();
}

template <int NC>
static cudaError_t fused_tma_cls(const FusedTmaArgs& a, const float2* tw, const SpecTables& T, cudaStream_t st) {
  const int kind = a.op[0].kind;
  const bool one = a.fanout == 1;
  if (kind == OP_GRAD_POS || kind == OP_GRAD_NEG || kind == OP_KAPPA || kind == OP_SHIFT_NEG ||
      kind == OP_KAPPA_SHIFT_NEG) {
    return one ? fused_tma_t<NC, FC_GRAD, 1>(a, tw, T, st) : fused_tma_t<NC, FC_GRAD, 0>(a, tw, T, st);
  }
  if (kind == OP_NABLA1 || kind == OP_NABLA2)
    return one ? fused_tma_t<NC, FC_NABLA, 1>(a, tw, T, st) : fused_tma_t<NC, FC_NABLA, 0>(a, tw, T, st);
  return one ? fused_tma_t<NC, FC_SRCK, 1>(a, tw, T, st) : fused_tma_t<NC, FC_SRCK, 0>(a, tw, T, st);
}

int tma_lines(int n) { return tma_lines_of(n); }

cudaError_t launch_col_tma(bool inv, int n, const ColTmaArgs& a, const float2* tw, cudaStream_t st) {
  switch (n) {
#define KWB_CASE(N) \
  case N:           \
    return inv ? col_tma_t<N, true>(a, tw, st) : col_tma_t<N, false>(a, tw, st);
    KWB_TMA_COL_SIZES(KWB_CASE)
#undef KWB_CASE
    default:
      return cudaErrorInvalidValue;
  }
}

cudaError_t launch_fused_tma(int n, const FusedTmaArgs& a, const float2* tw, const SpecTables& T, cudaStream_t st) {
  switch (n) {
    case 64: return fused_tma_cls<64>(a, tw, T, st);
    case 128: return fused_tma_cls<128>(a, tw, T, st);
    case 256: return fused_tma_cls<256>(a, tw, T, st);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace kwb
