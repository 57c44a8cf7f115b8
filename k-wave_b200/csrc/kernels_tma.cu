// Persistent, TMA-fed column passes for the compile-time transform lengths
// of tma_sizes.h (every 2^a 3^b 5^c length from 64 to 256): the y pass
// here, the fused last-axis operator in fused_tma.cuh (instantiated per
// length in generated translation units), and the host side of both.
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
#include "fused_tma.cuh"
#include "kernels.cuh"
#include "kernels_tma.cuh"
#include "spec_ops.cuh"
#include "tma.cuh"
#include "tma_sizes.h"

namespace kwb {

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

bool tma_fused_supported(int n) { return tma_col_supported(n); }

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
int tma_num_sms() {
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
  const int grid = std::min(ntiles, std::max(1, per_sm) * tma_num_sms());
  const cudaError_t e = launch_pdl(k, dim3(grid), dim3(TTile<NC>::THREADS), sm, st, a, tw);
  return e != cudaSuccess ? e : cudaGetLastError();
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
#define KWB_CASE(N) \
  case N:           \
    return fused_tma_cls<N>(a, tw, T, st);
    KWB_TMA_COL_SIZES(KWB_CASE)
#undef KWB_CASE
    default:
      return cudaErrorInvalidValue;
  }
}

}  // namespace kwb
