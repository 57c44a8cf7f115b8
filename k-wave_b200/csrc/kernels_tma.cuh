// Argument blocks of the TMA-fed column kernels.
#pragma once
#include <cuda.h>

#include "kernels.cuh"

namespace kwb {

// Limit of every mbarrier wait, and a test hook: the load of tile
// `skip_tile` (-1: none) is announced on its barrier but never issued, so
// that tile's wait can only end by running out (the failure-detection test
// uses it; sessions set it from KWAVE_B200_TEST_SKIP_TMA_TILE).
struct TmaWaitArgs {
  unsigned long long limit_ns;
  int skip_tile;
};

struct ColTmaArgs {
  CUtensorMap map[4];  // one per field; box {LINES, N, 1} (y pass) or {LINES, 1, N} (last axis)
  int nfields;
  int ncx;      // column tiles along kx
  int nouter;   // outer extent of this launch (z planes for the y pass)
  int outer0;   // first outer index
  int yaxis;    // 1: the transformed axis is the tensor's y dimension, 2: z
  // Optional derived field (dual_field >= 0): its tiles are loaded from
  // field dual_src, multiplied by dual_tab[position along the transformed
  // axis] and transformed, then stored to its own map.  Tiles are then dealt
  // field-fastest, so a source tile and its derived tile are loaded at about
  // the same time and the second load is served by L2.
  int dual_field, dual_src;
  const float2* dual_tab;
  int* err;
  TmaWaitArgs wait;
};

struct FusedTmaArgs {
  CUtensorMap in[3];
  CUtensorMap out[9];
  SpecOp op[9];
  float2* outp[9];      // output buffers (written with plain stores)
  float2* dual_outp[9];         // optional second output: outp times dual_tab[outer]
  const float2* dual_tab[9];
  long long lstride;    // element stride along the transformed axis
  long long ostride;    // stride of the outer index
  int nin, fanout, ncx, nouter, yaxis, dim;
  int ncols;  // valid kx columns (nx / 2 + 1)
  // Remainder tiles (3D): when the last column kx = ncols - 1 would be alone
  // in its column tile, it is gathered for rem_y consecutive outer indices
  // into one tile instead (box {2, rem_y, n}, lines alternating kx = ncols - 1
  // and the zero-filled padding bin), so the ncx column tiles stop at
  // ncols - 1.  nrem: remainder tiles per input (0: none).
  CUtensorMap in_rem[3];
  int nrem, rem_y;
  int* err;
  TmaWaitArgs wait;
};

}  // namespace kwb
