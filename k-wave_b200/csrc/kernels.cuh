// Device-side data structures shared by the solver kernels and the host
// orchestrator.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "fft_engine.cuh"

namespace kwb {

constexpr int kThreads = 256;

// Grid geometry.  Real fields are stored x-fastest ([z][y][x], the column-
// major order of the reference's MATLAB arrays); the half spectrum of a real
// field is stored [z][y][kx] with kx in [0, nx/2] and a row pitch of nxp.
struct Dims {
  int nx, ny, nz;   // nz == 1 in 2D
  int dim;          // 2 or 3
  int nxh;          // nx / 2 + 1
  int nxp;          // spectral row pitch (complex elements)
  long long nrows;  // ny * nz
  long long npts;   // nx * ny * nz
  long long row0, row1;  // rows [row0, row1) processed by a row-kernel launch
};

enum SpecOpKind {
  OP_GRAD_POS = 0,   // i k_a exp(+i k_a d_a / 2) * kappa
  OP_GRAD_NEG = 1,   // i k_a exp(-i k_a d_a / 2) * kappa
  OP_NABLA1 = 2,     // |k|^(y-2)
  OP_NABLA2 = 3,     // |k|^(y-1)
  OP_SRC_KAPPA = 4,  // cos(c_ref |k| dt / 2)
  OP_IDENTITY = 5,
  OP_KAPPA = 6,      // kappa alone (the axis factor applied elsewhere)
  OP_SHIFT_NEG = 7,  // exp(-i k_a d_a / 2): staggered -> regular grid along axis a, no kappa
  OP_KAPPA_SHIFT_NEG = 8,  // kappa * exp(-i k_a d_a / 2): the axisymmetric u_r / r term
};

struct SpecOp {
  int kind;
  int axis;
};

// 1D operator tables (built in FP64 on the host, stored FP32) and scalars
// from which the non-separable k-space operators are generated per point.
struct SpecTables {
  const float* k2[3];        // squared wavenumber per axis, FFT order (x: nxh entries)
  const float2* ddk_pos[3];  // i k exp(+i k d / 2), FFT order (x: nxh entries)
  const float2* ddk_neg[3];  // i k exp(-i k d / 2)
  const float2* shift_neg[3];  // exp(-i k d / 2) (kspaceFirstOrder_createStorageVariables.m)
  float cdt2;                // c_ref * dt / 2
  float ym2, ym1;            // alpha_power - 2, alpha_power - 1
  float scale;               // 1 / (nx ny nz): the inverse-FFT normalisation
};

// A medium property that is either a full map or a scalar.
struct Map {
  const float* p;
  float s;
  __device__ __forceinline__ float at(long long i) const { return p ? __ldg(p + i) : s; }
};

// Time-step clock: `t` points at the device-resident 1-based time index of
// the step being computed, so a captured step graph can be replayed.
struct Clock {
  const int* t;
  int start;  // record start index (1-based)
};

// Sparse sources applied inside the X-row kernels.  Indices are sorted
// 0-based linear indices; `slot` gives the signal row of each entry.
struct SparseSource {
  int n;             // number of source points (0: no sparse source)
  const int* idx;    // sorted linear indices
  const int* slot;   // signal row for each sorted entry
  const float* sig;  // signal matrix [t][row] (row fastest)
  int nrows_sig;     // rows in the signal matrix (1 or n)
  int len;           // number of signal samples (active while t <= len)
  int mode;          // 0 dirichlet (set), 1 additive without correction (add)
  // transducer sources (kspaceFirstOrder3D.m:886-902): one signal read at a
  // per-entry offset, sample delay + t - 1, times a per-entry weight
  const int* delay;    // nullptr: no offset
  const float* weight; // nullptr: 1
};

// Dense additive source field, added inside the update epilogue while
// t <= len: field * sig[t-1] (sig == nullptr: field * 1).
struct DenseSource {
  const float* field;
  const float* sig;
  int len;
};

// Sensor recording.  `mode` 0: off; 1: every grid point is a sensor point
// and the output slot is the linear index; 2: sorted sparse list with slots.
struct Sensor {
  int mode;
  int ns;
  int ring;        // raw series rows held on the device (0: every recorded step)
  const int* idx;
  const int* slot;
  float* raw;      // [nrec][ns] time series (nullptr: off)
  float* vmax;     // per-point reductions (nullptr: off)
  float* vmin;
  float2* rms;     // sum of squares of the completed blocks, Kahan {sum, compensation}
  float* rms_blk;  // plain sum of squares of the block in progress
  float* max_all;  // full-grid reductions (nullptr: off)
  float* min_all;
};

// The rms sum of squares is accumulated in blocks of kRmsBlock recorded
// steps: within a block in a plain FP32 partial sum (4 bytes read and
// written per point and step), and at each block's end the partial sum is
// added to a Kahan-compensated total (8 more bytes each way, once per
// block).  The rounding error stays near kRmsBlock ulp of the sum, where a
// plain running sum over Nt steps reaches Nt ulp, and the per-step traffic
// is half that of a Kahan pair updated every step.  Record index fi (1-based)
// is the ((fi - 1) % kRmsBlock)-th step of its block.
constexpr int kRmsBlock = 16;

// Bounded waits of the row kernels (the mbarrier waits on their bulk
// copies): time limit (0: the 2 s default) and the word a wait that runs
// out writes its error code to.
struct WaitCtl {
  int* err;
  unsigned long long limit_ns;
};

// ---------------------------------------------------------------------------
// kernel argument blocks
// ---------------------------------------------------------------------------
struct ColArgs {
  float2* buf[4];     // fields transformed in place (blockIdx.z)
  int outer0;         // first outer index (z plane) of this launch
  int ncols;          // valid columns (kx values)
  long long lstride;  // element stride along the transformed axis
  long long ostride;  // stride of the outer index (blockIdx.y)
  int tl;             // columns per tile
};

struct FusedArgs {
  const float2* in[3];  // inputs (blockIdx.z)
  float2* out[9];       // outputs [input * fanout + o]
  SpecOp op[9];
  float2* dual_out[9];         // optional second output: out times dual_tab[outer]
  const float2* dual_tab[9];
  int fanout;
  int ncols;
  long long lstride, ostride;
  int tl;
};

struct UArgs {
  const float2* S[3];  // gradient spectra, already inverse-transformed along y / z
  const float2* kmul[3];  // optional kx multiplier applied as the spectra are read
  float2* Sout[3];     // receives the x-transform of the new velocity
  float* u[3];
  Map rinv[3];         // 1 / rho0 on the staggered grids
  const float* pml_sg[3];
  float dt;
  int init;            // 1: u = dt * rinv * grad / 2 (initial-pressure start)
  int do_r2c;
  SparseSource src;    // velocity sources share one index list ...
  const float* src_sig[3];  // ... with one signal matrix per component
  int src_len[3];
  DenseSource dsrc[3];
  Sensor sens[3];
  Clock clk;
  WaitCtl wait;
};

// The box of grid points whose density is stored merged: rho_x holds
// rho_x + rho_y (+ rho_z) and rho_y, rho_z are neither read nor written.
// The split density exists for the split-field PML; where every PML factor
// of a point is 1 the split update summed over the axes,
// rho - dt (2 rho + rho0 or rho0) sum_i du_i/dx_i, needs only the sum, so
// such points save 16 bytes of traffic per step in 3D.  The box is a run of
// PML factors equal to 1 along each axis (the host picks it), x bounds
// multiples of 4 so the rule holds per aligned group of 4 x points (the
// vector epilogue's unit); an empty box stores every point split.  Every
// kernel that reads or writes the density uses this rule.
struct RhoBox {
  int lo[3], hi[3];
  __device__ __forceinline__ bool row(int y, int z, int dim) const {
    return y >= lo[1] && y < hi[1] && (dim < 3 || (z >= lo[2] && z < hi[2]));
  }
  __device__ __forceinline__ bool at(int x, int y, int z, int dim) const {
    const int g = x & ~3;
    return g >= lo[0] && g + 4 <= hi[0] && row(y, z, dim);
  }
};

struct RhoArgs {
  const float2* S[3];  // divergence spectra, inverse-transformed along y / z
  RhoBox box;          // merged-density points
  float* rho[3];
  Map rho0;
  const float* pml[3];
  float dt;
  int nonlinear;
  Map bona;
  Map c0sq;
  int eos;             // 0 lossless, 1 absorbing, 2 stokes
  Map tau;             // stokes coefficient
  SparseSource src;
  DenseSource dsrc;
  float* p_loc;        // absorbing: c0^2 (sum rho + B/A term)
  float2* S_q;         // absorbing: x-transform of rho0 * sum(du)
  float2* S_r;         // absorbing: x-transform of sum(rho)
  float* p_out;        // lossless / stokes: p (nullptr: not stored)
  float2* S_p;         // lossless / stokes: x-transform of p
  Sensor sens;
  Clock clk;
  const float2* S_rr;  // axisymmetric: the u_r / r spectrum, added to S[1] as it is read
  WaitCtl wait;
};

struct EosArgs {
  const float2* S_a;   // F^-1{nabla1 F{rho0 sum du}} (x still transformed)
  const float2* S_b;   // F^-1{nabla2 F{sum rho}}
  const float* p_loc;
  Map c2tau, c2eta;    // c0^2 tau, c0^2 eta
  float* p_out;
  float2* S_p;
  Sensor sens;
  Clock clk;
  WaitCtl wait;
};

}  // namespace kwb
