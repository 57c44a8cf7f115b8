/*
 * kwave_b200.h -- C ABI of the B200 k-space pseudospectral acoustic solver.
 *
 * This library is a drop-in for the external solver binaries that k-Wave's
 * C/G-suffixed MATLAB functions call (kspaceFirstOrder-OMP / -CUDA).  The
 * reference defines that boundary by three things, and each entry point
 * below replaces one of them:
 *
 *   1. the HDF5 input file that MATLAB writes
 *      (k-Wave/private/kspaceFirstOrder_saveToDisk.m:44-378, writeMatrix.m);
 *      -> struct kw_input holds exactly those datasets, in memory;
 *   2. the command line that MATLAB passes to the binary
 *      (k-Wave/kspaceFirstOrder3DC.m:462-545: -i, -o, --p_raw, --p_max, ...,
 *      -s, -g, --verbose);
 *      -> struct kw_options and kw_cli_main();
 *   3. the output datasets MATLAB reads back
 *      (k-Wave/kspaceFirstOrder3DC.m:569-776: /p, /p_max, /p_rms, /ux, ...);
 *      -> struct kw_output.
 *
 * Arrays use the reference's MATLAB layout: a grid array is Nx*Ny*Nz values
 * with x fastest (the HDF5 dataset (Nz, Ny, Nx) read in C order); linear
 * indices are 1-based column-major, as MATLAB's find() returns them.  Time
 * series are [time][point] (point fastest), i.e. MATLAB [Ns, Nt].
 *
 * Errors: every entry point returns a kw_status_code and, when `status` is
 * non-NULL, a NUL-terminated message.  Inputs are validated on the host
 * before any device work.  The library owns device memory; the caller owns
 * every host buffer.
 */
#ifndef KWAVE_B200_H
#define KWAVE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KW_ABI_VERSION 1

typedef enum {
  KW_OK = 0,
  KW_ERR_INVALID_ARGUMENT = 1,
  KW_ERR_CUDA = 2,
  KW_ERR_OUT_OF_MEMORY = 3,
  KW_ERR_IO = 4,
  KW_ERR_UNSUPPORTED = 5,
  KW_ERR_INTERNAL = 6
} kw_status_code;

typedef struct {
  int code;
  char message[512];
} kw_status;

/* A float dataset that is either a scalar ([1,1,1]) or a full grid map.
 * numel is 1 or Nx*Ny*Nz. */
typedef struct {
  const float* data;
  uint64_t numel;
} kw_field;

/*
 * In-memory copy of the HDF5 input file (file format 1.2), dataset by
 * dataset (k-Wave/private/kspaceFirstOrder_saveToDisk.m:44-106, 177-378).
 * Source signals are already scaled and p0 already smoothed, as MATLAB does
 * before writing the file (kspaceFirstOrder_scaleSourceTerms.m,
 * kspaceFirstOrder_inputChecking.m:1499-1553).
 */
typedef struct {
  /* grid: Nz = 1 for a 2D simulation (saveToDisk.m:147-150) */
  uint64_t Nx, Ny, Nz, Nt;
  float dx, dy, dz, dt;
  float c_ref;
  uint64_t pml_x_size, pml_y_size, pml_z_size;
  float pml_x_alpha, pml_y_alpha, pml_z_alpha;

  /* medium */
  kw_field c0;
  kw_field rho0;
  kw_field rho0_sgx, rho0_sgy, rho0_sgz; /* density on the staggered grids */
  uint64_t nonlinear_flag;
  kw_field BonA;
  uint64_t absorbing_flag; /* 0 lossless, 1 power law, 2 stokes */
  kw_field alpha_coeff;    /* dB / (MHz^y cm), as written by MATLAB */
  float alpha_power;

  /* initial pressure */
  uint64_t p0_source_flag;
  const float* p0_source_input; /* Nx*Ny*Nz */

  /* pressure source: flag = number of signal samples */
  uint64_t p_source_flag;
  uint64_t p_source_mode; /* 0 dirichlet, 1 additive-no-correction, 2 additive */
  uint64_t p_source_many; /* 0: one signal for all points, 1: one per point */
  const uint64_t* p_source_index; /* 1-based linear indices */
  uint64_t p_source_index_numel;
  const float* p_source_input; /* [p_source_flag][1 or index_numel] */

  /* velocity sources (share u_source_index) */
  uint64_t ux_source_flag, uy_source_flag, uz_source_flag;
  uint64_t u_source_mode;
  uint64_t u_source_many;
  const uint64_t* u_source_index;
  uint64_t u_source_index_numel;
  const float* ux_source_input;
  const float* uy_source_input;
  const float* uz_source_input;

  /* sensor: type 0 = linear indices, 1 = cuboid corners */
  uint64_t sensor_mask_type;
  const uint64_t* sensor_mask_index; /* 1-based */
  uint64_t sensor_mask_index_numel;
  const uint64_t* sensor_mask_corners; /* 6 x K, 1-based [x1 y1 z1 x2 y2 z2] per cuboid */
  uint64_t sensor_mask_corners_numel;  /* 6 * K */

  /*
   * Transducer source (3D; saveToDisk.m:289-293, 339-343): while the 1-based
   * time index t <= transducer_source_flag, the x velocity at each point of
   * u_source_index gains apodization[i] * transducer_source_input[delay_mask[i] + t - 2]
   * (kspaceFirstOrder3D.m:886-902).  delay_mask is 1-based, one entry per
   * u_source_index entry; the velocity source flags must then be 0.  The
   * input file carries no apodization: NULL means 1 for every point.
   */
  uint64_t transducer_source_flag;
  const float* transducer_source_input;
  uint64_t transducer_source_input_numel;
  const uint64_t* delay_mask;
  const float* transducer_source_apodization;

  /*
   * Axisymmetric simulation (kspaceFirstOrderAS.m; saveToDisk.m:90-100, 125):
   * x axial, y radial with the axis at y = 0, Nz = 1.  Medium, p0 and source
   * positions are given on the Nx x Ny grid; the radial PML sits at the
   * outer radius only.  Initial pressure, pressure sources and axial (x)
   * velocity sources, lossless or Stokes media (absorbing_flag 0 or 2), with
   * or without B/A.
   */
  uint64_t axisymmetric_flag;

  /*
   * Cartesian sensor points by linear interpolation (the in-memory solvers'
   * 'CartInterp' 'linear', kspaceFirstOrder_extractSensorData.m:296-420):
   * for each point, Nd + 1 vertex indices (1-based linear) and barycentric
   * weights, point-major (point j uses entries j*(Nd+1) .. j*(Nd+1)+Nd).
   * When set, sensor_mask_type must be 0, sensor_mask_index is not read,
   * and the sensor outputs are per point, interpolated on the device every
   * step; the full-grid outputs are unaffected.  No input-file dataset
   * carries this.
   */
  const uint64_t* sensor_interp_index;
  const float* sensor_interp_weight;
  uint64_t sensor_interp_numel; /* points * (Nd + 1) */
} kw_input;

/* What to record, and run settings: the binary's command-line flags. */
typedef struct {
  int p_raw, p_max, p_min, p_rms, p_max_all, p_min_all, p_final;
  int u_raw, u_max, u_min, u_rms, u_max_all, u_min_all, u_final;
  int u_non_staggered_raw;
  uint64_t start_index; /* -s, 1-based; 0 is read as 1 */
  int device;           /* -g, CUDA device ordinal; -1: current device */
  int verbose;          /* --verbose 0..2 */
} kw_options;

/*
 * Caller-owned host buffers for the outputs, sized as kw_output_sizes()
 * reports.  Pointers for outputs that were not requested may be NULL.
 * Sensor outputs are in sensor order: the order of sensor_mask_index, or,
 * for cuboids, the concatenation of each cuboid's points (x fastest).
 */
typedef struct {
  float* p;                       /* [Nt_rec][Ns] */
  float *p_max, *p_min, *p_rms;   /* [Ns] */
  float *p_max_all, *p_min_all;   /* [Nx*Ny*Nz] */
  float* p_final;                 /* [Nx*Ny*Nz] */
  float *ux, *uy, *uz;            /* [Nt_rec][Ns] */
  float *ux_max, *uy_max, *uz_max;
  float *ux_min, *uy_min, *uz_min;
  float *ux_rms, *uy_rms, *uz_rms;
  float *ux_max_all, *uy_max_all, *uz_max_all;
  float *ux_min_all, *uy_min_all, *uz_min_all;
  float *ux_final, *uy_final, *uz_final;
  float *ux_non_staggered, *uy_non_staggered, *uz_non_staggered; /* [Nt_rec][Ns] */
} kw_output;

typedef struct {
  uint64_t num_sensor_points;    /* Ns */
  uint64_t num_recorded_steps;   /* Nt_rec = Nt - start_index + 1 */
  uint64_t grid_points;          /* Nx*Ny*Nz */
  uint64_t device_bytes;         /* device memory the solve will allocate */
} kw_output_sizes;

/* Library version string. */
const char* kw_version(void);

/* Output sizes for an input / option pair (validates the input). */
int kw_output_sizes_query(const kw_input* in, const kw_options* opt, kw_output_sizes* sizes,
                          kw_status* status);

/*
 * Run one simulation from host buffers to host buffers: the whole job of
 * `kspaceFirstOrder-CUDA -i in.h5 -o out.h5 <flags>` without the files
 * (k-Wave/kspaceFirstOrder3DC.m:535-563 runs the binary; :569-776 reads
 * its outputs).
 */
int kw_solve(const kw_input* in, const kw_options* opt, kw_output* out, kw_status* status);

/*
 * The file-based drop-in: read a k-Wave HDF5 input file, run, and write the
 * output file that kspaceFirstOrder{2D,3D}{C,G} read back
 * (k-Wave/kspaceFirstOrder3DC.m:544 builds this call).
 */
int kw_run_file(const char* input_h5, const char* output_h5, const kw_options* opt, kw_status* status);

/*
 * kw_run_file with checkpoints (the binaries' --checkpoint_file,
 * --checkpoint_timesteps, --checkpoint_interval): the state is written to
 * `checkpoint_file` every `checkpoint_timesteps` steps and / or every
 * `checkpoint_interval_s` seconds; if the file exists when the run starts it
 * is resumed from; it is removed once the output file is written.
 */
int kw_run_file_checkpointed(const char* input_h5, const char* output_h5, const kw_options* opt,
                             const char* checkpoint_file, uint64_t checkpoint_timesteps, double checkpoint_interval_s,
                             kw_status* status);

/* Command-line entry: the binary's argv, e.g.
 * {"kspaceFirstOrder-B200", "-i", "in.h5", "-o", "out.h5", "--p_raw", "-s", "10"}.
 * Returns the process exit code. */
int kw_cli_main(int argc, char** argv);

/*
 * Resident simulations, for callers that keep inputs on the device and
 * advance a simulation in steps (batching, serving, benchmarking).  Not a
 * reference interface: the reference runs one whole solve per process.
 */
typedef struct kw_session kw_session;

int kw_session_create(const kw_input* in, const kw_options* opt, kw_session** session, kw_status* status);
/* Enqueue `nsteps` time steps (asynchronous on the session's stream). */
int kw_session_advance(kw_session* s, uint64_t nsteps, kw_status* status);
/* Device time of the last kw_session_advance() in ms (synchronises). */
int kw_session_elapsed_ms(kw_session* s, float* ms, kw_status* status);
/* Block until all queued work finished. */
int kw_session_sync(kw_session* s, kw_status* status);
/* Steps completed so far. */
uint64_t kw_session_steps_done(const kw_session* s);
/* Non-blocking: how many kw_session_advance() calls have steps still
 * running on the device (0: the session is idle).  What a scheduler that
 * interleaves many sessions polls instead of blocking in kw_session_sync. */
int kw_session_query(kw_session* s, uint64_t* in_flight, kw_status* status);
/* CUDA stream priorities of the current device: `least` is the default and
 * lowest, `greatest` (numerically smaller) the highest. */
int kw_stream_priority_range(int* least, int* greatest);
/* Run the session's work at a CUDA stream priority (clamped to the device's
 * range).  Waits for the session's queued work first.  A scheduler gives the
 * shortest jobs the highest priority: their kernels go first and longer
 * jobs' kernels fill the SMs they leave idle. */
int kw_session_set_priority(kw_session* s, int priority, kw_status* status);
/*
 * Checkpoints (the external binaries' --checkpoint_file; file_type
 * 'checkpoint', k-Wave/private/getH5Literals.m:48).  kw_session_save waits
 * for the session's work and writes its state between two steps -- fields,
 * the pressure spectrum, every sensor accumulator, the step index -- to an
 * HDF5 file.  kw_session_restore loads such a file into a freshly created
 * session of the same input and options; the run then continues bit for bit
 * as if it had never stopped.
 */
int kw_session_save(kw_session* s, const char* path, kw_status* status);
int kw_session_restore(kw_session* s, const char* path, kw_status* status);
/* Copy the outputs recorded so far into host buffers. */
int kw_session_read(kw_session* s, kw_output* out, kw_status* status);
/* The session's CUDA stream (a cudaStream_t), for event timing by callers. */
void* kw_session_stream(kw_session* s);
/* Number of kernel launches one time step issues (the hot-path kernels). */
uint64_t kw_session_launches_per_step(const kw_session* s);
void kw_session_destroy(kw_session* s);

/*
 * No counterpart in the reference (one solve per process there).
 *
 * Batches: many resident sessions advanced together, each time step of all
 * of them one CUDA graph launch (a parent graph whose independent branches
 * are the sessions' captured steps, so their kernels run side by side).
 * Steps that cannot be replayed (an initial-pressure start, a session's
 * last step, steps of a per-point corrected source) run on their own, in
 * order.  Sessions with different Nt stop at their own last step.  Work is
 * enqueued after each member's queued work, and each member's later work
 * (kw_session_read, kw_session_sync) waits for it.  Streamed sessions
 * cannot be batched.  The sessions must outlive the batch (destroy the
 * batch first).  Results are bit for bit those of kw_session_advance.
 */
typedef struct kw_batch kw_batch;
int kw_batch_create(kw_session* const* sessions, int n, kw_batch** batch, kw_status* status);
int kw_batch_advance(kw_batch* b, uint64_t nsteps, kw_status* status);
/* Device time of the last kw_batch_advance() in ms (synchronises). */
int kw_batch_elapsed_ms(kw_batch* b, float* ms, kw_status* status);
int kw_batch_sync(kw_batch* b, kw_status* status);
/* Parent-graph launches so far: one per time step advanced as a batch. */
uint64_t kw_batch_graph_launches(const kw_batch* b);
/* Destroys the batch only (its sessions stay). */
void kw_batch_destroy(kw_batch* b);

/*
 * No counterpart in the reference (its binaries launch one fixed way).
 *
 * Launch schedule of the time step.  The y-inverse / row / y-forward chains
 * of a 3D step run whole or as z slabs, the slabs on one stream or
 * alternating between two, and the runtime-plan FFT kernels (lengths with a
 * factor 7, or outside 64..1024) transform a chosen number of lines per
 * block: these give bit-identical results.  The runtime-plan engine's radix
 * order can be chosen too (0: radix 16 first, 1: odd radices first, 2: no
 * radix 16); another order rounds differently, within FP32 rounding.
 */
typedef struct {
  int slab_planes;   /* z planes per slab (Nz: the chains are not split) */
  int streams;       /* 1, or 2: slabs alternate between two streams */
  int row_lines;     /* lines per block of runtime-plan row (x) kernels */
  int col_lines;     /* cap on lines per block of runtime-plan column kernels */
  int radix_plan;    /* radix order of the runtime-plan engine (0, 1, 2) */
  int candidates;    /* schedules kw_tune timed (0: the grid offers no choice) */
  float ms_per_step; /* device time per step of the chosen schedule */
  float ms_default;  /* device time per step of the built-in schedule */
} kw_schedule;

/*
 * Time the candidate schedules on a scratch copy of the simulation (same
 * grid, medium, sources and sensor reductions; recorded series left out, so
 * the copy needs about the device memory of kw_output_sizes' device_bytes)
 * and remember the fastest for this grid, step class and device: sessions
 * and solves created afterwards in the process use it.  A challenger must
 * beat the current choice by more than 1 %.  Takes up to about 200 time
 * steps (80 on compile-time lengths) plus one set-up.  With KWAVE_B200_WISDOM=<file> the remembered schedules
 * are merged into that file and read from it by the first session of a
 * process; with KWAVE_B200_TUNE=1 a session whose key is not remembered
 * tunes itself at creation when free device memory allows.
 */
int kw_tune(const kw_input* in, const kw_options* opt, kw_schedule* chosen, kw_status* status);
/* Read / write remembered schedules (text: key slab_planes streams row_lines
 * col_lines radix_plan ms_per_step).  Export merges into an existing file. */
int kw_wisdom_import(const char* path, kw_status* status);
int kw_wisdom_export(const char* path, kw_status* status);
/* Forget every remembered schedule (and do not read KWAVE_B200_WISDOM again). */
void kw_wisdom_forget(void);
/* The schedule a session runs with (ms and candidate fields are 0). */
int kw_session_schedule(const kw_session* s, kw_schedule* sched);

/*
 * A plain real-to-complex transform of a 2D / 3D grid (nz = 1: 2D) run by the
 * solver's own FFT passes, standing where the reference calls MATLAB's
 * fftn / ifftn on a real field (kspaceFirstOrder3D.m:790, 905-907).  The
 * time loop does not use it (it fuses every pass with the physics); it lets
 * the passes be timed beside a library FFT (cuFFT) and checked on their own.
 *   d_real: nx*ny*nz floats, x fastest; d_spec: nz*ny*nxp complex floats
 *   ([z][y][kx], kx in [0, nx/2], nxp = nx/2 + 1 rounded up to even).
 * inverse = 0: d_spec = fftn(d_real) (half spectrum).  inverse = 1: d_real =
 * nx*ny*nz * ifftn(d_spec), unnormalised, and d_spec is overwritten.
 * `passes` selects the axes to run (bit 0: x, bit 1: y, bit 2: z; 7 = all),
 * so each pass can be timed alone.  Work is only enqueued on `stream`;
 * kw_fft3d_check reports a device-side wait that ran out.  The plan holds
 * the twiddle tables (device memory) of the device current at creation.
 */
typedef struct kw_fft3d_plan kw_fft3d_plan;
int kw_fft3d_create(uint64_t nx, uint64_t ny, uint64_t nz, kw_fft3d_plan** plan, kw_status* status);
int kw_fft3d_exec(kw_fft3d_plan* plan, int inverse, unsigned passes, float* d_real, void* d_spec, void* stream,
                  kw_status* status);
int kw_fft3d_check(kw_fft3d_plan* plan, kw_status* status);
void kw_fft3d_destroy(kw_fft3d_plan* plan);

/*
 * No counterpart in the reference.
 *
 * The k-space staggered gradient of a 2D field, for callers that cannot
 * allocate device memory: applications that keep all device memory in their
 * own pool (MATLAB's gpuArray data, a PyTorch caching allocator) or loops
 * where the device-wide synchronisation a cudaMalloc / cudaFree can cause is
 * not acceptable.  For f on an nx x ny grid (x fastest) it writes
 *   gx = real(ifft2(i kx exp(i kx dx/2) kappa fft2(f)))
 *   gy = real(ifft2(i ky exp(i ky dy/2) kappa fft2(f)))     (d_gy may be NULL)
 * with kappa = sinc(c_ref |k| dt / 2) -- the gradient kspaceFirstOrder2D.m:920-921
 * applies to an initial pressure.  d_f, d_gx, d_gy are nx*ny floats of the
 * current device, owned by the caller.  The call only enqueues work on
 * `stream` (a cudaStream_t, NULL for the default stream).
 *
 * It allocates nothing: its intermediate spectra live in a fixed static
 * device array sized for edges up to KW_NOALLOC_MAX_EDGE (8 MiB per device);
 * larger grids are rejected with KW_ERR_INVALID_ARGUMENT.  Every call looks
 * up that array's address on the current device; the first call on a device
 * may also load the library's device code there, so make it before any
 * stream capture.  A stream of another device is rejected.  The array is
 * shared by all calls on a
 * device: calls that overlap in time on one device race and must be
 * serialised by the caller.
 */
#define KW_NOALLOC_MAX_EDGE 1024
int kw_kspace_gradient_noalloc(const float* d_f, float* d_gx, float* d_gy, uint64_t nx, uint64_t ny, float dx,
                               float dy, float c_ref, float dt, void* stream, kw_status* status);

#ifdef __cplusplus
}
#endif

#endif /* KWAVE_B200_H */
