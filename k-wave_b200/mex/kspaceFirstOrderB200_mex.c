/*
 * kspaceFirstOrderB200_mex.c -- MEX gateway from MATLAB / GNU Octave to the
 * B200 solver's C ABI (include/kwave_b200.h), with no temporary files.
 *
 * It replaces the round trip of the C/G-suffixed wrappers
 * (kspaceFirstOrder3DC.m:159-212): instead of writing the input file
 * (kspaceFirstOrder_saveToDisk.m:44-485), running the binary and reading the
 * output file back (kspaceFirstOrder3DC.m:569-776), the wrapper hands the same
 * datasets to this function in memory and gets the same datasets back.
 *
 * Build
 *   MATLAB: mex -R2018a -I<repo>/include -L<repo>/k-wave_b200 -lkwave_b200 \
 *               LDFLAGS='$LDFLAGS -Wl,-rpath,<repo>/k-wave_b200' kspaceFirstOrderB200_mex.c
 *   Octave: mkoctfile --mex -I<repo>/include -L<repo>/k-wave_b200 -lkwave_b200 \
 *               -Wl,-rpath,<repo>/k-wave_b200 kspaceFirstOrderB200_mex.c
 *
 * Call
 *   sensor_data = kspaceFirstOrderB200_mex(datasets, options)
 *
 *   datasets  struct whose fields are the input-file datasets, named as
 *             kspaceFirstOrder_saveToDisk.m names them (Nx, dt, c0, rho0_sgx,
 *             p_source_index, sensor_mask_index, ...).  Floating-point data
 *             single or double, integers and flags any numeric class.
 *             Optional datasets are simply absent, as in the file.  Two
 *             fields have no dataset: transducer_source_apodization (one
 *             weight per u_source_index entry) and, for Cartesian sensors
 *             interpolated linearly on the device, sensor_interp_index /
 *             sensor_interp_weight (Nd + 1 vertices and weights per point).
 *   options   struct of the binary's command-line flags: logical p_raw,
 *             p_max, p_min, p_rms, p_max_all, p_min_all, p_final, u_raw,
 *             u_max, u_min, u_rms, u_max_all, u_min_all, u_final,
 *             u_non_staggered_raw; numeric start_index (-s), device (-g,
 *             -1 for the current one), verbose.  Absent fields are off / 1 / -1 / 0.
 *   sensor_data
 *             struct with the output file's datasets: Nx Ny Nz pml_x_size
 *             pml_y_size (pml_z_size in 3D), full-grid outputs (p_max_all,
 *             ux_final, ...) as [Nx Ny (Nz)], sensor outputs (p, p_max, ux,
 *             ux_non_staggered, ...) as [Ns Nt_rec] or [Ns 1].  With cuboid
 *             corners (sensor_mask_type 1) the sensor outputs come as a struct
 *             array, one element per cuboid, each output [cx cy (cz) (Nt_rec)],
 *             which is what kspaceFirstOrder3DC.m:713-767 assembles from the
 *             output file's groups.
 *
 * Errors (bad datasets, unsupported inputs, CUDA failures) are raised as
 * MATLAB errors with identifier kWaveB200:<status name> and the library's
 * message.  The caller owns every host buffer (mxArrays); the library owns
 * device memory.
 */
#include <stdint.h>
#include <string.h>

#include "kwave_b200.h"
#include "mex.h"

static const char* status_id(int code) {
  switch (code) {
    case KW_ERR_INVALID_ARGUMENT: return "kWaveB200:invalidArgument";
    case KW_ERR_CUDA: return "kWaveB200:cuda";
    case KW_ERR_OUT_OF_MEMORY: return "kWaveB200:outOfMemory";
    case KW_ERR_IO: return "kWaveB200:io";
    case KW_ERR_UNSUPPORTED: return "kWaveB200:unsupported";
    default: return "kWaveB200:internal";
  }
}

static void fail(const char* id, const char* msg) { mexErrMsgIdAndTxt(id, "%s", msg); }

/* ---- reading the datasets struct ---- */

static const mxArray* opt_field(const mxArray* s, const char* name) {
  const mxArray* a = mxGetField(s, 0, name);
  return (a && !mxIsEmpty(a)) ? a : NULL;
}

static const mxArray* req_field(const mxArray* s, const char* name) {
  const mxArray* a = opt_field(s, name);
  if (!a) mexErrMsgIdAndTxt("kWaveB200:missingDataset", "dataset %s is required", name);
  if (!mxIsNumeric(a) && !mxIsLogical(a)) mexErrMsgIdAndTxt("kWaveB200:badDataset", "dataset %s is not numeric", name);
  return a;
}

static uint64_t u64_of(const mxArray* a) { return (uint64_t)mxGetScalar(a); }

static uint64_t req_u64(const mxArray* s, const char* name) { return u64_of(req_field(s, name)); }

static uint64_t opt_u64(const mxArray* s, const char* name, uint64_t def) {
  const mxArray* a = opt_field(s, name);
  return a ? u64_of(a) : def;
}

static float req_f32(const mxArray* s, const char* name) { return (float)mxGetScalar(req_field(s, name)); }

/* A float array of the dataset: its own data when single, else a converted
 * copy (mxMalloc, freed when the MEX call returns). */
static const float* f32_data(const mxArray* a, uint64_t* numel) {
  const size_t n = mxGetNumberOfElements(a);
  *numel = (uint64_t)n;
  if (mxIsSingle(a)) return (const float*)mxGetData(a);
  if (!mxIsDouble(a)) fail("kWaveB200:badDataset", "floating-point datasets must be single or double");
  {
    const double* d = (const double*)mxGetData(a);
    float* f = (float*)mxMalloc(n * sizeof(float) + 1);
    size_t i;
    for (i = 0; i < n; ++i) f[i] = (float)d[i];
    return f;
  }
}

/* An index array of the dataset as uint64 (converted unless already uint64). */
static const uint64_t* u64_data(const mxArray* a, uint64_t* numel) {
  const size_t n = mxGetNumberOfElements(a);
  *numel = (uint64_t)n;
  if (mxGetClassID(a) == mxUINT64_CLASS) return (const uint64_t*)mxGetData(a);
  {
    uint64_t* u = (uint64_t*)mxMalloc(n * sizeof(uint64_t) + 1);
    size_t i;
    if (mxIsDouble(a)) {
      const double* d = (const double*)mxGetData(a);
      for (i = 0; i < n; ++i) u[i] = (uint64_t)d[i];
    } else if (mxIsSingle(a)) {
      const float* d = (const float*)mxGetData(a);
      for (i = 0; i < n; ++i) u[i] = (uint64_t)d[i];
    } else if (mxGetClassID(a) == mxINT32_CLASS) {
      const int32_t* d = (const int32_t*)mxGetData(a);
      for (i = 0; i < n; ++i) u[i] = (uint64_t)d[i];
    } else if (mxGetClassID(a) == mxUINT32_CLASS) {
      const uint32_t* d = (const uint32_t*)mxGetData(a);
      for (i = 0; i < n; ++i) u[i] = (uint64_t)d[i];
    } else if (mxGetClassID(a) == mxINT64_CLASS) {
      const int64_t* d = (const int64_t*)mxGetData(a);
      for (i = 0; i < n; ++i) u[i] = (uint64_t)d[i];
    } else {
      fail("kWaveB200:badDataset", "index datasets must be uint64, int64, (u)int32, single or double");
    }
    return u;
  }
}

static kw_field req_map(const mxArray* s, const char* name) {
  kw_field f;
  f.data = f32_data(req_field(s, name), &f.numel);
  return f;
}

static const float* req_f32_array(const mxArray* s, const char* name, uint64_t* numel) {
  return f32_data(req_field(s, name), numel);
}

static const uint64_t* req_u64_array(const mxArray* s, const char* name, uint64_t* numel) {
  return u64_data(req_field(s, name), numel);
}

/* Every dataset kspaceFirstOrder_saveToDisk.m writes for the fluid solver,
 * with the same required / optional rules as the binary's file reader. */
static void read_datasets(const mxArray* s, kw_input* in) {
  uint64_t n = 0;
  int three_d;
  memset(in, 0, sizeof(*in));
  in->Nx = req_u64(s, "Nx");
  in->Ny = req_u64(s, "Ny");
  in->Nz = req_u64(s, "Nz");
  in->Nt = req_u64(s, "Nt");
  three_d = in->Nz > 1;
  if (opt_u64(s, "elastic_flag", 0) || opt_u64(s, "nonuniform_grid_flag", 0))
    fail("kWaveB200:unsupported", "elastic and non-uniform-grid simulations are not supported");
  in->dx = req_f32(s, "dx");
  in->dy = req_f32(s, "dy");
  in->dz = three_d ? req_f32(s, "dz") : 0.f;
  in->dt = req_f32(s, "dt");
  in->c_ref = req_f32(s, "c_ref");
  in->pml_x_size = req_u64(s, "pml_x_size");
  in->pml_y_size = req_u64(s, "pml_y_size");
  in->pml_z_size = opt_u64(s, "pml_z_size", 0);
  in->pml_x_alpha = req_f32(s, "pml_x_alpha");
  in->pml_y_alpha = req_f32(s, "pml_y_alpha");
  in->pml_z_alpha = three_d ? req_f32(s, "pml_z_alpha") : 0.f;

  /* medium */
  in->c0 = req_map(s, "c0");
  in->rho0 = req_map(s, "rho0");
  in->rho0_sgx = req_map(s, "rho0_sgx");
  in->rho0_sgy = req_map(s, "rho0_sgy");
  if (three_d) in->rho0_sgz = req_map(s, "rho0_sgz");
  in->nonlinear_flag = opt_u64(s, "nonlinear_flag", 0);
  if (in->nonlinear_flag) in->BonA = req_map(s, "BonA");
  in->absorbing_flag = opt_u64(s, "absorbing_flag", 0);
  if (in->absorbing_flag) {
    in->alpha_coeff = req_map(s, "alpha_coeff");
    if (in->absorbing_flag == 1)
      in->alpha_power = req_f32(s, "alpha_power");
    else
      in->alpha_power = opt_field(s, "alpha_power") ? req_f32(s, "alpha_power") : 2.f;
  }

  /* initial pressure */
  in->p0_source_flag = opt_u64(s, "p0_source_flag", 0);
  if (in->p0_source_flag) {
    in->p0_source_input = req_f32_array(s, "p0_source_input", &n);
    if (n != in->Nx * in->Ny * in->Nz) fail("kWaveB200:badDataset", "p0_source_input must cover the grid");
  }

  /* pressure source */
  in->p_source_flag = opt_u64(s, "p_source_flag", 0);
  if (in->p_source_flag) {
    uint64_t rows;
    in->p_source_mode = req_u64(s, "p_source_mode");
    in->p_source_many = req_u64(s, "p_source_many");
    in->p_source_index = req_u64_array(s, "p_source_index", &in->p_source_index_numel);
    in->p_source_input = req_f32_array(s, "p_source_input", &n);
    rows = in->p_source_many ? in->p_source_index_numel : 1;
    if (n < rows * in->p_source_flag) fail("kWaveB200:badDataset", "p_source_input is shorter than its flag");
  }

  /* velocity sources */
  in->ux_source_flag = opt_u64(s, "ux_source_flag", 0);
  in->uy_source_flag = opt_u64(s, "uy_source_flag", 0);
  in->uz_source_flag = three_d ? opt_u64(s, "uz_source_flag", 0) : 0;
  if (in->ux_source_flag || in->uy_source_flag || in->uz_source_flag) {
    in->u_source_mode = req_u64(s, "u_source_mode");
    in->u_source_many = req_u64(s, "u_source_many");
    in->u_source_index = req_u64_array(s, "u_source_index", &in->u_source_index_numel);
    if (in->ux_source_flag) in->ux_source_input = req_f32_array(s, "ux_source_input", &n);
    if (in->uy_source_flag) in->uy_source_input = req_f32_array(s, "uy_source_input", &n);
    if (in->uz_source_flag) in->uz_source_input = req_f32_array(s, "uz_source_input", &n);
  }
  if (opt_u64(s, "sxx_source_flag", 0) || opt_u64(s, "syy_source_flag", 0) || opt_u64(s, "szz_source_flag", 0) ||
      opt_u64(s, "sxy_source_flag", 0) || opt_u64(s, "sxz_source_flag", 0) || opt_u64(s, "syz_source_flag", 0))
    fail("kWaveB200:unsupported", "stress sources belong to the elastic solver");

  /* axisymmetric grids and transducer sources */
  in->axisymmetric_flag = opt_u64(s, "axisymmetric_flag", 0);
  in->transducer_source_flag = opt_u64(s, "transducer_source_flag", 0);
  if (in->transducer_source_flag) {
    uint64_t nd = 0;
    if (!in->u_source_index) in->u_source_index = req_u64_array(s, "u_source_index", &in->u_source_index_numel);
    in->delay_mask = req_u64_array(s, "delay_mask", &nd);
    if (nd != in->u_source_index_numel)
      fail("kWaveB200:badDataset", "delay_mask must hold one entry per u_source_index entry");
    in->transducer_source_input =
        req_f32_array(s, "transducer_source_input", &in->transducer_source_input_numel);
    if (opt_field(s, "transducer_source_apodization")) {
      in->transducer_source_apodization = req_f32_array(s, "transducer_source_apodization", &n);
      if (n != in->u_source_index_numel)
        fail("kWaveB200:badDataset", "transducer_source_apodization needs one weight per u_source_index entry");
    }
  }

  /* sensor */
  in->sensor_mask_type = req_u64(s, "sensor_mask_type");
  if (opt_field(s, "sensor_interp_index")) {
    uint64_t nw = 0;
    in->sensor_interp_index = req_u64_array(s, "sensor_interp_index", &in->sensor_interp_numel);
    in->sensor_interp_weight = req_f32_array(s, "sensor_interp_weight", &nw);
    if (nw != in->sensor_interp_numel)
      fail("kWaveB200:badDataset", "sensor_interp_weight must match sensor_interp_index");
  } else if (in->sensor_mask_type == 0) {
    in->sensor_mask_index = req_u64_array(s, "sensor_mask_index", &in->sensor_mask_index_numel);
  } else {
    in->sensor_mask_corners = req_u64_array(s, "sensor_mask_corners", &in->sensor_mask_corners_numel);
    if (in->sensor_mask_corners_numel == 0 || in->sensor_mask_corners_numel % 6)
      fail("kWaveB200:badDataset", "sensor_mask_corners must hold 6 values per cuboid");
  }
}

static int flag_of(const mxArray* o, const char* name) {
  const mxArray* a = o ? opt_field(o, name) : NULL;
  return a ? (mxGetScalar(a) != 0.0) : 0;
}

static void read_options(const mxArray* o, kw_options* opt) {
  const mxArray* a;
  memset(opt, 0, sizeof(*opt));
  opt->p_raw = flag_of(o, "p_raw");
  opt->p_max = flag_of(o, "p_max");
  opt->p_min = flag_of(o, "p_min");
  opt->p_rms = flag_of(o, "p_rms");
  opt->p_max_all = flag_of(o, "p_max_all");
  opt->p_min_all = flag_of(o, "p_min_all");
  opt->p_final = flag_of(o, "p_final");
  opt->u_raw = flag_of(o, "u_raw");
  opt->u_max = flag_of(o, "u_max");
  opt->u_min = flag_of(o, "u_min");
  opt->u_rms = flag_of(o, "u_rms");
  opt->u_max_all = flag_of(o, "u_max_all");
  opt->u_min_all = flag_of(o, "u_min_all");
  opt->u_final = flag_of(o, "u_final");
  opt->u_non_staggered_raw = flag_of(o, "u_non_staggered_raw");
  a = o ? opt_field(o, "start_index") : NULL;
  opt->start_index = a ? u64_of(a) : 1;
  a = o ? opt_field(o, "device") : NULL;
  opt->device = a ? (int)mxGetScalar(a) : -1;
  a = o ? opt_field(o, "verbose") : NULL;
  opt->verbose = a ? (int)mxGetScalar(a) : 0;
  /* as the binary: nothing requested means the pressure series */
  if (!(opt->p_raw || opt->p_max || opt->p_min || opt->p_rms || opt->p_max_all || opt->p_min_all || opt->p_final ||
        opt->u_raw || opt->u_max || opt->u_min || opt->u_rms || opt->u_max_all || opt->u_min_all || opt->u_final ||
        opt->u_non_staggered_raw))
    opt->p_raw = 1;
}

/* ---- outputs ---- */

typedef struct {
  const char* name;
  float** slot;
  int series; /* 1: [Nt_rec][Ns], 0: [Ns] */
  int requested;
} SensorOut;

typedef struct {
  const char* name;
  float** slot;
  int requested;
} GridOut;

static mxArray* single_array(mwSize nd, const mwSize* dims) {
  return mxCreateNumericArray(nd, dims, mxSINGLE_CLASS, mxREAL);
}

static mxArray* u64_scalar(uint64_t v) {
  mxArray* a = mxCreateNumericMatrix(1, 1, mxUINT64_CLASS, mxREAL);
  *(uint64_t*)mxGetData(a) = v;
  return a;
}

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  kw_input in;
  kw_options opt;
  kw_output out;
  kw_output_sizes sz;
  kw_status st;
  uint64_t ns, nr, ng, ncub = 0, k;
  int three_d, dim, i, a;
  mwSize gdims[3];
  float* scratch[32];
  int nscratch = 0;

  if (nrhs < 1 || nrhs > 2 || !mxIsStruct(prhs[0]) || (nrhs == 2 && !mxIsStruct(prhs[1])))
    fail("kWaveB200:usage", "usage: sensor_data = kspaceFirstOrderB200_mex(datasets, options)");
  if (nlhs > 1) fail("kWaveB200:usage", "one output: the sensor data struct");
  read_datasets(prhs[0], &in);
  read_options(nrhs == 2 ? prhs[1] : NULL, &opt);
  if (kw_output_sizes_query(&in, &opt, &sz, &st) != KW_OK) fail(status_id(st.code), st.message);
  ns = sz.num_sensor_points;
  nr = sz.num_recorded_steps;
  ng = sz.grid_points;
  three_d = in.Nz > 1;
  dim = three_d ? 3 : 2;
  memset(&out, 0, sizeof(out));

  {
    /* full-grid outputs are written straight into their mxArrays */
    GridOut go[] = {
        {"p_max_all", &out.p_max_all, opt.p_max_all}, {"p_min_all", &out.p_min_all, opt.p_min_all},
        {"p_final", &out.p_final, opt.p_final},       {"ux_max_all", &out.ux_max_all, opt.u_max_all},
        {"uy_max_all", &out.uy_max_all, opt.u_max_all}, {"uz_max_all", &out.uz_max_all, opt.u_max_all && three_d},
        {"ux_min_all", &out.ux_min_all, opt.u_min_all}, {"uy_min_all", &out.uy_min_all, opt.u_min_all},
        {"uz_min_all", &out.uz_min_all, opt.u_min_all && three_d}, {"ux_final", &out.ux_final, opt.u_final},
        {"uy_final", &out.uy_final, opt.u_final},       {"uz_final", &out.uz_final, opt.u_final && three_d},
    };
    SensorOut so[] = {
        {"p", &out.p, 1, opt.p_raw},
        {"p_max", &out.p_max, 0, opt.p_max},
        {"p_min", &out.p_min, 0, opt.p_min},
        {"p_rms", &out.p_rms, 0, opt.p_rms},
        {"ux", &out.ux, 1, opt.u_raw},
        {"uy", &out.uy, 1, opt.u_raw},
        {"uz", &out.uz, 1, opt.u_raw && three_d},
        {"ux_max", &out.ux_max, 0, opt.u_max},
        {"uy_max", &out.uy_max, 0, opt.u_max},
        {"uz_max", &out.uz_max, 0, opt.u_max && three_d},
        {"ux_min", &out.ux_min, 0, opt.u_min},
        {"uy_min", &out.uy_min, 0, opt.u_min},
        {"uz_min", &out.uz_min, 0, opt.u_min && three_d},
        {"ux_rms", &out.ux_rms, 0, opt.u_rms},
        {"uy_rms", &out.uy_rms, 0, opt.u_rms},
        {"uz_rms", &out.uz_rms, 0, opt.u_rms && three_d},
        {"ux_non_staggered", &out.ux_non_staggered, 1, opt.u_non_staggered_raw},
        {"uy_non_staggered", &out.uy_non_staggered, 1, opt.u_non_staggered_raw},
        {"uz_non_staggered", &out.uz_non_staggered, 1, opt.u_non_staggered_raw && three_d},
    };
    const int ngo = (int)(sizeof(go) / sizeof(go[0])), nso = (int)(sizeof(so) / sizeof(so[0]));
    const int cuboids = in.sensor_mask_type == 1 && !in.sensor_interp_index;
    const char* head[] = {"Nx", "Ny", "Nz", "pml_x_size", "pml_y_size", "pml_z_size"};
    const char* names[64];
    int nnames = 0;
    mxArray* grid_arr[16];
    mxArray* sens_arr[32];
    mxArray* res;

    gdims[0] = (mwSize)in.Nx;
    gdims[1] = (mwSize)in.Ny;
    gdims[2] = (mwSize)in.Nz;
    for (i = 0; i < (three_d ? 6 : 5); ++i) names[nnames++] = head[i];
    for (i = 0; i < ngo; ++i) {
      grid_arr[i] = NULL;
      if (!go[i].requested) continue;
      grid_arr[i] = single_array(three_d ? 3 : 2, gdims);
      *go[i].slot = (float*)mxGetData(grid_arr[i]);
      names[nnames++] = go[i].name;
    }
    for (i = 0; i < nso; ++i) {
      sens_arr[i] = NULL;
      if (!so[i].requested) continue;
      names[nnames++] = so[i].name;
      if (!cuboids) {  /* [Ns, Nt_rec] in MATLAB order is [Nt_rec][Ns] in memory */
        mwSize d2[2];
        d2[0] = (mwSize)ns;
        d2[1] = so[i].series ? (mwSize)nr : 1;
        sens_arr[i] = single_array(2, d2);
        *so[i].slot = (float*)mxGetData(sens_arr[i]);
      } else {  /* cuboids: solved into scratch, split per cuboid below */
        scratch[nscratch] = (float*)mxMalloc(sizeof(float) * (size_t)ns * (so[i].series ? (size_t)nr : 1) + 1);
        *so[i].slot = scratch[nscratch++];
      }
    }
    (void)ng;

    if (kw_solve(&in, &opt, &out, &st) != KW_OK) fail(status_id(st.code), st.message);

    ncub = cuboids ? in.sensor_mask_corners_numel / 6 : 1;
    res = mxCreateStructMatrix((mwSize)ncub, 1, nnames, names);
    for (k = 0; k < ncub; ++k) {
      const uint64_t v[6] = {in.Nx, in.Ny, in.Nz, in.pml_x_size, in.pml_y_size, in.pml_z_size};
      for (i = 0; i < (three_d ? 6 : 5); ++i) mxSetField(res, (mwIndex)k, head[i], u64_scalar(v[i]));
    }
    for (i = 0; i < ngo; ++i)
      if (grid_arr[i]) mxSetField(res, 0, go[i].name, grid_arr[i]);
    if (!cuboids) {
      for (i = 0; i < nso; ++i)
        if (sens_arr[i]) mxSetField(res, 0, so[i].name, sens_arr[i]);
    } else {
      /* each cuboid's points are consecutive in sensor order (x fastest):
       * [cx cy cz] per step, steps last (kspaceFirstOrder_reorderCuboidCorners.m) */
      uint64_t start = 0;
      for (k = 0; k < ncub; ++k) {
        const uint64_t* c = in.sensor_mask_corners + 6 * k;
        mwSize cd[4];
        uint64_t npt = 1;
        for (a = 0; a < dim; ++a) {
          cd[a] = (mwSize)(c[3 + a] >= c[a] ? c[3 + a] - c[a] + 1 : 0);
          npt *= (uint64_t)cd[a];
        }
        for (i = 0; i < nso; ++i) {
          mxArray* arr;
          float* dst;
          uint64_t t;
          const float* src = *so[i].slot;
          if (!so[i].requested) continue;
          cd[dim] = (mwSize)nr;
          arr = single_array(so[i].series ? (mwSize)dim + 1 : (mwSize)dim, cd);
          dst = (float*)mxGetData(arr);
          if (so[i].series) {
            for (t = 0; t < nr; ++t) memcpy(dst + t * npt, src + t * ns + start, sizeof(float) * npt);
          } else {
            memcpy(dst, src + start, sizeof(float) * npt);
          }
          mxSetField(res, (mwIndex)k, so[i].name, arr);
        }
        start += npt;
      }
      for (i = 0; i < nscratch; ++i) mxFree(scratch[i]);
    }
    plhs[0] = res;
  }
}
