// File-based drop-in for kspaceFirstOrder-OMP / -CUDA: read the HDF5 input
// file written by k-Wave/private/kspaceFirstOrder_saveToDisk.m, run the
// solver, and write the output file that k-Wave/kspaceFirstOrder3DC.m:569-776
// reads back.  kw_cli_main() parses the command line those wrappers build
// (kspaceFirstOrder3DC.m:462-545).
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <stdexcept>
#include <string>
#include <vector>

#include "hdf5_lite.h"
#include "kwave_b200.h"

namespace {

struct IoError : std::runtime_error {
  int code;
  IoError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

int set_status(kw_status* st, int code, const std::string& msg) {
  if (st) {
    st->code = code;
    std::snprintf(st->message, sizeof(st->message), "%s", msg.c_str());
  }
  return code;
}

// The datasets of one input file, owned here, pointed to by kw_input.
struct InputFile {
  kw_input in{};
  std::vector<std::vector<float>> f;
  std::vector<std::vector<uint64_t>> u;
  std::vector<uint64_t> corner_dims;  // per cuboid: cx, cy, cz

  const float* keep_f(std::vector<float>&& v) {
    f.push_back(std::move(v));
    return f.back().data();
  }
  const uint64_t* keep_u(std::vector<uint64_t>&& v) {
    u.push_back(std::move(v));
    return u.back().data();
  }
};

uint64_t scalar_u64(h5::Reader& r, const char* name) {
  auto v = r.read_u64(std::string("/") + name);
  if (v.empty()) throw IoError(KW_ERR_IO, std::string(name) + " is empty");
  return v[0];
}

float scalar_f(h5::Reader& r, const char* name) {
  auto v = r.read_float(std::string("/") + name);
  if (v.empty()) throw IoError(KW_ERR_IO, std::string(name) + " is empty");
  return v[0];
}

uint64_t opt_u64(h5::Reader& r, const char* name, uint64_t dflt) {
  return r.exists(std::string("/") + name) ? scalar_u64(r, name) : dflt;
}

void need(h5::Reader& r, const char* name) {
  if (!r.exists(std::string("/") + name))
    throw IoError(KW_ERR_IO, std::string("input file lacks the dataset /") + name);
}

kw_field field(InputFile& F, h5::Reader& r, const char* name) {
  need(r, name);
  auto v = r.read_float(std::string("/") + name);
  kw_field fd;
  fd.numel = v.size();
  fd.data = F.keep_f(std::move(v));
  return fd;
}

// kspaceFirstOrder_saveToDisk.m:44-378 (file format 1.2)
void read_input(const std::string& path, InputFile& F) {
  h5::Reader r(path);
  const std::string ft = r.attribute_string("/", "file_type");
  if (!ft.empty() && ft != "input") throw IoError(KW_ERR_IO, path + " is a '" + ft + "' file, not an input file");
  for (const char* unsupported : {"elastic_flag", "nonuniform_grid_flag"})
    if (opt_u64(r, unsupported, 0) != 0)
      throw IoError(KW_ERR_UNSUPPORTED, std::string(unsupported) + " is set: only the fluid solver is supported");
  for (const char* sflag : {"sxx_source_flag", "syy_source_flag", "szz_source_flag", "sxy_source_flag",
                            "sxz_source_flag", "syz_source_flag"})
    if (opt_u64(r, sflag, 0) != 0) throw IoError(KW_ERR_UNSUPPORTED, "stress sources belong to the elastic solver");
  kw_input& in = F.in;
  for (const char* n : {"Nx", "Ny", "Nz", "Nt", "dx", "dy", "dt", "c_ref", "c0", "rho0", "rho0_sgx", "rho0_sgy",
                        "pml_x_size", "pml_y_size", "pml_x_alpha", "pml_y_alpha", "sensor_mask_type"})
    need(r, n);
  in.Nx = scalar_u64(r, "Nx");
  in.Ny = scalar_u64(r, "Ny");
  in.Nz = scalar_u64(r, "Nz");
  in.Nt = scalar_u64(r, "Nt");
  const bool three_d = in.Nz > 1;
  in.dx = scalar_f(r, "dx");
  in.dy = scalar_f(r, "dy");
  in.dz = three_d ? scalar_f(r, "dz") : 0.f;
  in.dt = scalar_f(r, "dt");
  in.c_ref = scalar_f(r, "c_ref");
  in.pml_x_size = scalar_u64(r, "pml_x_size");
  in.pml_y_size = scalar_u64(r, "pml_y_size");
  in.pml_z_size = opt_u64(r, "pml_z_size", 0);
  in.pml_x_alpha = scalar_f(r, "pml_x_alpha");
  in.pml_y_alpha = scalar_f(r, "pml_y_alpha");
  in.pml_z_alpha = three_d ? scalar_f(r, "pml_z_alpha") : 0.f;
  in.c0 = field(F, r, "c0");
  in.rho0 = field(F, r, "rho0");
  in.rho0_sgx = field(F, r, "rho0_sgx");
  in.rho0_sgy = field(F, r, "rho0_sgy");
  if (three_d) in.rho0_sgz = field(F, r, "rho0_sgz");
  in.nonlinear_flag = opt_u64(r, "nonlinear_flag", 0);
  if (in.nonlinear_flag) in.BonA = field(F, r, "BonA");
  in.absorbing_flag = opt_u64(r, "absorbing_flag", 0);
  if (in.absorbing_flag) {
    in.alpha_coeff = field(F, r, "alpha_coeff");
    if (in.absorbing_flag == 1) in.alpha_power = scalar_f(r, "alpha_power");
    else in.alpha_power = r.exists("/alpha_power") ? scalar_f(r, "alpha_power") : 2.f;
  }
  in.p0_source_flag = opt_u64(r, "p0_source_flag", 0);
  if (in.p0_source_flag) {
    need(r, "p0_source_input");
    in.p0_source_input = F.keep_f(r.read_float("/p0_source_input"));
  }
  in.p_source_flag = opt_u64(r, "p_source_flag", 0);
  if (in.p_source_flag) {
    for (const char* n : {"p_source_mode", "p_source_many", "p_source_index", "p_source_input"}) need(r, n);
    in.p_source_mode = scalar_u64(r, "p_source_mode");
    in.p_source_many = scalar_u64(r, "p_source_many");
    auto idx = r.read_u64("/p_source_index");
    in.p_source_index_numel = idx.size();
    in.p_source_index = F.keep_u(std::move(idx));
    auto sig = r.read_float("/p_source_input");
    const uint64_t rows = in.p_source_many ? in.p_source_index_numel : 1;
    if (sig.size() < rows * in.p_source_flag) throw IoError(KW_ERR_IO, "p_source_input is shorter than its flag");
    in.p_source_input = F.keep_f(std::move(sig));
  }
  in.ux_source_flag = opt_u64(r, "ux_source_flag", 0);
  in.uy_source_flag = opt_u64(r, "uy_source_flag", 0);
  in.uz_source_flag = three_d ? opt_u64(r, "uz_source_flag", 0) : 0;
  if (in.ux_source_flag || in.uy_source_flag || in.uz_source_flag) {
    for (const char* n : {"u_source_mode", "u_source_many", "u_source_index"}) need(r, n);
    in.u_source_mode = scalar_u64(r, "u_source_mode");
    in.u_source_many = scalar_u64(r, "u_source_many");
    auto idx = r.read_u64("/u_source_index");
    in.u_source_index_numel = idx.size();
    in.u_source_index = F.keep_u(std::move(idx));
    if (in.ux_source_flag) { need(r, "ux_source_input"); in.ux_source_input = F.keep_f(r.read_float("/ux_source_input")); }
    if (in.uy_source_flag) { need(r, "uy_source_input"); in.uy_source_input = F.keep_f(r.read_float("/uy_source_input")); }
    if (in.uz_source_flag) { need(r, "uz_source_input"); in.uz_source_input = F.keep_f(r.read_float("/uz_source_input")); }
  }
  in.axisymmetric_flag = opt_u64(r, "axisymmetric_flag", 0);
  in.transducer_source_flag = opt_u64(r, "transducer_source_flag", 0);
  if (in.transducer_source_flag) {
    for (const char* n : {"u_source_index", "delay_mask", "transducer_source_input"}) need(r, n);
    if (!in.u_source_index) {
      auto idx = r.read_u64("/u_source_index");
      in.u_source_index_numel = idx.size();
      in.u_source_index = F.keep_u(std::move(idx));
    }
    auto dm = r.read_u64("/delay_mask");
    if (dm.size() != in.u_source_index_numel)
      throw IoError(KW_ERR_IO, "delay_mask must hold one entry per u_source_index entry");
    in.delay_mask = F.keep_u(std::move(dm));
    auto sig = r.read_float("/transducer_source_input");
    in.transducer_source_input_numel = sig.size();
    in.transducer_source_input = F.keep_f(std::move(sig));
  }
  in.sensor_mask_type = scalar_u64(r, "sensor_mask_type");
  if (in.sensor_mask_type == 0) {
    need(r, "sensor_mask_index");
    auto idx = r.read_u64("/sensor_mask_index");
    in.sensor_mask_index_numel = idx.size();
    in.sensor_mask_index = F.keep_u(std::move(idx));
  } else {
    need(r, "sensor_mask_corners");
    auto c = r.read_u64("/sensor_mask_corners");
    if (c.empty() || c.size() % 6) throw IoError(KW_ERR_IO, "sensor_mask_corners must hold 6 values per cuboid");
    for (size_t k = 0; k < c.size() / 6; ++k)
      for (int a = 0; a < 3; ++a) F.corner_dims.push_back(c[6 * k + 3 + a] >= c[6 * k + a] ? c[6 * k + 3 + a] - c[6 * k + a] + 1 : 0);
    in.sensor_mask_corners_numel = c.size();
    in.sensor_mask_corners = F.keep_u(std::move(c));
  }
}

// Solve with checkpoints: a resident session advanced in chunks, its state
// written to `ckpt` every `every_steps` steps and / or `every_s` seconds of
// wall time; an existing checkpoint file is resumed from.
void solve_checkpointed(const kw_input& in, const kw_options& opt, kw_output& out, const char* ckpt,
                        uint64_t every_steps, double every_s) {
  kw_session* s = nullptr;
  kw_status e{};
  if (kw_session_create(&in, &opt, &s, &e) != KW_OK) throw IoError(e.code, e.message);
  struct Guard {
    kw_session* s;
    ~Guard() { kw_session_destroy(s); }
  } guard{s};
  if (FILE* f = std::fopen(ckpt, "rb")) {
    std::fclose(f);
    if (kw_session_restore(s, ckpt, &e) != KW_OK) throw IoError(e.code, e.message);
  }
  const uint64_t chunk = every_steps ? every_steps : 50;
  uint64_t done = kw_session_steps_done(s), since = 0;
  auto last = std::chrono::steady_clock::now();
  while (done < in.Nt) {
    const uint64_t n = std::min<uint64_t>(chunk - since % chunk, in.Nt - done);
    if (kw_session_advance(s, n, &e) != KW_OK || kw_session_sync(s, &e) != KW_OK) throw IoError(e.code, e.message);
    done += n;
    since += n;
    const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - last).count();
    const bool due = (every_steps && since >= every_steps) || (every_s > 0 && el >= every_s);
    if (due && done < in.Nt) {
      if (kw_session_save(s, ckpt, &e) != KW_OK) throw IoError(e.code, e.message);
      since = 0;
      last = std::chrono::steady_clock::now();
    }
  }
  if (kw_session_read(s, &out, &e) != KW_OK) throw IoError(e.code, e.message);
}

std::string now_string() {
  char buf[64];
  std::time_t t = std::time(nullptr);
  std::strftime(buf, sizeof(buf), "%d-%b-%Y-%H-%M-%S", std::localtime(&t));
  return buf;
}

}  // namespace

static int run_file(const char* input_h5, const char* output_h5, const kw_options* opt_in, const char* ckpt,
                    uint64_t ckpt_steps, double ckpt_s, kw_status* st) {
  try {
    if (!input_h5 || !output_h5 || !opt_in) throw IoError(KW_ERR_INVALID_ARGUMENT, "NULL argument");
    kw_options opt = *opt_in;
    InputFile F;
    try {
      read_input(input_h5, F);
    } catch (const h5::Error& e) {
      throw IoError(KW_ERR_IO, std::string(input_h5) + ": " + e.what());
    }
    kw_output_sizes sz;
    kw_status s2{};
    if (kw_output_sizes_query(&F.in, &opt, &sz, &s2) != KW_OK) throw IoError(s2.code, s2.message);
    const uint64_t ns = sz.num_sensor_points, nr = sz.num_recorded_steps, ng = sz.grid_points;
    const bool three_d = F.in.Nz > 1;
    const int dim = three_d ? 3 : 2;
    // host buffers for the requested outputs
    std::vector<std::vector<float>> store;
    kw_output out{};
    auto buf = [&](float** slot, uint64_t n) {
      store.emplace_back(n);
      *slot = store.back().data();
    };
    store.reserve(40);
    if (opt.p_raw) buf(&out.p, ns * nr);
    if (opt.p_max) buf(&out.p_max, ns);
    if (opt.p_min) buf(&out.p_min, ns);
    if (opt.p_rms) buf(&out.p_rms, ns);
    if (opt.p_max_all) buf(&out.p_max_all, ng);
    if (opt.p_min_all) buf(&out.p_min_all, ng);
    if (opt.p_final) buf(&out.p_final, ng);
    float** u_raw[3] = {&out.ux, &out.uy, &out.uz};
    float** u_max[3] = {&out.ux_max, &out.uy_max, &out.uz_max};
    float** u_min[3] = {&out.ux_min, &out.uy_min, &out.uz_min};
    float** u_rms[3] = {&out.ux_rms, &out.uy_rms, &out.uz_rms};
    float** u_mxa[3] = {&out.ux_max_all, &out.uy_max_all, &out.uz_max_all};
    float** u_mna[3] = {&out.ux_min_all, &out.uy_min_all, &out.uz_min_all};
    float** u_fin[3] = {&out.ux_final, &out.uy_final, &out.uz_final};
    float** u_nst[3] = {&out.ux_non_staggered, &out.uy_non_staggered, &out.uz_non_staggered};
    for (int a = 0; a < dim; ++a) {
      if (opt.u_raw) buf(u_raw[a], ns * nr);
      if (opt.u_max) buf(u_max[a], ns);
      if (opt.u_min) buf(u_min[a], ns);
      if (opt.u_rms) buf(u_rms[a], ns);
      if (opt.u_max_all) buf(u_mxa[a], ng);
      if (opt.u_min_all) buf(u_mna[a], ng);
      if (opt.u_final) buf(u_fin[a], ng);
      if (opt.u_non_staggered_raw) buf(u_nst[a], ns * nr);
    }
    if (ckpt) {
      solve_checkpointed(F.in, opt, out, ckpt, ckpt_steps, ckpt_s);
    } else {
      kw_status s3{};
      if (kw_solve(&F.in, &opt, &out, &s3) != KW_OK) throw IoError(s3.code, s3.message);
    }

    // output file (kspaceFirstOrder3DC.m:569-776)
    h5::Writer w;
    const std::map<std::string, std::string> fa = {{"data_type", "float"}, {"domain_type", "real"}};
    const std::map<std::string, std::string> la = {{"data_type", "long"}, {"domain_type", "real"}};
    const std::vector<uint64_t> one = {1, 1, 1};
    std::vector<uint64_t> scal;
    scal.reserve(8);
    auto put_u = [&](const char* name, uint64_t v) {
      scal.push_back(v);
      w.dataset(std::string("/") + name, h5::DType::U64, one, &scal.back(), la);
    };
    put_u("Nx", F.in.Nx);
    put_u("Ny", F.in.Ny);
    put_u("Nz", F.in.Nz);
    put_u("Nt", F.in.Nt);
    put_u("pml_x_size", F.in.pml_x_size);
    put_u("pml_y_size", F.in.pml_y_size);
    if (three_d) put_u("pml_z_size", F.in.pml_z_size);
    const std::vector<uint64_t> grid = {F.in.Nz, F.in.Ny, F.in.Nx};
    auto put_grid = [&](const std::string& name, const float* p) {
      if (p) w.dataset("/" + name, h5::DType::F32, grid, p, fa);
    };
    put_grid("p_max_all", out.p_max_all);
    put_grid("p_min_all", out.p_min_all);
    put_grid("p_final", out.p_final);
    const char* comp = "xyz";
    for (int a = 0; a < dim; ++a) {
      const std::string u = std::string("u") + comp[a];
      put_grid(u + "_max_all", *u_mxa[a]);
      put_grid(u + "_min_all", *u_mna[a]);
      put_grid(u + "_final", *u_fin[a]);
    }
    // sensor outputs: one dataset each, or one group per output with a
    // dataset per cuboid
    struct SensorOut {
      std::string name;
      const float* p;
      bool series;
    };
    std::vector<SensorOut> so = {{"p", out.p, true}, {"p_max", out.p_max, false}, {"p_min", out.p_min, false},
                                 {"p_rms", out.p_rms, false}};
    for (int a = 0; a < dim; ++a) {
      const std::string u = std::string("u") + comp[a];
      so.push_back({u, *u_raw[a], true});
      so.push_back({u + "_max", *u_max[a], false});
      so.push_back({u + "_min", *u_min[a], false});
      so.push_back({u + "_rms", *u_rms[a], false});
      so.push_back({u + "_non_staggered", *u_nst[a], true});
    }
    std::vector<std::vector<float>> cub;  // per-cuboid copies of time series
    cub.reserve(so.size() * (F.corner_dims.size() / 3 + 1));
    for (const SensorOut& s : so) {
      if (!s.p) continue;
      if (F.in.sensor_mask_type == 0) {
        if (s.series)
          w.dataset("/" + s.name, h5::DType::F32, {1, nr, ns}, s.p, fa);
        else
          w.dataset("/" + s.name, h5::DType::F32, {1, 1, ns}, s.p, fa);
        continue;
      }
      // cuboids: [x, y, z, t] in MATLAB order (kspaceFirstOrder_reorderCuboidCorners.m)
      uint64_t start = 0;
      for (size_t k = 0; k < F.corner_dims.size() / 3; ++k) {
        const uint64_t cx = F.corner_dims[3 * k], cy = F.corner_dims[3 * k + 1], cz = F.corner_dims[3 * k + 2];
        const uint64_t n = cx * cy * cz;
        const std::string path = "/" + s.name + "/" + std::to_string(k + 1);
        if (s.series) {
          cub.emplace_back(n * nr);
          for (uint64_t t = 0; t < nr; ++t)
            std::memcpy(cub.back().data() + t * n, s.p + t * ns + start, n * sizeof(float));
          if (three_d)
            w.dataset(path, h5::DType::F32, {nr, cz, cy, cx}, cub.back().data(), fa);
          else
            w.dataset(path, h5::DType::F32, {nr, cy, cx}, cub.back().data(), fa);
        } else {
          if (three_d)
            w.dataset(path, h5::DType::F32, {cz, cy, cx}, s.p + start, fa);
          else
            w.dataset(path, h5::DType::F32, {cy, cx}, s.p + start, fa);
        }
        start += n;
      }
    }
    w.root_attribute("created_by", kw_version());
    w.root_attribute("creation_date", now_string());
    w.root_attribute("file_description", std::string("Output of ") + input_h5);
    w.root_attribute("file_type", "output");
    w.root_attribute("major_version", "1");
    w.root_attribute("minor_version", "2");
    try {
      w.write(output_h5);
    } catch (const h5::Error& e) {
      throw IoError(KW_ERR_IO, e.what());
    }
    if (ckpt) std::remove(ckpt);  // the run is complete: the checkpoint is spent
    return set_status(st, KW_OK, "");
  } catch (const IoError& e) {
    return set_status(st, e.code, e.what());
  } catch (const std::bad_alloc&) {
    return set_status(st, KW_ERR_OUT_OF_MEMORY, "host allocation failed");
  } catch (const std::exception& e) {
    return set_status(st, KW_ERR_INTERNAL, e.what());
  }
}

extern "C" int kw_run_file(const char* input_h5, const char* output_h5, const kw_options* opt, kw_status* st) {
  return run_file(input_h5, output_h5, opt, nullptr, 0, 0.0, st);
}

extern "C" int kw_run_file_checkpointed(const char* input_h5, const char* output_h5, const kw_options* opt,
                                        const char* checkpoint_file, uint64_t checkpoint_timesteps,
                                        double checkpoint_interval_s, kw_status* st) {
  if (!checkpoint_file || (!checkpoint_timesteps && !(checkpoint_interval_s > 0)))
    return set_status(st, KW_ERR_INVALID_ARGUMENT, "a checkpoint file and an interval (steps or seconds) are needed");
  return run_file(input_h5, output_h5, opt, checkpoint_file, checkpoint_timesteps, checkpoint_interval_s, st);
}

// kspaceFirstOrder-B200 -i in.h5 -o out.h5 [--p_raw] [--p_max] ... [-s N] [-g N]
extern "C" int kw_cli_main(int argc, char** argv) {
  kw_options opt{};
  opt.device = -1;
  std::string in, out, ckpt;
  uint64_t ckpt_steps = 0;
  double ckpt_s = 0.0;
  bool any = false;
  struct Flag {
    const char* name;
    int* slot;
  } flags[] = {{"--p_raw", &opt.p_raw},         {"--p_max", &opt.p_max},         {"--p_min", &opt.p_min},
               {"--p_rms", &opt.p_rms},         {"--p_max_all", &opt.p_max_all}, {"--p_min_all", &opt.p_min_all},
               {"--p_final", &opt.p_final},     {"--u_raw", &opt.u_raw},         {"--u_max", &opt.u_max},
               {"--u_min", &opt.u_min},         {"--u_rms", &opt.u_rms},         {"--u_max_all", &opt.u_max_all},
               {"--u_min_all", &opt.u_min_all}, {"--u_final", &opt.u_final},
               {"--u_non_staggered_raw", &opt.u_non_staggered_raw}};
  const char* prog = argc > 0 ? argv[0] : "kspaceFirstOrder-B200";
  auto usage = [&]() {
    std::fprintf(stderr,
                 "usage: %s -i <input.h5> -o <output.h5> [--p_raw --p_max --p_min --p_rms --p_max_all --p_min_all "
                 "--p_final --u_raw --u_max --u_min --u_rms --u_max_all --u_min_all --u_final "
                 "--u_non_staggered_raw] [-s <start index>] [-g <device>] [-t <threads>] [--verbose <0-2>] "
                 "[--checkpoint_file <file> --checkpoint_timesteps <n> | --checkpoint_interval <seconds>]\n",
                 prog);
    return 2;
  };
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    auto value = [&]() -> const char* {
      if (i + 1 >= argc) return nullptr;
      return argv[++i];
    };
    bool matched = false;
    for (auto& f : flags)
      if (a == f.name) {
        *f.slot = 1;
        any = true;
        matched = true;
      }
    if (matched) continue;
    if (a == "-i") {
      const char* v = value();
      if (!v) return usage();
      in = v;
    } else if (a == "-o") {
      const char* v = value();
      if (!v) return usage();
      out = v;
    } else if (a == "-s") {
      const char* v = value();
      if (!v) return usage();
      opt.start_index = std::strtoull(v, nullptr, 10);
    } else if (a == "-g") {
      const char* v = value();
      if (!v) return usage();
      opt.device = std::atoi(v);
    } else if (a == "--verbose") {
      const char* v = value();
      if (!v) return usage();
      opt.verbose = std::atoi(v);
    } else if (a == "--checkpoint_file") {
      const char* v = value();
      if (!v) return usage();
      ckpt = v;
    } else if (a == "--checkpoint_timesteps") {
      const char* v = value();
      if (!v) return usage();
      ckpt_steps = std::strtoull(v, nullptr, 10);
    } else if (a == "--checkpoint_interval") {
      const char* v = value();
      if (!v) return usage();
      ckpt_s = std::atof(v);
    } else if (a == "-t" || a == "-c" || a == "--benchmark") {
      if (!value()) return usage();  // host threads / compression level: not used by the GPU solver
    } else if (a == "-h" || a == "--help") {
      usage();
      return 0;
    } else {
      std::fprintf(stderr, "%s: unknown option %s\n", prog, a.c_str());
      return usage();
    }
  }
  if (in.empty() || out.empty()) return usage();
  if (!any) opt.p_raw = 1;  // the binaries record p when no output is named
  kw_status st{};
  if (opt.verbose) std::printf("%s: %s -> %s\n", kw_version(), in.c_str(), out.c_str());
  if (!ckpt.empty() && !ckpt_steps && !(ckpt_s > 0)) {
    std::fprintf(stderr, "%s: --checkpoint_file needs --checkpoint_timesteps or --checkpoint_interval\n", prog);
    return usage();
  }
  const int rc = ckpt.empty() ? kw_run_file(in.c_str(), out.c_str(), &opt, &st)
                              : kw_run_file_checkpointed(in.c_str(), out.c_str(), &opt, ckpt.c_str(), ckpt_steps,
                                                         ckpt_s, &st);
  if (rc != KW_OK) {
    std::fprintf(stderr, "%s: error %d: %s\n", prog, rc, st.message);
    return 1;
  }
  if (opt.verbose) std::printf("%s: done\n", prog);
  return 0;
}
