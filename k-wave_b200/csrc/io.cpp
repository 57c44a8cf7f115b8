// File-based drop-in: HDF5 input -> solve -> HDF5 output, and the CLI.
#include <cstdio>
#include <cstring>
#include <string>

#include "kwave_b200.h"

extern "C" int kw_run_file(const char* input_h5, const char* output_h5, const kw_options* opt, kw_status* st) {
  (void)input_h5; (void)output_h5; (void)opt;
  if (st) {
    st->code = KW_ERR_UNSUPPORTED;
    std::snprintf(st->message, sizeof(st->message), "HDF5 I/O not built");
  }
  return KW_ERR_UNSUPPORTED;
}

extern "C" int kw_cli_main(int argc, char** argv) {
  (void)argc; (void)argv;
  return 1;
}
