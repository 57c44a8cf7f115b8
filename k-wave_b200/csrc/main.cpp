// kspaceFirstOrder-B200: command-line drop-in for kspaceFirstOrder-CUDA.
#include "kwave_b200.h"
int main(int argc, char** argv) { return kw_cli_main(argc, argv); }
