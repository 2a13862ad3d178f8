// cholesky_mustard: tiled lower Cholesky on one B200 (replaces
// mustard/cholesky_mustard.cu:544-579).
#include "cli_common.hpp"

int main(int argc, char **argv) { return mtdcli::run_main(argc, argv, MTD_KIND_CHOLESKY, "Cholesky"); }
