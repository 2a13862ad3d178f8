// lu_mustard: tiled no-pivot LU on one B200 (replaces mustard/lu_mustard.cu:682-716).
#include "cli_common.hpp"

int main(int argc, char **argv) { return mtdcli::run_main(argc, argv, MTD_KIND_LU, "LU"); }
