/* The drop-in executable L_CUDA (L_CUDA.cu:425-439). */
#include "../../../include/lnorms_b200.h"

int main(int argc, char **argv) { return ld_cli_main(argc, argv); }
