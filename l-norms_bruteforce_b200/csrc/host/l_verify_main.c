/* The strategy verifier executable: the value of a strategy file's labeling
 * on the matrix as read (no counterpart in the reference). */
#include "../../../include/lnorms_b200.h"

int main(int argc, char **argv) { return ld_verify_main(argc, argv); }
