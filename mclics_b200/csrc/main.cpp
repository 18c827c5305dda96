// mclics_b200 <input_file>: the reference program's command line (src/main.cpp:83-125) on the B200 engine.
// Exit status 0 on success, 1 for input errors, 2 for I/O errors, 20 for CUDA errors (the reference's code).
#include <stdio.h>

#include "mclics_b200.h"

int main(int argc, char **argv) {
  printf("============================================================\n");
  printf("  McLics checkerboard Metropolis sweep on B200 (%s)\n", mcl_version());
  printf("============================================================\n\n");
  int rc = mcl_run_input_file(argc > 1 ? argv[1] : "input.txt");
  if (rc != MCL_OK) {
    fprintf(stderr, "  mclics_b200: %s\n", mcl_last_error());
    return rc == MCL_ERR_INPUT ? 1 : (rc == MCL_ERR_IO ? 2 : 20);
  }
  printf("\n  SIMULATION COMPLETE\n");
  return 0;
}
