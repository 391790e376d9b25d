// `fluxos_gpu <modset.json>`: the FLUXOS-OVERLAND program on the GPU, with
// the command line, inputs and Results/<t>.txt outputs of the reference's
// `fluxos` (main.cpp:70-482).
#include <cstdio>

#include "fluxos_gpu.h"

int main(int argc, char** argv) {
  if (argc < 2) {
    fprintf(stderr, "usage: fluxos_gpu <modset.json>\n");
    return 2;
  }
  int rc = fx_run(argv[1]);
  if (rc != FX_OK) {
    fprintf(stderr, "fluxos_gpu: %s\n", fx_last_error(nullptr));
    return 1;
  }
  return 0;
}
