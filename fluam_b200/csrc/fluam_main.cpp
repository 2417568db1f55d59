// fluam_main.cpp -- the `fluam` executable of this build: `fluam [data.main]`.
// Mirrors src/main.cpp:28-112 for the stokesLimit scheme, including its exit
// status (1 when the run completed, 0 otherwise).
#include "../../include/fluamsl.h"

int main(int argc, char* argv[]) {
  const char* path = argc > 1 ? argv[1] : "data.main";  // src/loadDataMain.cu:304-309
  return fsl_run_data_main(path) == FSL_OK ? 1 : 0;
}
