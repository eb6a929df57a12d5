// `fip` command line: the reference's headless main() (src/main.cpp:204-263) on the C ABI.
//   fip parameters.yml
// Loads the parameter file, prints the sampling header and rows to stdout, runs until the
// target duration, writes the save_state dumps and reports the run time on stderr.
#include <cuda_runtime.h>

#include <chrono>
#include <cstdlib>
#include <iostream>
#include <string>

#include "fip.h"

int main(int argc, char** argv) {
  std::string sim_file = "inde.yml";
  if (argc < 2)
    std::cerr << "Warning: no config file given, using default " << sim_file << std::endl;
  else
    sim_file = argv[1];

  fip_handle* h = nullptr;
  int rc = fip_init(sim_file.c_str(), &h);
  if (rc != FIP_OK) {
    std::cerr << "Config error: " << fip_last_error() << std::endl;
    return EXIT_FAILURE;
  }
  const auto t0 = std::chrono::steady_clock::now();
  rc = fip_run(h);
  const auto t1 = std::chrono::steady_clock::now();
  if (rc != FIP_OK) {
    std::cerr << "Error: " << fip_last_error() << std::endl;
    fip_destroy(h);
    return EXIT_FAILURE;
  }
  double duration = 0;
  float dt = 0;
  int iteration = 0;
  fip_time(h, &duration, &dt, &iteration);
  const float seconds = std::chrono::duration<float>(t1 - t0).count();
  std::cerr << std::dec << "Finished " << iteration << " iterations after " << seconds << " s (" << std::fixed
            << seconds / iteration << " s/it)" << std::endl;
  fip_destroy(h);
  return 0;
}
