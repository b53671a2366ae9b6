// lsqt_b200: drop-in for the reference's lsqt_gpu / lsqt_cpu binaries
// (src/main.cu:34-56). Usage: lsqt_b200 input.txt [--fp32 | --fp32r]
// input.txt lists one input directory per line; each is run with lsqt().
#include <chrono>
#include <cstring>
#include <fstream>
#include <iostream>
#include <string>

#include "gpuqt.h"
#include "lsqt/lsqt.h"
#include "lsqt/vector.h"

int main(int argc, char* argv[])
{
  std::cout << "\n***************************************************************\n"
            << "*        LSQT (linear scaling quantum transport), B200        *\n"
            << "***************************************************************\n\n";
  const char* driver = nullptr;
  for (int i = 1; i < argc; ++i) {
    if (std::strcmp(argv[i], "--fp32") == 0)
      Vector::moment_precision = GQT_FP32;
    else if (std::strcmp(argv[i], "--fp32r") == 0)
      Vector::moment_precision = GQT_FP32R;  // needs batch_vectors 4 or 16
    else if (!driver)
      driver = argv[i];
    else
      driver = nullptr, i = argc;
  }
  if (!driver) {
    std::cout << "Usage: lsqt_b200 input.txt [--fp32 | --fp32r]" << std::endl;
    return 1;
  }
  std::ifstream input(driver);
  if (!input.is_open()) {
    std::cout << "Failed to open " << driver << std::endl;
    return 1;
  }
  std::string directory;
  while (std::getline(input, directory)) {
    if (directory.empty())
      continue;
    std::cout << "\n===============================================================\n"
              << "Run LSQT simulation for " << directory << "\n"
              << "===============================================================\n";
    const auto t0 = std::chrono::steady_clock::now();
    lsqt(directory);
    const double s =
      std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::cout << "\n===============================================================\n"
              << "Total time used for " << directory << " = " << s << " s\n"
              << "===============================================================\n";
  }
  return 0;
}
