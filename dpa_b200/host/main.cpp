// main.cpp -- `dpa_pipeline config.json`, the counterpart of the reference's
// `dpa config.json` (source/main.cpp, README.md:18) at world size 1.
#include <iostream>

#include "pipeline.hpp"

int main(int argc, char** argv) {
  if (argc < 2) {
    std::cerr << "usage: dpa_pipeline <config.json>\n";
    return 2;
  }
  return dpa_host::run(argv[1]);
}
