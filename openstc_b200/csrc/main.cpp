// Command-line entry mirroring the reference's main (src/main.cu:7-68): run
// the case in the current directory (or the one given as argv[1]).
#include <cstdio>
#include <exception>
#include <string>

#include "host/driver.hpp"

int main(int argc, char **argv) {
  const std::string dir = argc > 1 ? argv[1] : ".";
  try {
    ostc::DriverOptions opt;
    ostc::Driver driver(dir, opt);
    driver.initialize_computation();
    driver.simulate();
  } catch (const std::exception &e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 1;
  }
  return 0;
}
