// Binary Tecplot V112 flow-field file, as the reference writes it through
// MPI-IO (src/MPIIO.hpp:59-546) and reads it back on restart
// (src/Initialize.cuh:57-276).  One ordered zone per block, FP64 data,
// interior points only (the reference builds its writer with 0 ghost layers).
#pragma once

#include <string>
#include <vector>

#include "boundary.hpp"

namespace ostc {

struct PltBlockData {
  const Block *block = nullptr;
  const HostField *field = nullptr;   // bv, sv with ngg ghosts
  const std::vector<double> *mach = nullptr;  // ghosted layout
  const std::vector<double> *mut = nullptr;   // ghosted layout, RANS only
};

// Variable names in file order: x y z density u v w pressure temperature mach,
// species by index, tke omega (SST), mut (RANS).
std::vector<std::string> plt_variable_names(const Species &spec, bool rans);

void write_plt(const std::string &path, const std::vector<PltBlockData> &blocks, const Species &spec, bool rans);

// Restart: fills interior bv / sv of `field` by variable name.  Species or
// turbulence variables missing from the file are initialised from the
// default inflow, as the reference does.  Returns false if the file is absent.
bool read_plt_restart(const std::string &path, const Mesh &mesh, const Species &spec, Parameter &parameter,
                      std::vector<HostField> &field);

}  // namespace ostc
