// Internal host-side declarations shared by the opgpu translation units.
#pragma once
#include <stdint.h>
#include <string>
#include <vector>

namespace opgpu {

bool raw_read(const char* path, int nx, int ny, int nz, std::vector<int32_t>& counts,
              std::vector<int32_t>& idx, std::vector<double>& val, std::string& err);
bool raw_write(const char* path, int nx, int ny, int nz, const int32_t* counts, const int32_t* idx,
               const double* val, std::string& err);

}  // namespace opgpu
