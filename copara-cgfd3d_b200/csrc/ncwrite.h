// ncwrite.h -- NetCDF classic (64-bit offset) file writer for the solver's
// outputs (ncwrite.cpp).
#pragma once

#include <cstddef>
#include <string>
#include <utility>
#include <vector>

namespace cgfd {
namespace nc {

enum { NC_CHAR = 2, NC_INT = 4, NC_FLOAT = 5 };

struct Dim {
  std::string name;
  size_t len;  // 0: the record (unlimited) dimension, which must come first
};

// A variable of NC_INT or NC_FLOAT values, row-major over its dimensions;
// a record variable's first dimension is the record dimension and its data
// holds all records.
struct Var {
  std::string name;
  int type;
  std::vector<int> dims;
  const void *data;
};

// writes the file; numrecs = length of the record dimension
bool write_classic(const char *path, const std::vector<Dim> &dims,
                   const std::vector<std::pair<std::string, std::string>> &gatts,
                   const std::vector<Var> &vars, size_t numrecs);

}  // namespace nc
}  // namespace cgfd
