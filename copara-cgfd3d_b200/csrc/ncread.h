// ncread.h -- NetCDF classic file reader for the reference's model inputs
// (ncread.cpp).
#pragma once

#include <cstddef>
#include <cstdint>
#include <map>
#include <string>
#include <vector>

namespace cgfd {
namespace nc {

struct File {
  struct Dim {
    std::string name;
    uint64_t len = 0;  // 0: the record (unlimited) dimension
  };
  struct Var {
    std::string name;
    std::vector<int> dims;
    int type = 0;
    uint64_t vsize = 0, begin = 0;
  };
  std::string path, err;
  uint64_t numrecs = 0, recsize = 0;
  uint64_t fsize = 0;  // bytes in the file: every variable's data must lie inside
  std::vector<Dim> dims;
  std::vector<Var> vars;
  std::map<std::string, std::vector<double>> gatts;  // numeric global attributes

  bool open(const char *path);
  // length of a dimension (the record count for the record dimension), -1
  // when absent
  long long dim(const std::string &name) const;
  const Var *var(const std::string &name) const;
  bool is_record(const Var &v) const;
  // the variable's shape (record dimension first for record variables)
  bool shape(const std::string &name, std::vector<size_t> *out) const;
  // the whole variable, row-major, as double
  bool read(const std::string &name, std::vector<double> *out);
};

}  // namespace nc
}  // namespace cgfd
