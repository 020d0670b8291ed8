// ncwrite.cpp -- a small writer of NetCDF classic files (the 64-bit offset
// variant, "CDF\x02"), enough for the solver's outputs: fixed and record
// (unlimited) dimensions, global text attributes, int and float variables.
//
// The reference writes its seismograms, snapshots and peak velocities with
// libnetcdf in NetCDF-4 (HDF5) files (src/seisnc.cpp:1229-1364, 1671-1757);
// the same variables in the classic format are readable by every netCDF
// library (and by scipy.io.netcdf_file).  Layout, from the published format
// specification: big-endian header (magic, record count, dimension list,
// global attribute list, variable list with each variable's dimension ids,
// attributes, type, padded size and file offset), then the non-record
// variables in order, then the records, each holding one slab of every record
// variable in order.
#include "ncwrite.h"

#include <cstdint>
#include <cstdio>
#include <cstring>

namespace cgfd {
namespace nc {
namespace {

constexpr uint32_t NC_DIMENSION = 10, NC_VARIABLE = 11, NC_ATTRIBUTE = 12;

struct Buf {
  std::vector<unsigned char> b;
  void u32(uint32_t v) {
    for (int s = 24; s >= 0; s -= 8) b.push_back((unsigned char)(v >> s));
  }
  void u64(uint64_t v) {
    for (int s = 56; s >= 0; s -= 8) b.push_back((unsigned char)(v >> s));
  }
  void pad4() {
    while (b.size() % 4) b.push_back(0);
  }
  void name(const std::string &s) {
    u32((uint32_t)s.size());
    b.insert(b.end(), s.begin(), s.end());
    pad4();
  }
};

size_t type_size(int t) { return t == NC_INT || t == NC_FLOAT ? 4 : 1; }

}  // namespace

bool write_classic(const char *path, const std::vector<Dim> &dims,
                   const std::vector<std::pair<std::string, std::string>> &gatts,
                   const std::vector<Var> &vars, size_t numrecs) {
  auto is_rec = [&](const Var &v) { return !v.dims.empty() && dims[v.dims[0]].len == 0; };
  // bytes of one variable (per record for record variables), padded to 4
  auto vsize = [&](const Var &v) {
    size_t n = type_size(v.type);
    for (size_t q = is_rec(v) ? 1 : 0; q < v.dims.size(); ++q) n *= dims[v.dims[q]].len;
    return (n + 3) / 4 * 4;
  };
  // header with placeholder offsets, then again with the real ones
  std::vector<uint64_t> begin(vars.size(), 0);
  Buf h;
  for (int pass = 0; pass < 2; ++pass) {
    h.b.clear();
    h.b.insert(h.b.end(), {'C', 'D', 'F', 2});
    h.u32((uint32_t)numrecs);
    if (dims.empty()) { h.u32(0); h.u32(0); }
    else {
      h.u32(NC_DIMENSION);
      h.u32((uint32_t)dims.size());
      for (const Dim &d : dims) { h.name(d.name); h.u32((uint32_t)d.len); }
    }
    if (gatts.empty()) { h.u32(0); h.u32(0); }
    else {
      h.u32(NC_ATTRIBUTE);
      h.u32((uint32_t)gatts.size());
      for (const auto &a : gatts) {
        h.name(a.first);
        h.u32(NC_CHAR);
        h.u32((uint32_t)a.second.size());
        h.b.insert(h.b.end(), a.second.begin(), a.second.end());
        h.pad4();
      }
    }
    if (vars.empty()) { h.u32(0); h.u32(0); }
    else {
      h.u32(NC_VARIABLE);
      h.u32((uint32_t)vars.size());
      for (size_t q = 0; q < vars.size(); ++q) {
        const Var &v = vars[q];
        h.name(v.name);
        h.u32((uint32_t)v.dims.size());
        for (int d : v.dims) h.u32((uint32_t)d);
        h.u32(0); h.u32(0);  // no variable attributes
        h.u32((uint32_t)v.type);
        h.u32((uint32_t)vsize(v));
        h.u64(begin[q]);
      }
    }
    // offsets: non-record variables after the header, then the records
    uint64_t off = h.b.size();
    for (size_t q = 0; q < vars.size(); ++q)
      if (!is_rec(vars[q])) { begin[q] = off; off += vsize(vars[q]); }
    for (size_t q = 0; q < vars.size(); ++q)
      if (is_rec(vars[q])) { begin[q] = off; off += vsize(vars[q]); }
  }
  FILE *f = std::fopen(path, "wb");
  if (!f) return false;
  bool ok = std::fwrite(h.b.data(), 1, h.b.size(), f) == h.b.size();
  // values big-endian, each variable padded to 4 bytes
  auto put = [&](const Var &v, size_t first, size_t count) {
    std::vector<unsigned char> o(count * 4);
    const uint32_t *src = static_cast<const uint32_t *>(v.data) + first;
    for (size_t q = 0; q < count; ++q) {
      const uint32_t x = src[q];
      o[4 * q] = (unsigned char)(x >> 24); o[4 * q + 1] = (unsigned char)(x >> 16);
      o[4 * q + 2] = (unsigned char)(x >> 8); o[4 * q + 3] = (unsigned char)x;
    }
    ok = ok && std::fwrite(o.data(), 1, o.size(), f) == o.size();
  };
  auto slab = [&](const Var &v) {
    size_t n = 1;
    for (size_t q = is_rec(v) ? 1 : 0; q < v.dims.size(); ++q) n *= dims[v.dims[q]].len;
    return n;
  };
  for (const Var &v : vars)
    if (!is_rec(v)) put(v, 0, slab(v));
  for (size_t r = 0; r < numrecs; ++r)
    for (const Var &v : vars)
      if (is_rec(v)) put(v, r * slab(v), slab(v));
  ok = (std::fclose(f) == 0) && ok;
  return ok;
}

}  // namespace nc
}  // namespace cgfd
