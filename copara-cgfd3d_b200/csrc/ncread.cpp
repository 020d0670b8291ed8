// ncread.cpp -- a small reader of NetCDF classic files (CDF-1 "CDF\x01",
// 64-bit offset "CDF\x02" and 64-bit data "CDF\x05"), enough for the
// reference's model inputs: dimension lengths, numeric global attributes and
// whole numeric variables (fixed or record), converted to double.
//
// The reference reads its volume media (Vsim_gpu.nc: x, y, depth, Vp, Vs,
// rho; src/mediaparas.cpp:1273-1425) and its finite-fault series
// (stf-GPU.nc: dimensions NP, NT, attribute DT, Mxx..Myz [NP][NT], posx,
// posy, posz; src/source.cpp:43-56, 796-840) with libnetcdf.  Its example
// files are NetCDF-4 (HDF5); `nccopy -k classic` (or -k 64-bit-offset)
// converts them to this format, which this image can read without HDF5.
// Layout, from the published format specification: big-endian header
// (magic, record count, dimension list, global attribute list, variable
// list: name, dimension ids, attributes, type, padded size, file offset),
// then the non-record variables, then the records (one slab of every record
// variable each).
#include "ncread.h"

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>

namespace cgfd {
namespace nc {
namespace {

enum { T_BYTE = 1, T_CHAR = 2, T_SHORT = 3, T_INT = 4, T_FLOAT = 5, T_DOUBLE = 6,
       T_UBYTE = 7, T_USHORT = 8, T_UINT = 9, T_INT64 = 10, T_UINT64 = 11 };
constexpr uint32_t NC_DIMENSION = 10, NC_VARIABLE = 11, NC_ATTRIBUTE = 12;

size_t type_size(int t) {
  switch (t) {
    case T_BYTE: case T_CHAR: case T_UBYTE: return 1;
    case T_SHORT: case T_USHORT: return 2;
    case T_INT: case T_FLOAT: case T_UINT: return 4;
    case T_DOUBLE: case T_INT64: case T_UINT64: return 8;
    default: return 0;
  }
}

// one big-endian value of type t at p, as double
double value_at(const unsigned char *p, int t) {
  uint64_t u = 0;
  const size_t n = type_size(t);
  for (size_t q = 0; q < n; ++q) u = (u << 8) | p[q];
  switch (t) {
    case T_BYTE: return (double)(int8_t)u;
    case T_CHAR: case T_UBYTE: return (double)(uint8_t)u;
    case T_SHORT: return (double)(int16_t)u;
    case T_USHORT: return (double)(uint16_t)u;
    case T_INT: return (double)(int32_t)u;
    case T_UINT: return (double)(uint32_t)u;
    case T_INT64: return (double)(int64_t)u;
    case T_UINT64: return (double)u;
    case T_FLOAT: { uint32_t w = (uint32_t)u; float f; std::memcpy(&f, &w, 4); return f; }
    case T_DOUBLE: { double d; std::memcpy(&d, &u, 8); return d; }
    default: return 0.0;
  }
}

struct Reader {
  FILE *f = nullptr;
  int version = 0;
  std::string err;
  bool ok = true;
  ~Reader() { if (f) std::fclose(f); }
  uint64_t be(int n) {
    unsigned char b[8];
    if (ok && std::fread(b, 1, (size_t)n, f) != (size_t)n) { ok = false; err = "truncated header"; }
    uint64_t u = 0;
    for (int q = 0; q < n && ok; ++q) u = (u << 8) | b[q];
    return ok ? u : 0;
  }
  uint64_t count() { return be(version == 5 ? 8 : 4); }      // NON_NEG
  uint64_t offset() { return be(version == 1 ? 4 : 8); }     // OFFSET
  std::string name() {
    const uint64_t n = count();
    if (!ok || n > 4096) { ok = false; err = "bad name"; return {}; }
    std::string s(n, '\0');
    if (n && std::fread(&s[0], 1, n, f) != n) { ok = false; err = "truncated name"; }
    skip_pad(n);
    return s;
  }
  void skip_pad(uint64_t n) {
    const uint64_t p = (4 - n % 4) % 4;
    if (p) std::fseek(f, (long)p, SEEK_CUR);
  }
  // an attribute list; numeric attributes are kept as doubles
  void atts(std::map<std::string, std::vector<double>> *out) {
    const uint64_t tag = be(4), n = count();
    if (!ok) return;
    if (tag == 0 && n == 0) return;
    if (tag != NC_ATTRIBUTE) { ok = false; err = "bad attribute list"; return; }
    for (uint64_t a = 0; a < n && ok; ++a) {
      const std::string nm = name();
      const int t = (int)be(4);
      const uint64_t m = count();
      const size_t sz = type_size(t);
      if (!ok || sz == 0 || m > (1u << 26)) { ok = false; err = "bad attribute"; return; }
      std::vector<unsigned char> raw(m * sz);
      if (m && std::fread(raw.data(), 1, raw.size(), f) != raw.size()) {
        ok = false; err = "truncated attribute"; return;
      }
      skip_pad(m * sz);
      if (out && t != T_CHAR) {
        std::vector<double> v(m);
        for (uint64_t q = 0; q < m; ++q) v[q] = value_at(raw.data() + q * sz, t);
        (*out)[nm] = v;
      }
    }
  }
};

}  // namespace

bool File::open(const char *path) {
  *this = File();
  Reader r;
  r.f = std::fopen(path, "rb");
  if (!r.f) { err = std::string("cannot open ") + path; return false; }
  char magic[4];
  if (std::fread(magic, 1, 4, r.f) != 4 || std::memcmp(magic, "CDF", 3) != 0 ||
      (magic[3] != 1 && magic[3] != 2 && magic[3] != 5)) {
    err = std::string(path) + ": not a NetCDF classic file (NetCDF-4/HDF5 files need "
                              "`nccopy -k classic` first)";
    return false;
  }
  r.version = magic[3];
  if (fseeko(r.f, 0, SEEK_END) != 0) { err = std::string(path) + ": cannot seek"; return false; }
  fsize = (uint64_t)ftello(r.f);
  fseeko(r.f, 4, SEEK_SET);
  numrecs = r.count();
  // dimensions
  uint64_t tag = r.be(4), n = r.count();
  if (r.ok && !(tag == 0 && n == 0)) {
    if (tag != NC_DIMENSION) { err = "bad dimension list"; return false; }
    for (uint64_t q = 0; q < n && r.ok; ++q) {
      Dim d;
      d.name = r.name();
      d.len = r.count();
      dims.push_back(d);
    }
  }
  r.atts(&gatts);
  // variables
  tag = r.be(4);
  n = r.count();
  if (r.ok && !(tag == 0 && n == 0)) {
    if (tag != NC_VARIABLE) { err = "bad variable list"; return false; }
    for (uint64_t q = 0; q < n && r.ok; ++q) {
      Var v;
      v.name = r.name();
      const uint64_t nd = r.count();
      if (!r.ok || nd > 64) { err = "bad variable rank"; return false; }
      for (uint64_t d = 0; d < nd; ++d) {
        const uint64_t id = r.count();
        if (id >= dims.size()) { err = "bad dimension id"; return false; }
        v.dims.push_back((int)id);
      }
      r.atts(nullptr);
      v.type = (int)r.be(4);
      v.vsize = r.count();
      v.begin = r.offset();
      if (type_size(v.type) == 0) { err = v.name + ": unsupported type"; return false; }
      vars.push_back(v);
    }
  }
  if (!r.ok) { err = r.err; return false; }
  // record layout: one slab of every record variable per record
  recsize = 0;
  int nrecvars = 0;
  for (const Var &v : vars)
    if (is_record(v)) { recsize += v.vsize; ++nrecvars; }
  // a single record variable is not padded between records
  if (nrecvars == 1)
    for (const Var &v : vars)
      if (is_record(v)) {
        size_t per = type_size(v.type);
        for (size_t d = 1; d < v.dims.size(); ++d) per *= dims[v.dims[d]].len;
        recsize = per;
      }
  this->path = path;
  return true;
}

bool File::is_record(const Var &v) const {
  return !v.dims.empty() && dims[v.dims[0]].len == 0;
}

const File::Var *File::var(const std::string &name) const {
  for (const Var &v : vars)
    if (v.name == name) return &v;
  return nullptr;
}

long long File::dim(const std::string &name) const {
  for (const Dim &d : dims)
    if (d.name == name) return d.len == 0 ? (long long)numrecs : (long long)d.len;
  return -1;
}

bool File::shape(const std::string &name, std::vector<size_t> *out) const {
  const Var *v = var(name);
  if (!v) return false;
  out->clear();
  for (int d : v->dims) out->push_back(dims[d].len == 0 ? numrecs : dims[d].len);
  return true;
}

bool File::read(const std::string &name, std::vector<double> *out) {
  const Var *v = var(name);
  if (!v) { err = path + ": no variable " + name; return false; }
  const uint64_t sz = type_size(v->type);
  // values per record (or in all of a fixed variable), and the extent of the
  // data in the file, checked against the file's size before anything is
  // allocated (a damaged header cannot ask for more memory than the file holds)
  uint64_t per = 1;
  bool bad = false;
  for (size_t d = is_record(*v) ? 1 : 0; d < v->dims.size(); ++d)
    bad |= __builtin_mul_overflow(per, (uint64_t)dims[v->dims[d]].len, &per);
  const uint64_t nrec = is_record(*v) ? numrecs : 1;
  uint64_t bytes = 0, end = 0;
  bad |= __builtin_mul_overflow(per, sz, &bytes);
  bad |= nrec > 1 && recsize < bytes;  // records overlap
  if (!bad && nrec > 0 && per > 0) {
    uint64_t last = 0;
    bad |= __builtin_mul_overflow(nrec - 1, recsize, &last);
    bad |= __builtin_add_overflow(v->begin, last, &end);
    bad |= __builtin_add_overflow(end, bytes, &end);
    bad |= end > fsize;
  }
  if (bad) { err = path + ": data of " + name + " lies outside the file"; return false; }
  std::unique_ptr<FILE, int (*)(FILE *)> f(std::fopen(path.c_str(), "rb"), std::fclose);
  if (!f) { err = "cannot reopen " + path; return false; }
  out->assign(per * nrec, 0.0);
  std::vector<unsigned char> raw(per * sz);
  for (uint64_t r = 0; r < nrec; ++r) {
    const uint64_t off = v->begin + r * recsize;
    if (fseeko(f.get(), (off_t)off, SEEK_SET) != 0 ||
        (per && std::fread(raw.data(), 1, raw.size(), f.get()) != raw.size())) {
      err = path + ": truncated data of " + name;
      return false;
    }
    for (size_t q = 0; q < per; ++q) (*out)[r * per + q] = value_at(raw.data() + q * sz, v->type);
  }
  return true;
}

}  // namespace nc
}  // namespace cgfd
