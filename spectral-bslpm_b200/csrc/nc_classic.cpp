// Writer of netCDF classic files (64-bit offset format, "CDF\x02") for the
// drivers' output: the calls executables/bve_time_evo.cpp:125-358 and
// executables/swe_time_evo.cpp make through the netCDF library (nc_create,
// nc_def_dim, nc_def_var, nc_put_att_*, nc_enddef, nc_put_var*_*, nc_close),
// written from the published classic-format specification, without the
// library: fixed-size dimensions, int and double variables, text / int /
// double attributes, big-endian data.  The reference creates NETCDF4 (HDF5)
// files; the classic format carries the same dimensions, variables and
// attributes and is read by every netCDF reader.
//
// Attributes may be added after sbslpm_nc_enddef (the reference adds its
// global attributes then): enddef reserves room after the header, the header
// is rewritten in place, and a header that outgrows the room is an error.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "internal.hpp"

using sbslpm::set_last_error;

namespace {

constexpr uint32_t kDimTag = 0x0A, kVarTag = 0x0B, kAttTag = 0x0C;
constexpr int kInt = 4, kDouble = 6, kChar = 2;
constexpr long kHeaderSlack = 8192;

struct Att {
  std::string name;
  int type;
  std::vector<unsigned char> be;  // values, big-endian
  long n;
};

struct Var {
  std::string name;
  int type;
  std::vector<int> dims;
  std::vector<Att> atts;
  uint64_t begin = 0, bytes = 0;
};

void put32(std::vector<unsigned char>& b, uint32_t v) {
  for (int s = 24; s >= 0; s -= 8) b.push_back((unsigned char)(v >> s));
}
void put64(std::vector<unsigned char>& b, uint64_t v) {
  for (int s = 56; s >= 0; s -= 8) b.push_back((unsigned char)(v >> s));
}
void pad4(std::vector<unsigned char>& b) {
  while (b.size() % 4) b.push_back(0);
}
void put_name(std::vector<unsigned char>& b, const std::string& s) {
  put32(b, (uint32_t)s.size());
  b.insert(b.end(), s.begin(), s.end());
  pad4(b);
}
void put_atts(std::vector<unsigned char>& b, const std::vector<Att>& atts) {
  if (atts.empty()) {
    put32(b, 0);
    put32(b, 0);
    return;
  }
  put32(b, kAttTag);
  put32(b, (uint32_t)atts.size());
  for (const Att& a : atts) {
    put_name(b, a.name);
    put32(b, (uint32_t)a.type);
    put32(b, (uint32_t)a.n);
    b.insert(b.end(), a.be.begin(), a.be.end());
    pad4(b);
  }
}

int type_size(int t) { return t == kDouble ? 8 : (t == kInt ? 4 : 1); }

}  // namespace

struct sbslpm_nc {
  FILE* f = nullptr;
  bool defining = true;
  std::vector<std::pair<std::string, long>> dims;
  std::vector<Att> gatts;
  std::vector<Var> vars;
  long reserved = 0;  // header bytes reserved at enddef

  std::vector<unsigned char> header() const {
    std::vector<unsigned char> b = {'C', 'D', 'F', 2};
    put32(b, 0);  // numrecs: no record dimension
    if (dims.empty()) {
      put32(b, 0);
      put32(b, 0);
    } else {
      put32(b, kDimTag);
      put32(b, (uint32_t)dims.size());
      for (const auto& d : dims) {
        put_name(b, d.first);
        put32(b, (uint32_t)d.second);
      }
    }
    put_atts(b, gatts);
    if (vars.empty()) {
      put32(b, 0);
      put32(b, 0);
    } else {
      put32(b, kVarTag);
      put32(b, (uint32_t)vars.size());
      for (const Var& v : vars) {
        put_name(b, v.name);
        put32(b, (uint32_t)v.dims.size());
        for (int d : v.dims) put32(b, (uint32_t)d);
        put_atts(b, v.atts);
        put32(b, (uint32_t)v.type);
        put32(b, (uint32_t)((v.bytes + 3) / 4 * 4));
        put64(b, v.begin);
      }
    }
    return b;
  }
};

namespace {

sbslpm_status add_att(sbslpm_nc* nc, int varid, const char* name, int type, long n, const void* vals) {
  if (!nc || !name || n < 0 || (n > 0 && !vals) || varid < -1 || varid >= (int)nc->vars.size())
    return SBSLPM_ERR_ARG;
  Att a{name, type, {}, n};
  const unsigned char* p = static_cast<const unsigned char*>(vals);
  const int sz = type_size(type);
  for (long i = 0; i < n; i++)
    for (int k = sz - 1; k >= 0; k--) a.be.push_back(p[i * sz + k]);  // host little-endian to big-endian
  std::vector<Att>& list = varid < 0 ? nc->gatts : nc->vars[varid].atts;
  for (Att& old : list)
    if (old.name == a.name) {
      old = a;
      return SBSLPM_OK;
    }
  list.push_back(a);
  if (!nc->defining) {
    const std::vector<unsigned char> h = nc->header();
    if ((long)h.size() > nc->reserved)
      return set_last_error("netCDF header outgrew the room reserved at enddef"), SBSLPM_ERR_ARG;
    if (std::fseek(nc->f, 0, SEEK_SET) != 0 || std::fwrite(h.data(), 1, h.size(), nc->f) != h.size())
      return set_last_error("netCDF header write failed"), SBSLPM_ERR_ARG;
  }
  return SBSLPM_OK;
}

sbslpm_status put_vara(sbslpm_nc* nc, int varid, int type, const long* start, const long* count, const void* data) {
  if (!nc || nc->defining || varid < 0 || varid >= (int)nc->vars.size() || !data) return SBSLPM_ERR_ARG;
  const Var& v = nc->vars[varid];
  if (v.type != type) return set_last_error("netCDF variable type mismatch"), SBSLPM_ERR_ARG;
  const int nd = (int)v.dims.size(), sz = type_size(type);
  std::vector<long> len(nd), st(nd, 0), cnt(nd, 1);
  long total = 1;
  for (int k = 0; k < nd; k++) {
    len[k] = nc->dims[v.dims[k]].second;
    if (start) st[k] = start[k];
    cnt[k] = count ? count[k] : len[k];
    if (st[k] < 0 || cnt[k] < 0 || st[k] + cnt[k] > len[k]) return SBSLPM_ERR_ARG;
    total *= cnt[k];
  }
  if (total == 0) return SBSLPM_OK;
  // rows along the last dimension are contiguous in the file
  const long row = nd ? cnt[nd - 1] : 1, nrows = total / row;
  std::vector<unsigned char> buf((size_t)row * sz);
  std::vector<long> idx(nd, 0);
  const unsigned char* p = static_cast<const unsigned char*>(data);
  for (long r = 0; r < nrows; r++) {
    long off = 0;
    for (int k = 0; k < nd; k++) off = off * len[k] + st[k] + (k < nd - 1 ? idx[k] : 0);
    for (long e = 0; e < row; e++)
      for (int b = 0; b < sz; b++) buf[(size_t)e * sz + b] = p[((size_t)r * row + e) * sz + (sz - 1 - b)];
    if (std::fseek(nc->f, (long)(v.begin + (uint64_t)off * sz), SEEK_SET) != 0 ||
        std::fwrite(buf.data(), 1, buf.size(), nc->f) != buf.size())
      return set_last_error("netCDF data write failed"), SBSLPM_ERR_ARG;
    for (int k = nd - 2; k >= 0; k--) {  // next row: odometer over the leading dimensions
      if (++idx[k] < cnt[k]) break;
      idx[k] = 0;
    }
  }
  return SBSLPM_OK;
}

}  // namespace

extern "C" {

sbslpm_status sbslpm_nc_create(const char* path, sbslpm_nc** out) {
  if (!path || !out) return SBSLPM_ERR_ARG;
  *out = nullptr;
  FILE* f = std::fopen(path, "wb+");
  if (!f) return set_last_error(std::string("cannot create ") + path), SBSLPM_ERR_ARG;
  sbslpm_nc* nc = new sbslpm_nc();
  nc->f = f;
  *out = nc;
  return SBSLPM_OK;
}

sbslpm_status sbslpm_nc_def_dim(sbslpm_nc* nc, const char* name, long len, int* dimid) {
  if (!nc || !nc->defining || !name || len < 1 || len > 0x7fffffffL || !dimid) return SBSLPM_ERR_ARG;
  nc->dims.push_back({name, len});
  *dimid = (int)nc->dims.size() - 1;
  return SBSLPM_OK;
}

sbslpm_status sbslpm_nc_def_var(sbslpm_nc* nc, const char* name, int type, int ndims, const int* dimids,
                                int* varid) {
  if (!nc || !nc->defining || !name || !varid || (type != kInt && type != kDouble) || ndims < 0 ||
      (ndims > 0 && !dimids))
    return SBSLPM_ERR_ARG;
  Var v;
  v.name = name;
  v.type = type;
  for (int k = 0; k < ndims; k++) {
    if (dimids[k] < 0 || dimids[k] >= (int)nc->dims.size()) return SBSLPM_ERR_ARG;
    v.dims.push_back(dimids[k]);
  }
  nc->vars.push_back(v);
  *varid = (int)nc->vars.size() - 1;
  return SBSLPM_OK;
}

sbslpm_status sbslpm_nc_put_att_text(sbslpm_nc* nc, int varid, const char* name, const char* text) {
  if (!text) return SBSLPM_ERR_ARG;
  return add_att(nc, varid, name, kChar, (long)std::strlen(text), text);
}

sbslpm_status sbslpm_nc_put_att_int(sbslpm_nc* nc, int varid, const char* name, long n, const int* vals) {
  return add_att(nc, varid, name, kInt, n, vals);
}

sbslpm_status sbslpm_nc_put_att_double(sbslpm_nc* nc, int varid, const char* name, long n, const double* vals) {
  return add_att(nc, varid, name, kDouble, n, vals);
}

sbslpm_status sbslpm_nc_enddef(sbslpm_nc* nc) {
  if (!nc || !nc->defining) return SBSLPM_ERR_ARG;
  nc->reserved = (long)nc->header().size() + kHeaderSlack;
  nc->reserved = (nc->reserved + 511) / 512 * 512;
  uint64_t at = (uint64_t)nc->reserved;
  for (Var& v : nc->vars) {
    uint64_t n = 1;
    for (int d : v.dims) n *= (uint64_t)nc->dims[d].second;
    v.bytes = n * type_size(v.type);
    v.begin = at;
    at += (v.bytes + 3) / 4 * 4;
  }
  nc->defining = false;
  const std::vector<unsigned char> h = nc->header();
  std::vector<unsigned char> zeros(4096, 0);
  if (std::fwrite(h.data(), 1, h.size(), nc->f) != h.size())
    return set_last_error("netCDF header write failed"), SBSLPM_ERR_ARG;
  // zero-fill the reserved room and the data region (unwritten values read as 0)
  for (uint64_t pos = h.size(); pos < at;) {
    const size_t k = (size_t)std::min<uint64_t>(zeros.size(), at - pos);
    if (std::fwrite(zeros.data(), 1, k, nc->f) != k) return set_last_error("netCDF write failed"), SBSLPM_ERR_ARG;
    pos += k;
  }
  return SBSLPM_OK;
}

sbslpm_status sbslpm_nc_put_vara_double(sbslpm_nc* nc, int varid, const long* start, const long* count,
                                        const double* data) {
  return put_vara(nc, varid, kDouble, start, count, data);
}

sbslpm_status sbslpm_nc_put_vara_int(sbslpm_nc* nc, int varid, const long* start, const long* count,
                                     const int* data) {
  return put_vara(nc, varid, kInt, start, count, data);
}

sbslpm_status sbslpm_nc_close(sbslpm_nc* nc) {
  if (!nc) return SBSLPM_OK;
  sbslpm_status s = SBSLPM_OK;
  if (nc->defining) s = sbslpm_nc_enddef(nc);
  if (std::fclose(nc->f) != 0 && s == SBSLPM_OK) {
    set_last_error("netCDF close failed");
    s = SBSLPM_ERR_ARG;
  }
  delete nc;
  return s;
}

}  // extern "C"
