// NetCDFGrid3DWriter / NetCDFGrid3DReader (ocustorage/gridnetcdf.h:67-183): the reference's grid
// files, written and read here without libnetcdf, in the NetCDF classic file format (the
// published "NetCDF Classic Format Specification": CDF-1, or CDF-2 with 64-bit offsets, big-
// endian XDR values).  The file carries what the reference's writer puts there: an unlimited
// "Time" dimension and a float "Time" variable, global attributes nx, ny, nz (int) and hx, hy,
// hz (float), one dimension and float coordinate variable per distinct axis offset
// ("XAxisCentered", "XAxisUFace", "XAxisOffset%.4f", ..., values i * h + offset, as the reference
// computes them), and each grid variable on (Time, X, Y, Z), x slowest.  Host code only.
//
// The writer keeps the variables' slabs in memory and writes the file at close() (the header's
// record count and offsets are final then); a variable without data at a time level holds the
// format's default fill value there.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "ocu_internal.h"

namespace ocub {
namespace {

enum { NC_DIMENSION = 10, NC_VARIABLE = 11, NC_ATTRIBUTE = 12 };
enum { T_INT = 4, T_FLOAT = 5, T_DOUBLE = 6 };

int type_size(int t) { return t == T_DOUBLE ? 8 : 4; }

// ---- big-endian output ------------------------------------------------------------------------
struct Out {
  std::vector<unsigned char> b;
  void u32(uint32_t v) {
    for (int s = 24; s >= 0; s -= 8) b.push_back((unsigned char)(v >> s));
  }
  void u64(uint64_t v) {
    for (int s = 56; s >= 0; s -= 8) b.push_back((unsigned char)(v >> s));
  }
  void name(const std::string &n) {
    u32((uint32_t)n.size());
    b.insert(b.end(), n.begin(), n.end());
    while (b.size() % 4) b.push_back(0);
  }
};

void put_be(unsigned char *dst, const void *src, int size) {
  const unsigned char *s = static_cast<const unsigned char *>(src);
  for (int q = 0; q < size; q++) dst[q] = s[size - 1 - q];
}

void get_be(void *dst, const unsigned char *src, int size) {
  unsigned char *d = static_cast<unsigned char *>(dst);
  for (int q = 0; q < size; q++) d[q] = src[size - 1 - q];
}

// default fill values of the classic format
void fill_value(int t, unsigned char *dst) {
  if (t == T_DOUBLE) {
    const double v = 9.9692099683868690e+36;
    put_be(dst, &v, 8);
  } else if (t == T_FLOAT) {
    const float v = 9.96921e+36f;
    put_be(dst, &v, 4);
  } else {
    const int32_t v = -2147483647;
    put_be(dst, &v, 4);
  }
}

// value of a strided host grid converted to the file type (same type only, as the reference)
void pack(unsigned char *dst, const void *src, int t, long long xs, long long ys, int nx, int ny, int nz) {
  const int es = type_size(t);
  long long q = 0;
  for (int i = 0; i < nx; i++)
    for (int j = 0; j < ny; j++)
      for (int k = 0; k < nz; k++, q++)
        put_be(dst + q * es, static_cast<const unsigned char *>(src) + ((long long)i * xs + (long long)j * ys + k) * es,
               es);
}

}  // namespace

struct NcWriter {
  struct Var {
    std::string name;
    int type;
    int dx, dy, dz;        // dimension ids of the axes
    int nx, ny, nz;
    std::map<int, std::vector<unsigned char>> slabs;  // time level -> packed big-endian values
  };
  struct Axis {
    std::string name;
    int len;
    std::vector<float> values;
  };
  std::string path;
  int nx = 0, ny = 0, nz = 0;
  float hx = 1, hy = 1, hz = 1;
  std::vector<float> times;
  std::vector<Axis> axes;                  // dimension ids 1.. (0 is Time)
  std::map<std::pair<int, float>, int> axis_of;  // (axis, offset) -> dimension id
  std::vector<Var> vars;

  int axis(int a, float offset) {
    auto it = axis_of.find({a, offset});
    if (it != axis_of.end()) return it->second;
    const char *letter = a == 0 ? "X" : (a == 1 ? "Y" : "Z");
    const char *face = a == 0 ? "UFace" : (a == 1 ? "VFace" : "WFace");
    char buf[64];
    if (offset == 0.5f) std::snprintf(buf, sizeof buf, "%sAxisCentered", letter);
    else if (offset == 0.0f) std::snprintf(buf, sizeof buf, "%sAxis%s", letter, face);
    else std::snprintf(buf, sizeof buf, "%sAxisOffset%.4f", letter, offset);
    const int n = a == 0 ? nx : (a == 1 ? ny : nz);
    const float h = a == 0 ? hx : (a == 1 ? hy : hz);
    Axis ax;
    ax.name = buf;
    ax.len = offset == 0.0f ? n + 1 : n;
    for (int q = 0; q < ax.len; q++) ax.values.push_back(q * h + offset);  // the reference's coordinate values
    axes.push_back(ax);
    const int id = (int)axes.size();
    axis_of[{a, offset}] = id;
    return id;
  }

  ocu_status write_file() {
    const int nrec = (int)times.size();
    // header, with begin offsets filled in a second pass
    std::vector<int> coord_order;  // coordinate variables (non-record) in axis order
    auto header = [&](const std::vector<uint64_t> &begins, int version) {
      Out o;
      o.b = {'C', 'D', 'F', (unsigned char)version};
      o.u32((uint32_t)nrec);
      o.u32(NC_DIMENSION);
      o.u32((uint32_t)(1 + axes.size()));
      o.name("Time");
      o.u32(0);
      for (const Axis &ax : axes) {
        o.name(ax.name);
        o.u32((uint32_t)ax.len);
      }
      o.u32(NC_ATTRIBUTE);
      o.u32(6);
      const char *in[3] = {"nx", "ny", "nz"};
      const int iv[3] = {nx, ny, nz};
      for (int q = 0; q < 3; q++) {
        o.name(in[q]);
        o.u32(T_INT);
        o.u32(1);
        o.u32((uint32_t)iv[q]);
      }
      const char *fn[3] = {"hx", "hy", "hz"};
      const float fv[3] = {hx, hy, hz};
      for (int q = 0; q < 3; q++) {
        o.name(fn[q]);
        o.u32(T_FLOAT);
        o.u32(1);
        uint32_t bits;
        std::memcpy(&bits, &fv[q], 4);
        o.u32(bits);
      }
      o.u32(NC_VARIABLE);
      o.u32((uint32_t)(1 + axes.size() + vars.size()));
      size_t v = 0;
      auto var_entry = [&](const std::string &n, const std::vector<int> &dims, int t, uint64_t vsize) {
        o.name(n);
        o.u32((uint32_t)dims.size());
        for (int d : dims) o.u32((uint32_t)d);
        o.u32(0);  // no variable attributes
        o.u32(0);
        o.u32((uint32_t)t);
        o.u32((uint32_t)std::min<uint64_t>(vsize, 0xffffffffu));
        if (version == 1) o.u32((uint32_t)begins[v]);
        else o.u64(begins[v]);
        v++;
      };
      var_entry("Time", {0}, T_FLOAT, 4);
      for (size_t a = 0; a < axes.size(); a++) var_entry(axes[a].name, {(int)a + 1}, T_FLOAT, 4ull * axes[a].len);
      for (const Var &x : vars)
        var_entry(x.name, {0, x.dx, x.dy, x.dz}, x.type, (uint64_t)type_size(x.type) * x.nx * x.ny * x.nz);
      return o.b;
    };
    // sizes: non-record coordinate variables first, then the records (Time and every variable)
    uint64_t nonrec = 0;
    for (const Axis &ax : axes) nonrec += 4ull * ax.len;
    uint64_t recsize = 4;
    for (const Var &x : vars) recsize += (uint64_t)type_size(x.type) * x.nx * x.ny * x.nz;
    const uint64_t total_guess = nonrec + recsize * nrec;
    const int version = total_guess > 0x7fffffffull ? 2 : 1;
    std::vector<uint64_t> begins(1 + axes.size() + vars.size(), 0);
    const size_t hsize = header(begins, version).size();
    uint64_t off = hsize;
    for (size_t a = 0; a < axes.size(); a++) {
      begins[1 + a] = off;
      off += 4ull * axes[a].len;
    }
    uint64_t roff = off;
    begins[0] = roff;
    roff += 4;
    for (size_t x = 0; x < vars.size(); x++) {
      begins[1 + axes.size() + x] = roff;
      roff += (uint64_t)type_size(vars[x].type) * vars[x].nx * vars[x].ny * vars[x].nz;
    }
    const std::vector<unsigned char> hdr = header(begins, version);
    std::FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] NetCDFGrid3DWriter::close - could not open \"%s\" for writing", path.c_str());
    bool ok = std::fwrite(hdr.data(), 1, hdr.size(), f) == hdr.size();
    for (const Axis &ax : axes) {
      std::vector<unsigned char> buf(4 * ax.values.size());
      for (size_t q = 0; q < ax.values.size(); q++) put_be(&buf[4 * q], &ax.values[q], 4);
      ok = ok && std::fwrite(buf.data(), 1, buf.size(), f) == buf.size();
    }
    for (int r = 0; r < nrec && ok; r++) {
      unsigned char tb[4];
      put_be(tb, &times[r], 4);
      ok = std::fwrite(tb, 1, 4, f) == 4;
      for (const Var &x : vars) {
        const size_t n = (size_t)x.nx * x.ny * x.nz, es = type_size(x.type);
        auto it = x.slabs.find(r);
        if (it != x.slabs.end()) {
          ok = ok && std::fwrite(it->second.data(), 1, n * es, f) == n * es;
        } else {
          std::vector<unsigned char> fill(n * es);
          for (size_t q = 0; q < n; q++) fill_value(x.type, &fill[q * es]);
          ok = ok && std::fwrite(fill.data(), 1, fill.size(), f) == fill.size();
        }
      }
    }
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] NetCDFGrid3DWriter::close - write to \"%s\" failed", path.c_str());
    return OCU_OK;
  }
};

struct NcReader {
  struct Var {
    std::string name;
    int type = 0;
    std::vector<int> dims;
    uint64_t begin = 0;
    bool record = false;
  };
  std::vector<unsigned char> data;
  int nx = 0, ny = 0, nz = 0;
  float hx = 0, hy = 0, hz = 0;
  int nrec = 0;
  uint64_t recsize = 0;
  std::vector<std::pair<std::string, int>> dims;  // name, length (0: record)
  std::vector<Var> vars;
  std::vector<float> times;
  size_t pos = 0;
  bool bad = false;

  uint32_t u32() {
    if (pos + 4 > data.size()) { bad = true; return 0; }
    uint32_t v = 0;
    for (int q = 0; q < 4; q++) v = (v << 8) | data[pos + q];
    pos += 4;
    return v;
  }
  uint64_t u64() {
    const uint64_t hi = u32();
    return (hi << 32) | u32();
  }
  std::string name() {
    const uint32_t n = u32();
    if (bad || pos + n > data.size()) { bad = true; return ""; }
    std::string s(reinterpret_cast<const char *>(&data[pos]), n);
    pos += (n + 3) & ~3u;
    return s;
  }
  // attributes: keeps the global nx..hz, skips the rest
  void attributes(bool global) {
    const uint32_t tag = u32(), n = u32();
    if (tag == 0) return;
    for (uint32_t q = 0; q < n && !bad; q++) {
      const std::string an = name();
      const uint32_t t = u32(), cnt = u32();
      const int es = (t == 1 || t == 2) ? 1 : (t == 3 ? 2 : (t == T_DOUBLE ? 8 : 4));
      const size_t bytes = ((size_t)es * cnt + 3) & ~size_t(3);
      if (pos + bytes > data.size()) { bad = true; return; }
      if (global && cnt >= 1) {
        if (t == T_INT && (an == "nx" || an == "ny" || an == "nz")) {
          int32_t v;
          get_be(&v, &data[pos], 4);
          (an == "nx" ? nx : an == "ny" ? ny : nz) = v;
        } else if (t == T_FLOAT && (an == "hx" || an == "hy" || an == "hz")) {
          float v;
          get_be(&v, &data[pos], 4);
          (an == "hx" ? hx : an == "hy" ? hy : hz) = v;
        }
      }
      pos += bytes;
    }
  }

  ocu_status parse(const char *path) {
    std::FILE *f = std::fopen(path, "rb");
    if (!f) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] NetCDFGrid3DReader::open - Could not open \"%s\"", path);
    std::fseek(f, 0, SEEK_END);
    const long sz = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    data.resize(sz > 0 ? (size_t)sz : 0);
    const bool rd = data.empty() || std::fread(data.data(), 1, data.size(), f) == data.size();
    std::fclose(f);
    if (!rd || data.size() < 8 || data[0] != 'C' || data[1] != 'D' || data[2] != 'F' || (data[3] != 1 && data[3] != 2))
      return fail(OCU_ERR_INVALID_VALUE, "[ERROR] NetCDFGrid3DReader::open - \"%s\" is not a NetCDF classic file", path);
    const int version = data[3];
    pos = 4;
    nrec = (int)u32();
    uint32_t tag = u32(), n = u32();
    if (tag == NC_DIMENSION)
      for (uint32_t q = 0; q < n && !bad; q++) {
        const std::string dn = name();
        dims.push_back({dn, (int)u32()});
      }
    attributes(true);
    tag = u32();
    n = u32();
    if (tag == NC_VARIABLE)
      for (uint32_t q = 0; q < n && !bad; q++) {
        Var v;
        v.name = name();
        const uint32_t nd = u32();
        for (uint32_t d = 0; d < nd && !bad; d++) v.dims.push_back((int)u32());
        attributes(false);
        v.type = (int)u32();
        u32();  // vsize
        v.begin = version == 1 ? u32() : u64();
        for (int d : v.dims)
          if (d < 0 || d >= (int)dims.size()) bad = true;
        v.record = !bad && !v.dims.empty() && dims[v.dims[0]].second == 0;
        vars.push_back(v);
      }
    if (bad) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] NetCDFGrid3DReader::open - malformed header in \"%s\"", path);
    // record size: the padded sizes of every record variable (one record variable alone: unpadded)
    int nrecvars = 0;
    for (const Var &v : vars) nrecvars += v.record;
    recsize = 0;
    for (const Var &v : vars)
      if (v.record) {
        uint64_t s = type_size(v.type);
        for (size_t d = 1; d < v.dims.size(); d++) s *= (uint64_t)dims[v.dims[d]].second;
        recsize += nrecvars == 1 ? s : ((s + 3) & ~3ull);
      }
    times.assign(nrec, 0.f);
    for (const Var &v : vars)
      if (v.name == "Time" && v.record && v.dims.size() == 1 && v.type == T_FLOAT)
        for (int r = 0; r < nrec; r++) {
          const uint64_t o = v.begin + (uint64_t)r * recsize;
          if (o + 4 <= data.size()) get_be(&times[r], &data[o], 4);
        }
    return OCU_OK;
  }

  const Var *find(const char *n) const {
    for (const Var &v : vars)
      if (v.name == n) return &v;
    return nullptr;
  }
  bool grid_var(const Var &v) const { return v.record && v.dims.size() == 4; }
};

}  // namespace ocub

// ---- C ABI ----------------------------------------------------------------------------------
struct ocu_nc_writer {
  ocub::NcWriter w;
};
struct ocu_nc_reader {
  ocub::NcReader r;
};

using namespace ocub;

static bool nc_type_ok(int t) { return t == OCU_NC_FLOAT || t == OCU_NC_DOUBLE || t == OCU_NC_INT; }

extern "C" {

ocu_status ocu_nc_writer_open(const char *path, int nx, int ny, int nz, float hx, float hy, float hz,
                              ocu_nc_writer **out) {
  if (!path || !out) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] NetCDFGrid3DWriter::open - null argument");
  *out = nullptr;
  if (nx < 1 || ny < 1 || nz < 1) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] NetCDFGrid3DWriter::open - bad dimensions");
  std::FILE *f = std::fopen(path, "wb");  // NC_CLOBBER: the file is created (truncated) now
  if (!f) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] NetCDFGrid3DWriter::open - Could not open \"%s\"", path);
  std::fclose(f);
  std::unique_ptr<ocu_nc_writer> w(new ocu_nc_writer());
  w->w.path = path;
  w->w.nx = nx; w->w.ny = ny; w->w.nz = nz;
  w->w.hx = hx; w->w.hy = hy; w->w.hz = hz;
  *out = w.release();
  return OCU_OK;
}

ocu_status ocu_nc_writer_define_variable(ocu_nc_writer *w, const char *name, int nc_type, int staggering,
                                         float offsetx, float offsety, float offsetz) {
  if (!w || !name) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] NetCDFGrid3DWriter::define_variable - null argument");
  if (!nc_type_ok(nc_type))
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] NetCDFGrid3DWriter::define_variable - only NC_FLOAT, NC_DOUBLE, NC_INT types supported");
  for (const auto &v : w->w.vars)
    if (v.name == name)
      return fail(OCU_ERR_INVALID_VALUE, "[ERROR] NetCDFGrid3DWriter::define_variable - variable \"%s\" previously defined", name);
  if (std::strcmp(name, "Time") == 0)
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] NetCDFGrid3DWriter::define_variable - \"Time\" is the time coordinate");
  // grid_staggering_to_offset / _to_dimension (gridnetcdf.h:41-63); GS_CUSTOM keeps the offsets
  switch (staggering) {
    case OCU_GS_CENTER_POINT: offsetx = offsety = offsetz = 0.5f; break;
    case OCU_GS_U_FACE: offsetx = 0.0f; offsety = offsetz = 0.5f; break;
    case OCU_GS_V_FACE: offsety = 0.0f; offsetx = offsetz = 0.5f; break;
    case OCU_GS_W_FACE: offsetz = 0.0f; offsetx = offsety = 0.5f; break;
    case OCU_GS_CUSTOM: break;
    default: return fail(OCU_ERR_INVALID_VALUE, "[ERROR] NetCDFGrid3DWriter::define_variable - bad staggering %d", staggering);
  }
  NcWriter::Var v;
  v.name = name;
  v.type = nc_type;
  v.dx = w->w.axis(0, offsetx);
  v.dy = w->w.axis(1, offsety);
  v.dz = w->w.axis(2, offsetz);
  v.nx = w->w.nx + (staggering == OCU_GS_U_FACE);
  v.ny = w->w.ny + (staggering == OCU_GS_V_FACE);
  v.nz = w->w.nz + (staggering == OCU_GS_W_FACE);
  w->w.vars.push_back(std::move(v));
  return OCU_OK;
}

ocu_status ocu_nc_writer_add_time_level(ocu_nc_writer *w, float time, int *level) {
  if (!w) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] NetCDFGrid3DWriter::add_time_level - null handle");
  w->w.times.push_back(time);
  if (level) *level = (int)w->w.times.size() - 1;
  return OCU_OK;
}

ocu_status ocu_nc_writer_add_data(ocu_nc_writer *w, const char *name, const void *origin, int nc_type,
                                  long long xstride, long long ystride, int nx, int ny, int nz, int time_level) {
  if (!w || !name || !origin) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] NetCDFGrid3DWriter::add_data - null argument");
  NcWriter::Var *v = nullptr;
  for (auto &x : w->w.vars)
    if (x.name == name) v = &x;
  if (!v) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] NetCDFGrid3DWriter::add_data_internal - variable \"%s\" not found", name);
  if (nx != v->nx || ny != v->ny || nz != v->nz)
    return fail(OCU_ERR_LAYOUT, "[ERROR] NetCDFGrid3DWriter::add_data_internal - dimension mismatch, expected (%d %d %d), grid has (%d %d %d)",
                v->nx, v->ny, v->nz, nx, ny, nz);
  if (nc_type != v->type)
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] NetCDFGrid3DWriter::add_data_internal - variable \"%s\" type does not match data_type", name);
  if (time_level < 0) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] NetCDFGrid3DWriter::add_data - bad time level");
  // add_zero_time_level (gridnetcdf.cpp): writing level 0 of an empty time axis creates time 0
  if (time_level == 0 && w->w.times.empty()) w->w.times.push_back(0.0f);
  if (time_level >= (int)w->w.times.size())
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] NetCDFGrid3DWriter::add_data - time level %d not added", time_level);
  std::vector<unsigned char> slab((size_t)type_size(nc_type) * nx * ny * nz);
  pack(slab.data(), origin, nc_type, xstride, ystride, nx, ny, nz);
  v->slabs[time_level] = std::move(slab);
  return OCU_OK;
}

ocu_status ocu_nc_writer_add_grid(ocu_nc_writer *w, const char *name, const ocu_grid *g, int time_level) {
  if (!w || !g) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] NetCDFGrid3DWriter::add_data - null argument");
  std::vector<unsigned char> host((size_t)dtype_size(g->dtype) * g->L.allocated);
  OCU_TRY(check_cuda(cudaMemcpy(host.data(), g->buf, host.size(), cudaMemcpyDeviceToHost), "add_data download"));
  const int t = g->dtype == OCU_F64 ? OCU_NC_DOUBLE : OCU_NC_FLOAT;
  return ocu_nc_writer_add_data(w, name, host.data() + (size_t)dtype_size(g->dtype) * g->L.shift, t, g->L.xstride,
                                g->L.ystride, g->L.nx, g->L.ny, g->L.nz, time_level);
}

ocu_status ocu_nc_writer_close(ocu_nc_writer *w) {
  if (!w) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] NetCDFGrid3DWriter::close - null handle");
  const ocu_status st = w->w.write_file();
  delete w;
  return st;
}

ocu_status ocu_nc_reader_open(const char *path, ocu_nc_reader **out) {
  if (!path || !out) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] NetCDFGrid3DReader::open - null argument");
  *out = nullptr;
  std::unique_ptr<ocu_nc_reader> r(new ocu_nc_reader());
  OCU_TRY(r->r.parse(path));
  *out = r.release();
  return OCU_OK;
}

void ocu_nc_reader_close(ocu_nc_reader *r) { delete r; }

ocu_status ocu_nc_reader_info(const ocu_nc_reader *r, int *nx, int *ny, int *nz, float *hx, float *hy, float *hz,
                              int *num_time_levels) {
  if (!r) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] NetCDFGrid3DReader - null handle");
  if (nx) *nx = r->r.nx;
  if (ny) *ny = r->r.ny;
  if (nz) *nz = r->r.nz;
  if (hx) *hx = r->r.hx;
  if (hy) *hy = r->r.hy;
  if (hz) *hz = r->r.hz;
  if (num_time_levels) *num_time_levels = r->r.nrec;
  return OCU_OK;
}

ocu_status ocu_nc_reader_get_time(const ocu_nc_reader *r, int time_level, float *time) {
  if (!r || !time || time_level < 0 || time_level >= r->r.nrec)
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] NetCDFGrid3DReader::get_time - bad time level");
  *time = r->r.times[time_level];
  return OCU_OK;
}

// list_variables: the grid variables (on Time, X, Y, Z), in file order
ocu_status ocu_nc_reader_num_variables(const ocu_nc_reader *r, int *n) {
  if (!r || !n) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] NetCDFGrid3DReader - null argument");
  int c = 0;
  for (const auto &v : r->r.vars) c += r->r.grid_var(v);
  *n = c;
  return OCU_OK;
}

ocu_status ocu_nc_reader_variable(const ocu_nc_reader *r, int index, char *name, int name_size, int *nc_type,
                                  int *nx, int *ny, int *nz) {
  if (!r) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] NetCDFGrid3DReader - null handle");
  int c = 0;
  for (const auto &v : r->r.vars) {
    if (!r->r.grid_var(v)) continue;
    if (c++ != index) continue;
    if (name && name_size > 0) {
      std::strncpy(name, v.name.c_str(), (size_t)name_size - 1);
      name[name_size - 1] = 0;
    }
    if (nc_type) *nc_type = v.type;
    if (nx) *nx = r->r.dims[v.dims[1]].second;
    if (ny) *ny = r->r.dims[v.dims[2]].second;
    if (nz) *nz = r->r.dims[v.dims[3]].second;
    return OCU_OK;
  }
  return fail(OCU_ERR_INVALID_VALUE, "[ERROR] NetCDFGrid3DReader - no variable %d", index);
}

// read_variable: into a strided host grid of the variable's type and dimensions
ocu_status ocu_nc_reader_read(const ocu_nc_reader *r, const char *name, void *origin, int nc_type, long long xstride,
                              long long ystride, int nx, int ny, int nz, int time_level) {
  if (!r || !name || !origin) return fail(OCU_ERR_INVALID_VALUE, "[ERROR] NetCDFGrid3DReader::read_variable - null argument");
  const NcReader::Var *v = r->r.find(name);
  if (!v || !r->r.grid_var(*v))
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] NetCDFGrid3DReader::read_variable - variable \"%s\" not found", name);
  const int vx = r->r.dims[v->dims[1]].second, vy = r->r.dims[v->dims[2]].second, vz = r->r.dims[v->dims[3]].second;
  if (nx != vx || ny != vy || nz != vz)
    return fail(OCU_ERR_LAYOUT, "[ERROR] NetCDFGrid3DReader::read_variable - dimension mismatch, file has (%d %d %d)", vx, vy, vz);
  if (nc_type != v->type)
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] NetCDFGrid3DReader::read_variable - variable \"%s\" type mismatch", name);
  if (time_level < 0 || time_level >= r->r.nrec)
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] NetCDFGrid3DReader::read_variable - bad time level %d", time_level);
  const int es = type_size(v->type);
  const uint64_t base = v->begin + (uint64_t)time_level * r->r.recsize;
  if (base + (uint64_t)es * vx * vy * vz > r->r.data.size())
    return fail(OCU_ERR_INVALID_VALUE, "[ERROR] NetCDFGrid3DReader::read_variable - file truncated");
  const unsigned char *src = &r->r.data[base];
  long long q = 0;
  for (int i = 0; i < nx; i++)
    for (int j = 0; j < ny; j++)
      for (int k = 0; k < nz; k++, q++)
        get_be(static_cast<unsigned char *>(origin) + ((long long)i * xstride + (long long)j * ystride + k) * es,
               src + q * es, es);
  return OCU_OK;
}

}  // extern "C"
