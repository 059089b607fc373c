// Minimal read-only HDF5 parser for TART observation files.
//
// Replaces Observation::from_hdf5 (observation.rs:48-92), which reads the
// datasets `config` (JSON string), `timestamp` (ISO-8601 string) and `data`
// (2-D uint8, one row of numpy.packbits'd samples per antenna) through the
// hdf5-reader crate.  Implemented from the public HDF5 file-format
// specification, for the subset TART files use:
//   * superblock version 0 or 1;
//   * root group stored as a symbol table (version-1 B-tree of SNOD nodes
//     and a local heap for the link names);
//   * version-1 object headers, with continuation blocks;
//   * datatypes: fixed-point (uint8), fixed-length string, variable-length
//     string (global heap collections);
//   * layouts: compact and contiguous.
// Anything else is reported as an error rather than guessed.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/tga.h"

namespace {

struct Reader {
  std::vector<uint8_t> f;
  int so = 8, sl = 8;  // size of offsets / lengths

  void need(uint64_t at, uint64_t n) const {
    if (at > f.size() || n > f.size() - at) throw std::runtime_error("HDF5: read past end of file");
  }
  uint64_t u(uint64_t at, int n) const {
    need(at, n);
    uint64_t v = 0;
    for (int i = 0; i < n; ++i) v |= (uint64_t)f[at + i] << (8 * i);
    return v;
  }
  uint64_t off(uint64_t at) const { return u(at, so); }
  uint64_t len(uint64_t at) const { return u(at, sl); }
  bool undef(uint64_t a) const { return so == 8 ? a == ~0ull : a == ((1ull << (8 * so)) - 1); }
};

struct Dataset {
  std::vector<uint64_t> dims;
  int dclass = -1;          // datatype class
  uint32_t dsize = 0;       // element size
  bool vlen_string = false;
  int layout = -1;          // 0 compact, 1 contiguous
  uint64_t addr = 0, size = 0;
  std::vector<uint8_t> compact;
};

void parse_messages(const Reader& r, uint64_t start, uint64_t end, Dataset& ds, int depth);

void parse_message(const Reader& r, int type, uint64_t p, uint64_t n, Dataset& ds, int depth) {
  switch (type) {
    case 0x0001: {  // dataspace
      const int ver = (int)r.u(p, 1);
      const int rank = (int)r.u(p + 1, 1);
      uint64_t q = (ver == 1) ? p + 8 : p + 4;
      ds.dims.clear();
      for (int i = 0; i < rank; ++i) ds.dims.push_back(r.len(q + (uint64_t)i * r.sl));
      break;
    }
    case 0x0003: {  // datatype
      const int cv = (int)r.u(p, 1);
      ds.dclass = cv & 0x0F;
      ds.dsize = (uint32_t)r.u(p + 4, 4);
      if (ds.dclass == 9) ds.vlen_string = (r.u(p + 1, 1) & 0x0F) == 1;
      break;
    }
    case 0x0008: {  // data layout
      const int ver = (int)r.u(p, 1);
      if (ver == 3 || ver == 4) {
        const int cls = (int)r.u(p + 1, 1);
        ds.layout = cls;
        if (cls == 0) {
          const uint64_t sz = r.u(p + 2, 2);
          r.need(p + 4, sz);
          ds.compact.assign(r.f.begin() + p + 4, r.f.begin() + p + 4 + sz);
        } else if (cls == 1) {
          ds.addr = r.off(p + 2);
          ds.size = r.len(p + 2 + r.so);
        } else {
          throw std::runtime_error("HDF5: chunked storage is not supported");
        }
      } else if (ver == 1 || ver == 2) {
        const int dimensionality = (int)r.u(p + 1, 1);
        const int cls = (int)r.u(p + 2, 1);
        ds.layout = cls;
        uint64_t q = p + 8;
        if (cls == 1) {
          ds.addr = r.off(q);
          q += r.so;
          uint64_t total = 1;
          for (int i = 0; i < dimensionality; ++i) total *= r.u(q + 4 * i, 4);
          ds.size = total;
        } else if (cls == 0) {
          q += 4 * dimensionality;
          const uint64_t sz = r.u(q, 4);
          r.need(q + 4, sz);
          ds.compact.assign(r.f.begin() + q + 4, r.f.begin() + q + 4 + sz);
        } else {
          throw std::runtime_error("HDF5: chunked storage is not supported");
        }
      } else {
        throw std::runtime_error("HDF5: unsupported layout message version");
      }
      break;
    }
    case 0x0010: {  // continuation
      if (depth > 16) throw std::runtime_error("HDF5: continuation loop");
      const uint64_t a = r.off(p), l = r.len(p + r.so);
      parse_messages(r, a, a + l, ds, depth + 1);
      break;
    }
    default:
      break;
  }
  (void)n;
}

void parse_messages(const Reader& r, uint64_t p, uint64_t end, Dataset& ds, int depth) {
  while (p + 8 <= end) {
    const int type = (int)r.u(p, 2);
    const uint64_t n = r.u(p + 2, 2);
    r.need(p + 8, n);
    parse_message(r, type, p + 8, n, ds, depth);
    p += 8 + n;
    p = (p + 7) & ~7ull;  // messages are 8-byte aligned in v1 headers
  }
}

Dataset read_object(const Reader& r, uint64_t addr) {
  const int ver = (int)r.u(addr, 1);
  if (ver != 1) throw std::runtime_error("HDF5: only version-1 object headers are supported");
  const uint64_t hsize = r.u(addr + 8, 4);
  Dataset ds;
  parse_messages(r, addr + 16, addr + 16 + hsize, ds, 0);
  return ds;
}

// name -> object header address of the root group's members
std::map<std::string, uint64_t> root_members(const Reader& r, uint64_t btree, uint64_t heap) {
  if (memcmp(&r.f[heap], "HEAP", 4) != 0) throw std::runtime_error("HDF5: bad local heap");
  const uint64_t heap_data = r.off(heap + 8 + 2 * r.sl);
  std::map<std::string, uint64_t> out;
  std::vector<uint64_t> stack{btree};
  int guard = 0;
  while (!stack.empty()) {
    if (++guard > 100000) throw std::runtime_error("HDF5: B-tree walk did not terminate");
    const uint64_t node = stack.back();
    stack.pop_back();
    r.need(node, 8);
    if (memcmp(&r.f[node], "TREE", 4) == 0) {
      const int level = (int)r.u(node + 5, 1);
      const int used = (int)r.u(node + 6, 2);
      uint64_t q = node + 8 + 2 * r.so;  // after siblings
      for (int i = 0; i < used; ++i) {
        q += r.sl;  // key
        stack.push_back(r.off(q));
        q += r.so;
      }
      (void)level;
    } else if (memcmp(&r.f[node], "SNOD", 4) == 0) {
      const int n = (int)r.u(node + 6, 2);
      uint64_t q = node + 8;
      const uint64_t entry = 2 * r.so + 4 + 4 + 16;
      for (int i = 0; i < n; ++i, q += entry) {
        const uint64_t name_off = r.off(q), obj = r.off(q + r.so);
        const uint64_t s = heap_data + name_off;
        r.need(s, 1);
        std::string name;
        for (uint64_t k = s; k < r.f.size() && r.f[k]; ++k) name.push_back((char)r.f[k]);
        out[name] = obj;
      }
    } else {
      throw std::runtime_error("HDF5: unexpected node in the group B-tree");
    }
  }
  return out;
}

std::string read_string(const Reader& r, const Dataset& ds) {
  std::vector<uint8_t> raw;
  if (ds.layout == 0) raw = ds.compact;
  else if (ds.layout == 1) {
    r.need(ds.addr, ds.vlen_string ? 4 + r.so + 4 : ds.dsize);
    raw.assign(r.f.begin() + ds.addr, r.f.begin() + ds.addr + (ds.vlen_string ? 4 + r.so + 4 : ds.dsize));
  }
  if (ds.dclass == 3) {  // fixed-length string
    std::string s(raw.begin(), raw.begin() + std::min<size_t>(raw.size(), ds.dsize));
    while (!s.empty() && (s.back() == '\0' || s.back() == ' ')) s.pop_back();
    return s;
  }
  if (ds.dclass == 9 && ds.vlen_string) {
    if (raw.size() < (size_t)(4 + r.so + 4)) throw std::runtime_error("HDF5: short vlen string");
    Reader t;
    t.f = raw;
    t.so = r.so;
    const uint64_t slen = t.u(0, 4), coll = t.off(4), index = t.u(4 + r.so, 4);
    if (memcmp(&r.f[coll], "GCOL", 4) != 0) throw std::runtime_error("HDF5: bad global heap");
    const uint64_t csize = r.len(coll + 8);
    uint64_t q = coll + 8 + r.sl;
    while (q + 8 + r.sl <= coll + csize) {
      const uint64_t idx = r.u(q, 2);
      const uint64_t osz = r.len(q + 8);
      if (idx == 0) break;
      if (idx == index) {
        r.need(q + 8 + r.sl, osz);
        return std::string((const char*)&r.f[q + 8 + r.sl], (size_t)std::min(osz, slen));
      }
      q += 8 + r.sl + ((osz + 7) & ~7ull);
    }
    throw std::runtime_error("HDF5: global heap object not found");
  }
  throw std::runtime_error("HDF5: dataset is not a string");
}

// The two fields Config reads (config.rs:10-19); extra keys are ignored.
bool json_number(const std::string& js, const char* key, double* out) {
  const std::string k = std::string("\"") + key + "\"";
  size_t p = js.find(k);
  if (p == std::string::npos) return false;
  p = js.find(':', p + k.size());
  if (p == std::string::npos) return false;
  ++p;
  while (p < js.size() && (js[p] == ' ' || js[p] == '\t' || js[p] == '\n' || js[p] == '\r')) ++p;
  char* e = nullptr;
  const double v = strtod(js.c_str() + p, &e);
  if (e == js.c_str() + p) return false;
  *out = v;
  return true;
}

}  // namespace

extern "C" int tga_observation_read_hdf5(const char* path, tga_observation* out) {
  if (!path || !out) return TGA_ERR_INVALID_ARG;
  std::memset(out, 0, sizeof *out);
  try {
    FILE* fp = std::fopen(path, "rb");
    if (!fp) {
      std::snprintf(out->error, sizeof out->error, "cannot open %s", path);
      return TGA_ERR_INVALID_ARG;
    }
    Reader r;
    std::fseek(fp, 0, SEEK_END);
    const long sz = std::ftell(fp);
    std::fseek(fp, 0, SEEK_SET);
    r.f.resize(sz > 0 ? (size_t)sz : 0);
    const size_t got = r.f.empty() ? 0 : std::fread(r.f.data(), 1, r.f.size(), fp);
    std::fclose(fp);
    if (got != r.f.size() || r.f.size() < 96 || std::memcmp(r.f.data(), "\x89HDF\r\n\x1a\n", 8) != 0)
      throw std::runtime_error("not an HDF5 file");
    const int sb = (int)r.u(8, 1);
    if (sb > 1) throw std::runtime_error("HDF5: superblock version >= 2 is not supported");
    r.so = (int)r.u(13, 1);
    r.sl = (int)r.u(14, 1);
    if (r.so != 8 || r.sl != 8) throw std::runtime_error("HDF5: only 8-byte offsets/lengths are supported");
    uint64_t q = 24 + (sb == 1 ? 4 : 0) + 4 * (uint64_t)r.so;  // root symbol table entry
    const uint64_t cache = r.u(q + 2 * r.so, 4);
    if (cache != 1) throw std::runtime_error("HDF5: root group without a cached symbol table");
    const uint64_t btree = r.off(q + 2 * r.so + 8), heap = r.off(q + 2 * r.so + 8 + r.so);
    auto members = root_members(r, btree, heap);
    for (const char* need : {"config", "timestamp", "data"})
      if (!members.count(need)) throw std::runtime_error(std::string("HDF5: dataset '") + need + "' missing");
    const std::string cfg = read_string(r, read_object(r, members["config"]));
    const std::string ts = read_string(r, read_object(r, members["timestamp"]));
    Dataset d = read_object(r, members["data"]);
    if (d.dims.size() != 2 || d.dclass != 0 || d.dsize != 1)
      throw std::runtime_error("HDF5: `data` must be a 2-D uint8 dataset");
    double n_ant = 0, fs = 0;
    if (!json_number(cfg, "num_antenna", &n_ant) || !json_number(cfg, "sampling_frequency", &fs))
      throw std::runtime_error("config JSON lacks num_antenna / sampling_frequency");
    const uint64_t rows = d.dims[0], row_bytes = d.dims[1];
    if ((uint64_t)n_ant != rows) {
      // observation.rs:78-85 compares the unpacked row count with the shape
      throw std::runtime_error("data antenna count (" + std::to_string(rows) + ") != config num_antenna (" +
                               std::to_string((uint64_t)n_ant) + ")");
    }
    const uint64_t bytes = rows * row_bytes;
    out->data = (uint8_t*)std::malloc(bytes ? bytes : 1);
    if (!out->data) return TGA_ERR_OUT_OF_MEMORY;
    if (d.layout == 1) {
      r.need(d.addr, bytes);
      std::memcpy(out->data, &r.f[d.addr], bytes);
    } else if (d.layout == 0 && d.compact.size() >= bytes) {
      std::memcpy(out->data, d.compact.data(), bytes);
    } else {
      throw std::runtime_error("HDF5: unsupported storage for `data`");
    }
    out->num_antenna = (uint32_t)rows;
    out->row_bytes = (size_t)row_bytes;
    out->sampling_frequency = fs;
    std::snprintf(out->timestamp, sizeof out->timestamp, "%s", ts.c_str());
    out->config_json = (char*)std::malloc(cfg.size() + 1);
    if (out->config_json) std::memcpy(out->config_json, cfg.c_str(), cfg.size() + 1);
    return TGA_OK;
  } catch (const std::exception& e) {
    tga_observation_free(out);
    std::snprintf(out->error, sizeof out->error, "%s", e.what());
    return TGA_ERR_INVALID_ARG;
  }
}

extern "C" void tga_observation_free(tga_observation* o) {
  if (!o) return;
  std::free(o->data);
  std::free(o->config_json);
  o->data = nullptr;
  o->config_json = nullptr;
}
