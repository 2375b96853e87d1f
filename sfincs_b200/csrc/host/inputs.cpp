#include "inputs.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>

namespace sfg {

InpFile::InpFile(const std::string& path) {
  std::ifstream f(path);
  if (!f) throw std::runtime_error("cannot open " + path);
  std::string raw;
  while (std::getline(f, raw)) {
    std::string line;
    line.reserve(raw.size() + 16);
    for (char ch : raw) {
      if (ch == '\t') {
        do line.push_back(' '); while (line.size() % 8 != 0);
      } else {
        line.push_back(ch);
      }
    }
    const size_t cr = line.find('\r');
    if (cr != std::string::npos) line.resize(cr);
    if (line.empty() || line[0] == '#' || line[0] == '!' || line[0] == '@') continue;
    const size_t eq = line.find('=');
    if (eq == std::string::npos) continue;
    std::string key = line.substr(0, eq);
    key.erase(key.find_last_not_of(' ') + 1);
    std::string val = line.substr(eq + 1);
    const size_t hash = val.find('#');
    if (hash != std::string::npos) val.resize(hash);
    const size_t b = val.find_first_not_of(' ');
    val = b == std::string::npos ? std::string() : val.substr(b);
    val.erase(val.find_last_not_of(' ') + 1);
    if (!kv_.count(key)) kv_[key] = val;  // first occurrence wins
  }
}

float InpFile::real(const std::string& k, float def) const {
  auto it = kv_.find(k);
  return it == kv_.end() ? def : (float)std::strtod(it->second.c_str(), nullptr);
}
int InpFile::integer(const std::string& k, int def) const {
  auto it = kv_.find(k);
  return it == kv_.end() ? def : (int)std::strtol(it->second.c_str(), nullptr, 10);
}
std::string InpFile::str(const std::string& k, const std::string& def) const {
  auto it = kv_.find(k);
  return it == kv_.end() ? def : it->second;
}
bool InpFile::logical(const std::string& k, bool def) const {
  auto it = kv_.find(k);
  if (it == kv_.end()) return def;
  const char c = it->second.empty() ? ' ' : it->second[0];
  return std::strchr("1yYtT", c) != nullptr && c != 0;
}

static long long julian(long long y, long long m, long long d) {  // Fliegel & Van Flandern
  return d - 32075 + 1461 * (y + 4800 + (m - 14) / 12) / 4 + 367 * (m - 2 - ((m - 14) / 12) * 12) / 12 -
         3 * ((y + 4900 + (m - 14) / 12) / 100) / 4;
}

long long seconds_between(const std::string& a, const std::string& b) {
  auto parse = [](const std::string& s, long long* v) {
    if (s.size() < 15) throw std::runtime_error("bad date string '" + s + "' (expected yyyymmdd HHMMSS)");
    const int pos[6] = {0, 4, 6, 9, 11, 13}, len[6] = {4, 2, 2, 2, 2, 2};
    for (int i = 0; i < 6; i++) v[i] = std::strtoll(s.substr(pos[i], len[i]).c_str(), nullptr, 10);
  };
  long long x[6], y[6];
  parse(a, x);
  parse(b, y);
  return (julian(y[0], y[1], y[2]) - julian(x[0], x[1], x[2])) * 86400 + (y[3] * 3600 + y[4] * 60 + y[5]) -
         (x[3] * 3600 + x[4] * 60 + x[5]);
}

std::vector<std::vector<double>> read_table(const std::string& path) {
  std::ifstream f(path);
  if (!f) throw std::runtime_error("cannot open " + path);
  std::vector<std::vector<double>> rows;
  std::string line;
  while (std::getline(f, line)) {
    std::istringstream is(line);
    std::vector<double> r;
    double x;
    while (is >> x) r.push_back(x);
    if (!r.empty()) rows.push_back(std::move(r));
  }
  return rows;
}

template <class X>
std::vector<X> read_binary(const std::string& path, size_t n, size_t offset_bytes) {
  std::ifstream f(path, std::ios::binary);
  if (!f) throw std::runtime_error("cannot open " + path);
  f.seekg((std::streamoff)offset_bytes);
  std::vector<X> v(n);
  f.read(reinterpret_cast<char*>(v.data()), (std::streamsize)(n * sizeof(X)));
  if ((size_t)f.gcount() != n * sizeof(X)) throw std::runtime_error("file too short: " + path);
  return v;
}
template std::vector<int32_t> read_binary<int32_t>(const std::string&, size_t, size_t);
template std::vector<int8_t> read_binary<int8_t>(const std::string&, size_t, size_t);
template std::vector<float> read_binary<float>(const std::string&, size_t, size_t);

// ---------------------------------------------------------------- netCDF-3
namespace {
struct Cursor {
  const std::vector<uint8_t>& b;
  size_t p;
  uint32_t u32() {
    if (p + 4 > b.size()) throw std::runtime_error("truncated netCDF header");
    uint32_t v = (uint32_t)b[p] << 24 | (uint32_t)b[p + 1] << 16 | (uint32_t)b[p + 2] << 8 | b[p + 3];
    p += 4;
    return v;
  }
  std::string name() {
    uint32_t n = u32();
    std::string s(reinterpret_cast<const char*>(&b[p]), n);
    p += (n + 3) & ~3u;
    return s;
  }
};
const int kTypeSize[7] = {0, 1, 1, 2, 4, 4, 8};
}  // namespace

NcFile::NcFile(const std::string& path) : path_(path) {
  std::ifstream f(path, std::ios::binary);
  if (!f) throw std::runtime_error("cannot open " + path);
  std::vector<uint8_t> h(4 << 20);
  f.read(reinterpret_cast<char*>(h.data()), (std::streamsize)h.size());
  h.resize((size_t)f.gcount());
  if (h.size() < 8 || h[0] != 'C' || h[1] != 'D' || h[2] != 'F' || (h[3] != 1 && h[3] != 2))
    throw std::runtime_error("not a netCDF-3 classic file: " + path);
  const bool off64 = h[3] == 2;
  Cursor c{h, 8};
  std::vector<long long> dimlen;
  uint32_t tag = c.u32(), cnt = c.u32();
  for (uint32_t i = 0; i < (tag ? cnt : 0); i++) {
    std::string n = c.name();
    dimlen.push_back(c.u32());
    dims_[n] = dimlen.back();
  }
  auto skip_attrs = [&](std::map<std::string, double>* keep) {
    uint32_t t = c.u32(), k = c.u32();
    for (uint32_t i = 0; i < (t ? k : 0); i++) {
      std::string an = c.name();
      uint32_t ty = c.u32(), ne = c.u32();
      if (ty < 1 || ty > 6) throw std::runtime_error("bad netCDF attribute type in " + path_);
      if (keep && ty != 2 && ne > 0) (*keep)[an] = value_of((int)ty, &c.b[c.p]);
      c.p += ((size_t)ne * kTypeSize[ty] + 3) & ~(size_t)3;
    }
  };
  skip_attrs(&gatts_);
  tag = c.u32();
  cnt = c.u32();
  for (uint32_t i = 0; i < (tag ? cnt : 0); i++) {
    std::string n = c.name();
    uint32_t nd = c.u32();
    uint64_t count = 1;
    for (uint32_t d = 0; d < nd; d++) count *= (uint64_t)dimlen.at(c.u32());
    skip_attrs(nullptr);
    Var v;
    v.type = (int)c.u32();
    c.u32();
    v.begin = off64 ? ((uint64_t)c.u32() << 32 | c.u32()) : c.u32();
    v.count = count;
    vars_[n] = v;
  }
}

long long NcFile::dim(const std::string& n) const {
  auto it = dims_.find(n);
  if (it == dims_.end()) throw std::runtime_error("netCDF dimension '" + n + "' missing in " + path_);
  return it->second;
}

double NcFile::att(const std::string& n) const {
  auto it = gatts_.find(n);
  if (it == gatts_.end()) throw std::runtime_error("netCDF global attribute '" + n + "' missing in " + path_);
  return it->second;
}

std::vector<float> NcFile::floats(const std::string& n) const {
  auto d = doubles(n);
  return std::vector<float>(d.begin(), d.end());
}

std::vector<double> NcFile::doubles(const std::string& n) const {
  auto it = vars_.find(n);
  if (it == vars_.end()) throw std::runtime_error("netCDF variable '" + n + "' missing in " + path_);
  const Var& v = it->second;
  if (v.type < 1 || v.type > 6 || v.type == 2) throw std::runtime_error("unsupported netCDF type for " + n);
  const int sz = kTypeSize[v.type];
  std::vector<uint8_t> raw((size_t)v.count * sz);
  std::ifstream f(path_, std::ios::binary);
  f.seekg((std::streamoff)v.begin);
  f.read(reinterpret_cast<char*>(raw.data()), (std::streamsize)raw.size());
  if ((size_t)f.gcount() != raw.size()) throw std::runtime_error("short read of netCDF variable " + n);
  std::vector<double> out((size_t)v.count);
  for (size_t i = 0; i < out.size(); i++) out[i] = value_of(v.type, &raw[i * sz]);
  return out;
}

// One big-endian value of netCDF type t (byte, short, int, float, double).
double NcFile::value_of(int t, const uint8_t* p) {
  const int sz = kTypeSize[t];
  uint64_t be = 0;
  for (int k = 0; k < sz; k++) be = be << 8 | p[k];
  switch (t) {
    case 1: return (double)(int8_t)be;
    case 3: return (double)(int16_t)be;
    case 4: return (double)(int32_t)be;
    case 5: { uint32_t u = (uint32_t)be; float x; std::memcpy(&x, &u, 4); return (double)x; }
    case 6: { double x; std::memcpy(&x, &be, 8); return x; }
  }
  throw std::runtime_error("unsupported netCDF type");
}

}  // namespace sfg
