// Minimal netCDF-3 classic (CDF-1/CDF-2) reader for the oracle (test infrastructure).
// Reads fixed-size variables of type byte/short/int/float/double from the
// big-endian classic layout described in the public Unidata format spec.
#pragma once
#include <cstdint>
#include <cstring>
#include <fstream>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

namespace nc3 {

struct Var {
  int type = 0;
  std::vector<int> dimids;
  uint64_t begin = 0;
  uint64_t count = 1;
};

class File {
 public:
  explicit File(const std::string& path) : path_(path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("cannot open " + path);
    hdr_.resize(1 << 20);
    f.read(reinterpret_cast<char*>(hdr_.data()), (std::streamsize)hdr_.size());
    hdr_.resize((size_t)f.gcount());
    if (hdr_.size() < 8 || std::memcmp(hdr_.data(), "CDF", 3) != 0) throw std::runtime_error("not netCDF-3: " + path);
    off64_ = hdr_[3] == 2;
    pos_ = 8;
    uint32_t tag = u32(), n = u32();
    for (uint32_t i = 0; i < (tag ? n : 0); i++) {
      std::string nm = name();
      dims_.push_back((uint64_t)u32());
      dimnames_[nm] = (int)dims_.size() - 1;
    }
    read_attrs(&gatts_);
    tag = u32();
    n = u32();
    for (uint32_t i = 0; i < (tag ? n : 0); i++) {
      std::string nm = name();
      Var v;
      uint32_t nd = u32();
      for (uint32_t d = 0; d < nd; d++) {
        v.dimids.push_back((int)u32());
        v.count *= dims_[v.dimids.back()];
      }
      skip_attrs();
      v.type = (int)u32();
      u32();  // vsize
      v.begin = off64_ ? u64() : (uint64_t)u32();
      vars_[nm] = v;
    }
  }
  uint64_t dim(const std::string& n) const {
    auto it = dimnames_.find(n);
    if (it == dimnames_.end()) throw std::runtime_error("missing dimension " + n);
    return dims_[it->second];
  }
  bool has(const std::string& n) const { return vars_.count(n) != 0; }
  // numeric global attribute (first value), as double
  double att(const std::string& n) const {
    auto it = gatts_.find(n);
    if (it == gatts_.end()) throw std::runtime_error("missing global attribute " + n + " in " + path_);
    return it->second;
  }
  std::vector<float> read_float(const std::string& n) const {
    auto d = read_double(n);
    return std::vector<float>(d.begin(), d.end());
  }
  std::vector<double> read_double(const std::string& n) const {
    auto it = vars_.find(n);
    if (it == vars_.end()) throw std::runtime_error("missing variable " + n + " in " + path_);
    const Var& v = it->second;
    static const int sz[] = {0, 1, 1, 2, 4, 4, 8};
    std::vector<uint8_t> raw((size_t)(v.count * sz[v.type]));
    std::ifstream f(path_, std::ios::binary);
    f.seekg((std::streamoff)v.begin);
    f.read(reinterpret_cast<char*>(raw.data()), (std::streamsize)raw.size());
    if (!f) throw std::runtime_error("short read of " + n);
    std::vector<double> out((size_t)v.count);
    for (size_t i = 0; i < out.size(); i++) out[i] = value(v.type, raw.data() + i * sz[v.type]);
    return out;
  }

 private:
  static double value(int type, const uint8_t* p) {
    switch (type) {
      case 1: return (double)(int8_t)p[0];
      case 3: return (double)(int16_t)((p[0] << 8) | p[1]);
      case 4: return (double)(int32_t)be32(p);
      case 5: { uint32_t b = be32(p); float x; std::memcpy(&x, &b, 4); return (double)x; }
      case 6: { uint64_t b = ((uint64_t)be32(p) << 32) | be32(p + 4); double x; std::memcpy(&x, &b, 8); return x; }
      default: throw std::runtime_error("unsupported netCDF type");
    }
  }
  static uint32_t be32(const uint8_t* p) { return ((uint32_t)p[0] << 24) | ((uint32_t)p[1] << 16) | ((uint32_t)p[2] << 8) | p[3]; }
  uint32_t u32() {
    if (pos_ + 4 > hdr_.size()) throw std::runtime_error("truncated netCDF header");
    uint32_t v = be32(&hdr_[pos_]);
    pos_ += 4;
    return v;
  }
  uint64_t u64() { uint64_t a = u32(); return (a << 32) | u32(); }
  std::string name() {
    uint32_t n = u32();
    std::string s(reinterpret_cast<const char*>(&hdr_[pos_]), n);
    pos_ += (n + 3) & ~3u;
    return s;
  }
  void read_attrs(std::map<std::string, double>* into) {
    static const int sz[] = {0, 1, 1, 2, 4, 4, 8};
    uint32_t tag = u32(), n = u32();
    for (uint32_t i = 0; i < (tag ? n : 0); i++) {
      std::string nm = name();
      uint32_t t = u32(), cnt = u32();
      if (t != 2 && cnt > 0 && t <= 6) (*into)[nm] = value((int)t, &hdr_[pos_]);
      pos_ += ((size_t)cnt * sz[t] + 3) & ~(size_t)3;
    }
  }
  void skip_attrs() {
    static const int sz[] = {0, 1, 1, 2, 4, 4, 8};
    uint32_t tag = u32(), n = u32();
    for (uint32_t i = 0; i < (tag ? n : 0); i++) {
      name();
      uint32_t t = u32(), cnt = u32();
      pos_ += ((size_t)cnt * sz[t] + 3) & ~(size_t)3;
    }
  }
  std::string path_;
  std::vector<uint8_t> hdr_;
  size_t pos_ = 0;
  bool off64_ = false;
  std::vector<uint64_t> dims_;
  std::map<std::string, int> dimnames_;
  std::map<std::string, Var> vars_;
  std::map<std::string, double> gatts_;
};

}  // namespace nc3
