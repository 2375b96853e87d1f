// netCDF classic writer, 64-bit offset variant (CDF-2), written from the
// published file-format specification: big-endian header of dimensions,
// global attributes and variables, then the fixed-size variables one after
// another, then the records (one slab of every record variable per record).
// The model's output files (map, his) are written through it: netCDF readers
// (netCDF-C, netCDF4-python, xarray) open CDF-2 files as they open the
// netCDF-4 files the reference writes.
#pragma once
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <algorithm>
#include <vector>

namespace sfg {

class NcWriter {
 public:
  enum Type { BYTE = 1, CHAR = 2, SHORT = 3, INT = 4, FLOAT = 5, DOUBLE = 6 };
  static constexpr int UNLIMITED = 0;

  int def_dim(const std::string& name, long long len) {
    if (defined_) throw std::runtime_error("netCDF: dimension after enddef");
    if (len == UNLIMITED) {
      for (const Dim& d : dims_)
        if (d.len == UNLIMITED) throw std::runtime_error("netCDF: a second unlimited dimension");
    }
    dims_.push_back({name, len});
    return (int)dims_.size() - 1;
  }
  // dims: outermost first (C order); an unlimited dimension must come first
  int def_var(const std::string& name, Type t, const std::vector<int>& dims) {
    if (defined_) throw std::runtime_error("netCDF: variable after enddef");
    for (size_t i = 0; i < dims.size(); i++)
      if (dims_.at(dims[i]).len == UNLIMITED && i != 0)
        throw std::runtime_error("netCDF: the unlimited dimension must be the first of " + name);
    vars_.push_back(Var{name, t, dims, {}, 0, 0, false});
    return (int)vars_.size() - 1;
  }
  void att_text(int var, const std::string& name, const std::string& v) { atts(var).push_back({name, CHAR, bytes_of(v)}); }
  void att_int(int var, const std::string& name, const std::vector<int32_t>& v) { atts(var).push_back({name, INT, be(v)}); }
  void att_float(int var, const std::string& name, float v) { atts(var).push_back({name, FLOAT, be(std::vector<float>{v})}); }
  void att_double(int var, const std::string& name, double v) {
    atts(var).push_back({name, DOUBLE, be(std::vector<double>{v})});
  }
  static constexpr int GLOBAL = -1;

  // Lays the file out, writes the header and fills every fixed-size variable
  // with its _FillValue (or the format's default fill).
  void create(const std::string& path) {
    if (defined_) throw std::runtime_error("netCDF: create twice");
    path_ = path;
    // sizes
    recsize_ = 0;
    for (Var& v : vars_) {
      long long n = 1;
      for (int d : v.dims)
        if (dims_[d].len != UNLIMITED) n *= dims_[d].len;
      v.record = !v.dims.empty() && dims_[v.dims[0]].len == UNLIMITED;
      v.vsize = pad4(n * tsize(v.type));
      if (v.record) recsize_ += v.vsize;
    }
    // header length with placeholder offsets, then the offsets
    std::vector<uint8_t> hdr = header();
    long long off = (long long)hdr.size();
    for (Var& v : vars_)
      if (!v.record) {
        v.begin = off;
        off += v.vsize;
      }
    recstart_ = off;
    for (Var& v : vars_)
      if (v.record) {
        v.begin = off;
        off += v.vsize;
      }
    hdr = header();
    fp_ = std::fopen(path.c_str(), "wb+");
    if (!fp_) throw std::runtime_error("cannot create " + path);
    write_at(0, hdr.data(), hdr.size());
    for (const Var& v : vars_)
      if (!v.record) {
        std::vector<uint8_t> f((size_t)v.vsize);
        fill_pattern(v, f.data(), f.size());
        write_at(v.begin, f.data(), f.size());
      }
    defined_ = true;
    std::fflush(fp_);
  }
  ~NcWriter() { close(); }
  void close() {
    if (fp_) std::fclose(fp_);
    fp_ = nullptr;
  }

  // Whole fixed-size variable, or the hyperslab that starts at element
  // `start` (C order, elements) and holds n values.
  template <class X>
  void put(int var, const X* data, size_t n, size_t start = 0) {
    const Var& v = vars_.at(var);
    if (v.record) throw std::runtime_error("netCDF: put on a record variable " + v.name);
    check_type<X>(v);
    if ((long long)((start + n) * sizeof(X)) > v.vsize) throw std::runtime_error("netCDF: put beyond " + v.name);
    std::vector<uint8_t> b = be_raw(data, n);
    write_at(v.begin + (long long)(start * sizeof(X)), b.data(), b.size());
  }
  // One record's slab of a record variable; the record count grows to rec + 1.
  template <class X>
  void put_record(int var, long long rec, const X* data, size_t n) {
    const Var& v = vars_.at(var);
    if (!v.record) throw std::runtime_error("netCDF: put_record on a fixed variable " + v.name);
    check_type<X>(v);
    if ((long long)(n * sizeof(X)) > v.vsize) throw std::runtime_error("netCDF: record beyond " + v.name);
    std::vector<uint8_t> b = be_raw(data, n);
    write_at(v.begin + rec * recsize_, b.data(), b.size());
    if (rec + 1 > numrecs_) {
      numrecs_ = rec + 1;
      const uint32_t nr = (uint32_t)numrecs_;
      uint8_t w[4] = {(uint8_t)(nr >> 24), (uint8_t)(nr >> 16), (uint8_t)(nr >> 8), (uint8_t)nr};
      write_at(4, w, 4);
    }
  }
  int var_id(const std::string& name) const {
    for (size_t i = 0; i < vars_.size(); i++)
      if (vars_[i].name == name) return (int)i;
    throw std::runtime_error("netCDF: no variable " + name);
  }
  void sync() {
    if (fp_) std::fflush(fp_);
  }
  long long numrecs() const { return numrecs_; }

 private:
  struct Dim {
    std::string name;
    long long len;
  };
  struct Att {
    std::string name;
    Type type;
    std::vector<uint8_t> data;  // big-endian values
  };
  struct Var {
    std::string name;
    Type type;
    std::vector<int> dims;
    std::vector<Att> atts;
    long long vsize, begin;
    bool record;
  };
  std::vector<Dim> dims_;
  std::vector<Att> gatts_;
  std::vector<Var> vars_;
  bool defined_ = false;
  std::string path_;
  FILE* fp_ = nullptr;
  long long recsize_ = 0, recstart_ = 0, numrecs_ = 0;

  std::vector<Att>& atts(int var) { return var == GLOBAL ? gatts_ : vars_.at(var).atts; }
  static long long pad4(long long n) { return (n + 3) & ~3LL; }
  static int tsize(Type t) { return t == BYTE || t == CHAR ? 1 : t == SHORT ? 2 : t == DOUBLE ? 8 : 4; }
  template <class X>
  static void check_type(const Var& v) {
    const int want = std::is_same<X, float>::value ? FLOAT : std::is_same<X, double>::value ? DOUBLE
                     : std::is_same<X, int32_t>::value ? INT : std::is_same<X, char>::value ? CHAR : 0;
    if (want != v.type) throw std::runtime_error("netCDF: wrong value type for " + v.name);
  }
  template <class X>
  static std::vector<uint8_t> be_raw(const X* data, size_t n) {
    std::vector<uint8_t> b(n * sizeof(X));
    for (size_t i = 0; i < n; i++) {
      uint8_t w[sizeof(X)];
      std::memcpy(w, &data[i], sizeof(X));
      for (size_t k = 0; k < sizeof(X); k++) b[i * sizeof(X) + k] = w[sizeof(X) - 1 - k];
    }
    return b;
  }
  template <class X>
  static std::vector<uint8_t> be(const std::vector<X>& v) {
    return be_raw(v.data(), v.size());
  }
  static std::vector<uint8_t> bytes_of(const std::string& s) { return std::vector<uint8_t>(s.begin(), s.end()); }
  static void u32(std::vector<uint8_t>& o, uint32_t x) {
    for (int k = 3; k >= 0; k--) o.push_back((uint8_t)(x >> (8 * k)));
  }
  static void u64(std::vector<uint8_t>& o, uint64_t x) {
    for (int k = 7; k >= 0; k--) o.push_back((uint8_t)(x >> (8 * k)));
  }
  static void name(std::vector<uint8_t>& o, const std::string& s) {
    u32(o, (uint32_t)s.size());
    o.insert(o.end(), s.begin(), s.end());
    while (o.size() % 4) o.push_back(0);
  }
  static void att_list(std::vector<uint8_t>& o, const std::vector<Att>& a) {
    if (a.empty()) {
      u32(o, 0);
      u32(o, 0);
      return;
    }
    u32(o, 0x0C);
    u32(o, (uint32_t)a.size());
    for (const Att& x : a) {
      name(o, x.name);
      u32(o, (uint32_t)x.type);
      u32(o, (uint32_t)(x.data.size() / tsize(x.type)));
      o.insert(o.end(), x.data.begin(), x.data.end());
      while (o.size() % 4) o.push_back(0);
    }
  }
  std::vector<uint8_t> header() const {
    std::vector<uint8_t> o = {'C', 'D', 'F', 2};
    u32(o, (uint32_t)numrecs_);
    if (dims_.empty()) {
      u32(o, 0);
      u32(o, 0);
    } else {
      u32(o, 0x0A);
      u32(o, (uint32_t)dims_.size());
      for (const Dim& d : dims_) {
        name(o, d.name);
        u32(o, (uint32_t)d.len);
      }
    }
    att_list(o, gatts_);
    if (vars_.empty()) {
      u32(o, 0);
      u32(o, 0);
    } else {
      u32(o, 0x0B);
      u32(o, (uint32_t)vars_.size());
      for (const Var& v : vars_) {
        name(o, v.name);
        u32(o, (uint32_t)v.dims.size());
        for (int d : v.dims) u32(o, (uint32_t)d);
        att_list(o, v.atts);
        u32(o, (uint32_t)v.type);
        u32(o, (uint32_t)std::min<long long>(v.vsize, 0xFFFFFFFFLL));
        u64(o, (uint64_t)v.begin);
      }
    }
    return o;
  }
  // _FillValue of the variable when set, else the format's default fill
  void fill_pattern(const Var& v, uint8_t* dst, size_t n) const {
    std::vector<uint8_t> one;
    for (const Att& a : v.atts)
      if (a.name == "_FillValue" && a.type == v.type) one = a.data;
    if (one.empty()) {
      if (v.type == FLOAT) one = be(std::vector<float>{9.9692099683868690e+36f});
      else if (v.type == DOUBLE) one = be(std::vector<double>{9.9692099683868690e+36});
      else if (v.type == INT) one = be(std::vector<int32_t>{-2147483647});
      else one = {0};
    }
    const size_t w = one.size();
    for (size_t i = 0; i + w <= n; i += w) std::memcpy(dst + i, one.data(), w);
  }
  void write_at(long long off, const void* p, size_t n) {
    if (std::fseek(fp_, (long)off, SEEK_SET) != 0 || std::fwrite(p, 1, n, fp_) != n)
      throw std::runtime_error("netCDF: write failed on " + path_);
  }
};

}  // namespace sfg
